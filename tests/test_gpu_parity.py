"""Parity of every stage of the device step with the oracle, through the C
ABI, on seeded clouds.

Bars (stated per test): bit-exact for the sort permutation, the cell lists,
the out-of-stencil list, the table columns / nout and the Verlet update of
(k, delta); relative L2 for the float32 fields against the float64 oracle.
"""
import math

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

vb = load_package()
L = vb._lib


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


class Case:
    """A packed cloud on the xenon geometry: Thomas-Fermi positions, a tenth
    moved outside the fine grid (and a few outside both grids)."""

    def __init__(self, orc, nfine=28, npart=40_000, seed=-1, nbdt=1000):
        self.p = vb.SimulationParameters.for_grid(nfine, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)
        self.meshes = vb.build_meshes(nfine, self.p.ninner, self.p.nouter, 78.0, 235.0)
        self.sm = vb.gaussian_smoothing(self.meshes.fine.axis, nbdt=nbdt)
        self.w = 196.0 / npart
        pos, mom = vb.sample_thomas_fermi(vb.thomas_fermi_profile(), npart, self.w, seed=seed)
        rng = np.random.default_rng(7)
        far = rng.random(npart) < 0.1
        pos[far] *= rng.uniform(2.5, 4.0, (far.sum(), 1))
        pos[:5] = [[300.0, 0, 0], [0, -260.0, 10], [80.0, 1.0, 1.0], [-78.5, 0, 0], [0, 0, 77.9]]
        self.pos, self.mom = pos, mom
        acc_x0 = float(self.meshes.fine.axis.knots[0])
        kn = self.meshes.fine.axis.knots
        self.x0, self.h = acc_x0, float((kn[-1] - kn[0]) / (len(kn) - 1))
        self.k, self.d = vb.pack_positions(pos, self.x0, self.h)
        prev = pos - 0.5 * mom / self.w
        self.pk, self.pd = vb.pack_positions(prev, self.x0, self.h)
        self.jel = vb.Jellium.of(196.0)
        self.orc = orc
        self.O = orc.DeviceSemanticsStep(self.meshes, self.sm, self.w, self.jel, 0.5, 100.0,
                                         vb.xenon_projectile(x0=-10.0, impact=20.0))


@pytest.fixture(scope="module")
def case(orc, cuda_device):
    return Case(orc)


@pytest.fixture(scope="module")
def acc(case):
    a = vb.DeviceAccelerator(case.meshes, case.sm, case.p.nparticles, case.w)
    yield a
    a.close()


def sorted_reference(case):
    perm, occ, bnd, keys = case.orc.cellsort(case.k, case.meshes.fine.axis.nknots)
    ks = np.ascontiguousarray(case.k[:, perm])
    out = case.orc.outside(ks, case.meshes.fine.n)
    return perm, occ, bnd, out


def test_sort_is_the_stable_cellsort(case, acc):
    acc.upload(case.k, case.d, case.pk, case.pd)
    nocc, outc = acc.sort()
    perm, occ, bnd, out = acc.sort_products()
    rperm, rocc, rbnd, rout = sorted_reference(case)
    assert nocc == len(rocc) and outc == len(rout)
    assert np.array_equal(perm, rperm)          # bit-exact permutation
    assert np.array_equal(occ, rocc)
    assert np.array_equal(bnd, rbnd)
    assert np.array_equal(out, rout)
    k, d, pk, pdl = acc.download()              # the records moved with it
    assert np.array_equal(k, case.k[:, rperm]) and np.array_equal(d, case.d[:, rperm])
    assert np.array_equal(pk, case.pk[:, rperm]) and np.array_equal(pdl, case.pd[:, rperm])
    # a second sort of a sorted cloud is the identity
    acc.sort()
    perm2, *_ = acc.sort_products()
    assert np.array_equal(perm2, np.arange(case.p.nparticles))


def test_sort_of_a_shuffled_cloud_with_extreme_knots(case):
    """Random order (the first step's case) and knots far outside [1, nk]."""
    rng = np.random.default_rng(11)
    n = 30_001
    k = rng.integers(-400, 500, (3, n)).astype(np.int32)
    k[:, : n // 2] = rng.integers(1, 30, (3, n // 2))
    d = rng.uniform(-1, 1, (3, n)).astype(np.float32)
    a = vb.DeviceAccelerator(case.meshes, case.sm, n, 196.0 / n)
    try:
        a.upload(k, d, k, d)
        a.sort()
        perm, occ, bnd, out = a.sort_products()
        rperm, rocc, rbnd, _ = case.orc.cellsort(k, case.meshes.fine.axis.nknots)
        assert np.array_equal(perm, rperm) and np.array_equal(occ, rocc) and np.array_equal(bnd, rbnd)
        assert np.array_equal(out, case.orc.outside(np.ascontiguousarray(k[:, rperm]), case.meshes.fine.n))
    finally:
        a.close()


def oracle_sorted(case):
    perm, occ, bnd, _ = sorted_reference(case)
    O = case.O
    O.occ, O.bnd = occ, bnd
    return (np.ascontiguousarray(a[:, perm]) for a in (case.k, case.d, case.pk, case.pd))


def test_fine_deposit(case, acc):
    acc.upload(case.k, case.d, case.pk, case.pd)
    acc.sort()
    nout, q = acc.deposit_smoothed(case.w)
    rho = acc.grid(L.VLB_GRID_RHO_FINE)
    k, d, _, _ = oracle_sorted(case)
    c = case.O.c
    cols, rnout = case.orc.columns(k, d, c["x0f"], c["hf"], c["lo"], c["hi"], c["spacing"], c["nbdt"])
    assert nout == rnout                                   # exact
    O = case.O
    qr = case.orc.lib().orc_deposit_sorted(O.F.ref(), O.S.ref(), k.shape[1], case.orc.pi(np.ascontiguousarray(cols)),
                                           case.orc.pi(O.occ), case.orc.pi(O.bnd), len(O.occ), rnout, case.w,
                                           case.orc.pd(O.rhof))
    assert rel_l2(rho, O.rhof) < 2e-6                      # float32 sums vs float64
    assert abs(q - qr) < 1e-5 * abs(qr)
    tc = case.orc.lib().orc_total_charge(O.F.ref(), case.orc.pd(rho.astype(np.float64).ravel()))
    assert abs(tc - (case.p.nparticles - nout) * case.w) < 1e-4 * 196


def test_fixed_point_deposit_is_bit_identical_across_runs(case, acc):
    acc.upload(case.k, case.d, case.pk, case.pd)
    acc.sort()
    acc.deposit_smoothed(case.w, fixed_point=True)
    r1 = acc.grid(L.VLB_GRID_RHO_FINE)
    acc.deposit_smoothed(case.w, fixed_point=True)
    r2 = acc.grid(L.VLB_GRID_RHO_FINE)
    assert np.array_equal(r1.view(np.uint32), r2.view(np.uint32))
    acc.deposit_smoothed(case.w)
    rf = acc.grid(L.VLB_GRID_RHO_FINE)
    assert rel_l2(r1, rf) < 2e-6


def test_coarse_cic_deposit(case, acc):
    acc.upload(case.k, case.d, case.pk, case.pd)
    acc.sort()
    acc.deposit_cic(case.w)
    rho = acc.grid(L.VLB_GRID_RHO_COARSE)
    k, d, _, _ = oracle_sorted(case)
    O, c = case.O, case.O.c
    case.orc.lib().orc_deposit_cic_device(O.Cl.ref(), k.shape[1], case.orc.pi(k), case.orc.pf(d), c["x0f"], c["hf"],
                                          case.w, case.orc.pd(O.rhoc))
    assert rel_l2(rho, O.rhoc) < 2e-6


def _set_rho_from_oracle(case, acc):
    O = case.O
    acc.set_grid(L.VLB_GRID_RHO_FINE, O.rhof.astype(np.float32))
    acc.set_grid(L.VLB_GRID_RHO_COARSE, O.rhoc.astype(np.float32))
    rf = acc.grid(L.VLB_GRID_RHO_FINE).astype(np.float64).ravel()
    rc = acc.grid(L.VLB_GRID_RHO_COARSE).astype(np.float64).ravel()
    return rf, rc


def test_nested_poisson(case, acc):
    O = case.O
    k, d, _, _ = oracle_sorted(case)
    O.forces(k, d)                      # fills the oracle's densities
    rf, rc = _set_rho_from_oracle(case, acc)
    acc.poisson()
    phf, phc = np.zeros_like(rf), np.zeros_like(rc)
    case.orc.lib().orc_poisson(O.F.ref(), O.Cl.ref(), case.orc.pd(rf), case.orc.pd(rc), case.orc.pd(phf),
                               case.orc.pd(phc))
    assert rel_l2(acc.grid(L.VLB_GRID_PHI_COARSE), phc) < 2e-5
    assert rel_l2(acc.grid(L.VLB_GRID_PHI_FINE), phf) < 2e-5


def test_coefficients_and_mean_field(case, acc):
    O = case.O
    k, d, _, _ = oracle_sorted(case)
    O.forces(k, d)
    rf, rc = _set_rho_from_oracle(case, acc)
    for lev, wphi, wcs, rho in ((0, L.VLB_GRID_PHI_FINE, L.VLB_GRID_CSOL_FINE, rf),
                                (1, L.VLB_GRID_PHI_COARSE, L.VLB_GRID_CSOL_COARSE, rc)):
        Lv = O.F if lev == 0 else O.Cl
        phi = np.asarray(O.phif if lev == 0 else O.phic)
        acc.set_grid(wphi, phi.astype(np.float32))
        phi32 = acc.grid(wphi).astype(np.float64).ravel()
        acc.spline_coefficients(lev)
        c = np.zeros_like(phi32)
        case.orc.lib().orc_spline_coefficients(Lv.ref(), case.orc.pd(phi32), case.orc.pd(c))
        assert rel_l2(acc.grid(wcs), c) < 2e-5
        acc.effective_potential(lev, case.jel)
        case.orc.lib().orc_effective_potential(Lv.ref(), case.orc.pd(c), case.orc.pd(rho), case.jel.nions,
                                               case.jel.radius)
        assert rel_l2(acc.grid(wcs), c) < 2e-5


@pytest.mark.parametrize("softening", [L.VLB_SOFTENING_DEVICE, L.VLB_SOFTENING_BALL], ids=["device-gauss", "cpu-ball"])
@pytest.mark.parametrize("tensor_cores", [1, 0], ids=["tcgen05-3xtf32", "fp32-fma"])
def test_forces_with_projectile(case, acc, tensor_cores, softening):
    """Both forms of the gather (sums over y as 3xTF32 MMAs, or FP32 FMAs)
    against the float64 oracle, same bars, with the projectile softened as
    the reference's device path does (Gaussian in the stencil, ball in the
    tail) and as its CPU path does (the ball everywhere)."""
    O = case.O
    O.proj.softening_mode = softening
    O.softening = softening
    try:
        k, d, pk, pdl = oracle_sorted(case)
        O.forces(k, d)
        acc.set_tuning(field_tensor_cores=tensor_cores)
        acc.upload(case.k, case.d, case.pk, case.pd)
        acc.sort()
        acc.set_grid(L.VLB_GRID_CSOL_FINE, O.csolf.astype(np.float32))
        acc.set_grid(L.VLB_GRID_CSOL_COARSE, O.csolc.astype(np.float32))
        # the oracle reads the same float32-rounded coefficients
        O.csolf = acc.grid(L.VLB_GRID_CSOL_FINE).astype(np.float64).ravel()
        O.csolc = acc.grid(L.VLB_GRID_CSOL_COARSE).astype(np.float64).ravel()
        N = k.shape[1]
        force = np.empty((3, N))
        red = np.zeros(4)
        pr = case.orc.projectile_struct(O.proj, softening=softening)
        outc = case.orc.lib().orc_forces_device(O.F.ref(), O.Cl.ref(), O.S.ref(), N, case.orc.pi(k), case.orc.pf(d),
                                                case.orc.pi(O.occ), case.orc.pi(O.bnd), len(O.occ), case.orc.pd(O.csolf),
                                                case.orc.pd(O.csolc), case.w, O.c["x0"], O.c["h"],
                                                __import__("ctypes").byref(pr), case.orc.pd(force), case.orc.pd(red))
        gred, goutc = acc.forces(O.proj)
        f = acc.force()
        assert goutc == outc
        out = case.orc.outside(k, case.meshes.fine.n)
        inside = np.ones(N, bool)
        inside[out] = False
        acc.set_tuning(field_tensor_cores=1)
        e_in = rel_l2(f[:, inside], force[:, inside])
        print(f"\n[gather, tensor cores {tensor_cores}, softening {softening}] rel L2 vs the oracle: {e_in:.2e}")
        assert e_in < 2e-5
        assert rel_l2(f[:, out], force[:, out]) < 1e-5
        assert np.all(np.isfinite(f))
        assert rel_l2(gred[:3], red[:3]) < 1e-4 and abs(gred[3] - red[3]) < 1e-4 * abs(red[3])
    finally:
        O.proj.softening_mode = L.VLB_SOFTENING_DEVICE
        O.softening = L.VLB_SOFTENING_DEVICE
        acc.set_tuning(field_tensor_cores=1)


def test_verlet_push_is_bit_exact(case, acc):
    rng = np.random.default_rng(2)
    acc.upload(case.k, case.d, case.pk, case.pd)
    f = (rng.standard_normal((3, case.p.nparticles)) * 1e-3).astype(np.float32)
    acc.set_force(f)
    diag = acc.push(0.5, 20.0)
    k, d, pk, pdl = acc.download()
    case.O.rcmax = 20.0
    rk, rd, rpk, rpd, rdiag = case.O.push(case.k.copy(), case.d.copy(), case.pk.copy(), case.pd.copy(), f)
    case.O.rcmax = 100.0
    assert np.array_equal(k, rk) and np.array_equal(d.view(np.uint32), rd.view(np.uint32))
    assert np.array_equal(pk, case.k) and np.array_equal(pdl, case.d)
    assert abs(diag["kinetic"] - rdiag[0]) < 1e-5 * rdiag[0]
    assert abs(diag["escaped"] - rdiag[1]) <= 1e-5 * rdiag[0]
    assert rdiag[1] > 0  # some particles sit beyond rcmax = 20


def test_enclosed_charge(case, acc):
    acc.upload(case.k, case.d, case.pk, case.pd)
    P = np.array([1.0, -2.0, 0.5])
    q = acc.enclosed_charge(P, 8.0)
    old = case.O.proj.position
    case.O.proj.position = P
    rq = case.O.enclosed_charge(case.k, case.d, 8.0)
    case.O.proj.position = old
    assert abs(q - rq) < 1e-12


def test_state_errors_are_status_codes(case):
    a = vb.DeviceAccelerator(case.meshes, case.sm, 100, 1.96)
    try:
        with pytest.raises(L.VlbError) as e:
            a.forces(None)
        assert e.value.code == L.VLB_ERR_STATE
        with pytest.raises(L.VlbError) as e:
            a.grid(17)
        assert e.value.code == L.VLB_ERR_ARG
        with pytest.raises(L.VlbError):
            a.deposit_smoothed(1.0)
    finally:
        a.close()
