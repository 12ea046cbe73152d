"""Parity at the headline sizes: the 130^3 grids (nfine = 64) with 8e6
particles for the sort and 2e6 for the per-stage fields, and one 8e7 cloud
(about 11 GB of device state).

The sort is held bit-exact to the stable cellsort! (src/sorting.jl:163-204)
at 8e6 particles over the 274,625 cells of the 130^3 grid, both from a
random order (a first step) and from the nearly sorted order a step leaves
(the previous sort's order, with a seventh of the particles moved to a
neighbouring cell).  The fine and coarse deposits and the forces (both
gather forms) meet the same bars as the small-grid tests: relative L2 2e-6
for the deposits and 2e-5 for the forces against the float64 oracle.  At
8e7: the sort against cellsort!, two fixed-point steps bit-identical from
the same state, and the forces of a sample of the occupied cells against the
oracle on the step's own coefficients."""
import ctypes as C

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


class Cloud:
    """A packed Thomas-Fermi cloud on the 130^3 xenon geometry, a tenth of it
    moved outside the fine grid (a few outside both grids)."""

    def __init__(self, npart, nfine=64, seed=-1):
        self.p = vb.SimulationParameters.for_grid(nfine, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)
        self.meshes = vb.build_meshes(nfine, self.p.ninner, self.p.nouter, 78.0, 235.0)
        self.sm = vb.gaussian_smoothing(self.meshes.fine.axis)
        self.w = 196.0 / npart
        pos, mom = vb.sample_thomas_fermi(vb.thomas_fermi_profile(), npart, self.w, seed=seed)
        rng = np.random.default_rng(7)
        far = rng.random(npart) < 0.1
        pos[far] *= rng.uniform(2.5, 4.0, (far.sum(), 1))
        kn = self.meshes.fine.axis.knots
        self.x0, self.h = float(kn[0]), float((kn[-1] - kn[0]) / (len(kn) - 1))
        self.k, self.d = vb.pack_positions(pos, self.x0, self.h)
        self.pk, self.pd = vb.pack_positions(pos - 0.5 * mom / self.w, self.x0, self.h)
        del pos, mom
        self.nk = self.meshes.fine.axis.nknots
        self.n = self.meshes.fine.n


def check_sort(orc, acc, c, k, d, pk, pd):
    acc.upload(k, d, pk, pd)
    nocc, outc = acc.sort()
    perm, occ, bnd, out = acc.sort_products()
    rperm, rocc, rbnd, _ = orc.cellsort(k, c.nk)
    assert nocc == len(rocc)
    assert np.array_equal(perm, rperm)          # bit-exact permutation
    assert np.array_equal(occ, rocc) and np.array_equal(bnd, rbnd)
    ks = np.ascontiguousarray(k[:, rperm])
    assert np.array_equal(out, orc.outside(ks, c.n)) and outc == len(out)
    gk, gd, gpk, gpd = acc.download()
    assert np.array_equal(gk, ks) and np.array_equal(gd.view(np.uint32), d[:, rperm].view(np.uint32))
    assert np.array_equal(gpk, pk[:, rperm]) and np.array_equal(gpd.view(np.uint32), pd[:, rperm].view(np.uint32))
    return gk, gd, gpk, gpd


@pytest.fixture(scope="module")
def cloud8(cuda_device):
    return Cloud(8_000_000)


def test_sort_at_8e6_on_130_cubed_is_the_stable_cellsort(orc, cloud8):
    c = cloud8
    acc = vb.DeviceAccelerator(c.meshes, c.sm, c.p.nparticles, c.w)
    try:
        # the sampled (random) order
        k, d, pk, pd = check_sort(orc, acc, c, c.k, c.d, c.pk, c.pd)
        # the order a step leaves: sorted, then a seventh of the particles
        # one knot away on one axis (movers cross into neighbouring cells)
        rng = np.random.default_rng(3)
        mv = rng.random(k.shape[1]) < 1 / 7
        ax = rng.integers(0, 3, k.shape[1])
        step = rng.choice(np.array([-1, 1], np.int32), k.shape[1])
        k2 = k.copy()
        for a in range(3):
            sel = mv & (ax == a)
            k2[a, sel] += step[sel]
        check_sort(orc, acc, c, k2, d, pk, pd)
    finally:
        acc.close()


@pytest.fixture(scope="module")
def stage2(orc, cuda_device):
    """2e6 particles on 130^3: the device context and the oracle's step on
    the same sorted cloud."""
    c = Cloud(2_000_000)
    acc = vb.DeviceAccelerator(c.meshes, c.sm, c.p.nparticles, c.w)
    jel = vb.Jellium.of(196.0)
    O = orc.DeviceSemanticsStep(c.meshes, c.sm, c.w, jel, 0.5, 100.0, vb.xenon_projectile(x0=-10.0, impact=20.0))
    k, d, pk, pd = O.sort(c.k, c.d, c.pk, c.pd)
    yield c, acc, O, (k, d, pk, pd), jel
    acc.close()


def test_fine_and_coarse_deposits_at_2e6_on_130_cubed(orc, stage2):
    c, acc, O, (k, d, pk, pd), _ = stage2
    acc.upload(c.k, c.d, c.pk, c.pd)
    acc.sort()
    nout, q = acc.deposit_smoothed(c.w)
    rho = acc.grid(L.VLB_GRID_RHO_FINE)
    cc = O.c
    cols, rnout = orc.columns(k, d, cc["x0f"], cc["hf"], cc["lo"], cc["hi"], cc["spacing"], cc["nbdt"])
    assert nout == rnout
    qr = orc.lib().orc_deposit_sorted(O.F.ref(), O.S.ref(), k.shape[1], orc.pi(np.ascontiguousarray(cols)),
                                      orc.pi(O.occ), orc.pi(O.bnd), len(O.occ), rnout, c.w, orc.pd(O.rhof))
    e_f = rel_l2(rho, O.rhof)
    assert e_f < 2e-6 and abs(q - qr) < 1e-5 * abs(qr)
    acc.deposit_cic(c.w)
    orc.lib().orc_deposit_cic_device(O.Cl.ref(), k.shape[1], orc.pi(k), orc.pf(d), cc["x0f"], cc["hf"], c.w,
                                     orc.pd(O.rhoc))
    e_c = rel_l2(acc.grid(L.VLB_GRID_RHO_COARSE), O.rhoc)
    print(f"\n[2e6, 130^3] fine deposit rel L2 {e_f:.2e}, coarse {e_c:.2e}")
    assert e_c < 2e-6
    # the fixed-point deposit gives the same density
    acc.deposit_smoothed(c.w, fixed_point=True)
    assert rel_l2(acc.grid(L.VLB_GRID_RHO_FINE), O.rhof) < 2e-6


@pytest.mark.parametrize("tensor_cores", [1, 0], ids=["tcgen05-3xtf32", "fp32-fma"])
def test_forces_at_2e6_on_130_cubed(orc, stage2, tensor_cores):
    c, acc, O, (k, d, pk, pd), _ = stage2
    if not hasattr(O, "csolf_done"):
        O.forces(k, d)
        O.csolf_done = True
    acc.set_tuning(field_tensor_cores=tensor_cores)
    try:
        acc.upload(c.k, c.d, c.pk, c.pd)
        acc.sort()
        acc.set_grid(L.VLB_GRID_CSOL_FINE, O.csolf.astype(np.float32))
        acc.set_grid(L.VLB_GRID_CSOL_COARSE, O.csolc.astype(np.float32))
        csf = acc.grid(L.VLB_GRID_CSOL_FINE).astype(np.float64).ravel()
        csc = acc.grid(L.VLB_GRID_CSOL_COARSE).astype(np.float64).ravel()
        N = k.shape[1]
        force, red = np.empty((3, N)), np.zeros(4)
        pr = orc.projectile_struct(O.proj)
        outc = orc.lib().orc_forces_device(O.F.ref(), O.Cl.ref(), O.S.ref(), N, orc.pi(k), orc.pf(d),
                                           orc.pi(O.occ), orc.pi(O.bnd), len(O.occ), orc.pd(csf), orc.pd(csc), c.w,
                                           O.c["x0"], O.c["h"], C.byref(pr), orc.pd(force), orc.pd(red))
        gred, goutc = acc.forces(O.proj)
        f = acc.force()
        assert goutc == outc
        out = orc.outside(k, c.n)
        inside = np.ones(N, bool)
        inside[out] = False
        e_in = rel_l2(f[:, inside], force[:, inside])
        print(f"\n[2e6, 130^3, tensor cores {tensor_cores}] forces rel L2 {e_in:.2e}")
        assert e_in < 2e-5
        assert rel_l2(f[:, out], force[:, out]) < 1e-5
        assert rel_l2(gred[:3], red[:3]) < 1e-4 and abs(gred[3] - red[3]) < 1e-4 * abs(red[3])
    finally:
        acc.set_tuning(field_tensor_cores=1)


def test_8e7_sort_fixed_point_and_forces(orc, cuda_device):
    """Config 3's size: the sort against cellsort!, two fixed-point steps
    run twice from the same state bit for bit, and the forces of every
    40th occupied cell against the oracle on the step's coefficients."""
    npart = 80_000_000
    p = vb.SimulationParameters.for_grid(64, rcluster=78.0, rbox=235.0, nparticles=npart, dt=0.5)
    proj = vb.xenon_projectile(x0=-20.0, impact=10.0)
    sim = vb.Simulation(p, vb.thomas_fermi_profile(), projectile=proj, fixed_point=True, use_graph=True,
                        precision=L.VLB_POISSON_3XTF32)
    acc = sim.accelerator
    try:
        snap = sim.snapshot()
        runs = []
        for _ in range(2):
            sim.restore(snap)
            ds = [sim.step(), sim.step()]
            runs.append((ds, sim.projectile.position.copy(), acc.download()))
        (d1, P1, c1), (d2, P2, c2) = runs
        for a, b in zip(d1, d2):
            assert a.status == 0 and b.status == 0
            assert (a.kinetic, a.enclosed_charge, a.outcount, a.nout) == (b.kinetic, b.enclosed_charge, b.outcount,
                                                                          b.nout)
        assert np.array_equal(P1, P2)
        for x, y in zip(c1, c2):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
        del c2, runs
        # the sort of the stepped cloud (nearly sorted) against cellsort!
        k, d, pk, pd = c1
        del c1
        acc.upload(k, d, pk, pd)
        nocc, outc = acc.sort()
        perm, occ, bnd, out = acc.sort_products()
        rperm, rocc, rbnd, _ = orc.cellsort(k, sim.meshes.fine.axis.nknots)
        assert np.array_equal(perm, rperm) and np.array_equal(occ, rocc) and np.array_equal(bnd, rbnd)
        del perm, rperm
        # forces of a sample of the cells, on the coefficients of a
        # forces-only step (its own density, Poisson solve and mean field)
        acc.upload(k, d, pk, pd)
        r = acc.fused_step(sim.projectile, sim._params(advance=False, push=False, capture=0.0))
        assert r.status == 0
        acc.sort()  # the identity on the step's sorted cloud: its lists, the forces still in slot order
        ks, ds, _, _ = acc.download()
        _, occ, bnd, _ = acc.sort_products()
        f = acc.force()
        csf = acc.grid(L.VLB_GRID_CSOL_FINE).astype(np.float64).ravel()
        csc = acc.grid(L.VLB_GRID_CSOL_COARSE).astype(np.float64).ravel()
        sel = np.arange(0, len(occ), 40)
        counts = bnd[sel + 1] - bnd[sel]
        idx = np.concatenate([np.arange(bnd[g], bnd[g + 1]) for g in sel])
        sub_k = np.ascontiguousarray(ks[:, idx])
        sub_d = np.ascontiguousarray(ds[:, idx])
        sub_b = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
        sub_o = np.ascontiguousarray(occ[sel])
        jel = vb.Jellium.of(196.0)
        O = orc.DeviceSemanticsStep(sim.meshes, sim.smoothing, sim.weight, jel, 0.5, p.rcmax, sim.projectile)
        n_sub = sub_k.shape[1]
        force, red = np.empty((3, n_sub)), np.zeros(4)
        pr = orc.projectile_struct(sim.projectile)
        orc.lib().orc_forces_device(O.F.ref(), O.Cl.ref(), O.S.ref(), n_sub, orc.pi(sub_k), orc.pf(sub_d),
                                    orc.pi(sub_o), orc.pi(sub_b), len(sub_o), orc.pd(csf), orc.pd(csc), sim.weight,
                                    O.c["x0"], O.c["h"], C.byref(pr), orc.pd(force), orc.pd(red))
        e = rel_l2(f[:, idx], force)
        print(f"\n[8e7, 130^3] forces of {len(sel)} cells ({n_sub} particles): rel L2 {e:.2e}")
        assert e < 2e-5
    finally:
        acc.close()
