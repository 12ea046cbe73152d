"""The oracle pinned against the reference's known-answer tests
(test/runtests.jl).  No Fortran dumps ship with the reference and Julia is
absent here, so these analytic identities, invariants and tolerances -- the
reference's own -- are what pin the float64 restatement."""
import ctypes as C
import math

import numpy as np
import pytest

from conftest import load_package

vb = load_package()
T = vb.tables


@pytest.fixture(scope="module")
def O(orc):
    return orc


def level(O, m):
    return O.Level(m)


def _laplacian(O, lev, phi_in):
    """sum_d D_d phi along each axis (src/mesh.jl:460-467), interior operator."""
    D = lev.mesh.laplacian[1:-1, 1:-1]
    ni = D.shape[0]
    x = phi_in.reshape(ni, ni, ni)  # [k][j][i]
    out = np.einsum("ai,kji->kja", D, x) + np.einsum("aj,kji->kai", D, x) + np.einsum("ak,kji->aji", D, x)
    return out.ravel()


def test_ran2_python_restatement_matches_library(O, vb):
    from oracle.ran2 import Ran2
    r = Ran2(-1)
    py = np.array([r.next() for _ in range(500)], dtype=np.float32)
    assert np.array_equal(py, vb.ran2(-1, 500))
    assert not np.array_equal(vb.ran2(-7, 50), vb.ran2(-1, 50))
    assert not np.array_equal(vb.ran2(-1, 100), vb.ran2(-1, 100, consistent=True))
    for cons in (False, True):  # test/runtests.jl:44-50
        v = vb.ran2(-3, 100_000, consistent=cons).astype(np.float64)
        assert abs(v.mean() - 0.5) < 0.01
        assert abs(v.var() - 1 / 12) < 0.002
        assert np.all((v >= 0) & (v < 1))


def test_sampling_python_restatement_matches_library(vb):
    from oracle.ran2 import sample_thomas_fermi
    prof = vb.thomas_fermi_profile()
    pos, mom = vb.sample_thomas_fermi(prof, 300, 196 / 300)
    p2, m2 = sample_thomas_fermi(prof.quantiles, prof.density, prof.rmax, 300, 196 / 300)
    assert np.array_equal(pos, p2) and np.array_equal(mom, m2)


def test_oracle_sampler_matches_the_python_restatement_and_the_library(O, vb):
    """The oracle's own C++ draw (the CPU baseline's, which loads nothing of
    the product) against the pure-Python ran2 restatement and the library's
    sampler, bit for bit."""
    from oracle.ran2 import sample_thomas_fermi
    prof = vb.thomas_fermi_profile()
    pos, mom = O.sample_thomas_fermi(prof, 300, 196 / 300)
    p2, m2 = sample_thomas_fermi(prof.quantiles, prof.density, prof.rmax, 300, 196 / 300)
    assert np.array_equal(pos, p2) and np.array_equal(mom, m2)
    for seed, cons in ((-1, False), (-5, True)):
        a = O.sample_thomas_fermi(prof, 50_000, 196 / 50_000, seed=seed, consistent=cons)
        b = vb.sample_thomas_fermi(prof, 50_000, 196 / 50_000, seed=seed, consistent=cons)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_uniform_sphere_sampling():
    # test/runtests.jl:979-1026 on the cluster-size ball
    prof = vb.uniform_sphere_profile()
    R = prof.rmax
    pos, mom = vb.sample_thomas_fermi(prof, 20_000, 196 / 20_000)
    r = np.linalg.norm(pos, axis=1)
    assert r.max() <= R + 1e-9
    assert abs(np.mean((r / R) ** 3) - 0.5) < 0.02
    assert np.all(np.abs(pos.mean(axis=0)) < 0.3)


def test_cellsort_invariants(O, vb):
    # test/runtests.jl:745-778 (with the uniform axis h = 2.5, 9 knots)
    n = 500
    rng = vb.ran2(-1, 3 * n).astype(np.float64).reshape(n, 3)
    pos = 20 * (rng - 0.5)
    k, _ = vb.pack_positions(pos, -10.0, 2.5)
    perm, occ, bnd, keys = O.cellsort(k, 9)
    assert np.array_equal(np.sort(perm), np.arange(n))
    cells = keys[perm]
    assert np.all(np.diff(cells) >= 0)
    assert bnd[0] == 0 and bnd[-1] == n and len(bnd) == len(occ) + 1
    for g in range(len(occ)):
        assert np.all(cells[bnd[g]:bnd[g + 1]] == occ[g])
    assert np.all(np.diff(occ) > 0) and np.all(np.diff(bnd) > 0)
    # stability: within a cell the original order is kept
    for g in range(len(occ)):
        assert np.all(np.diff(perm[bnd[g]:bnd[g + 1]]) > 0)
    perm2, occ2, bnd2, _ = O.cellsort(k, 9)
    assert np.array_equal(perm, perm2) and np.array_equal(occ, occ2) and np.array_equal(bnd, bnd2)


def test_cic_charge_conservation(O):
    # test/runtests.jl:283-337
    ax = T.uniform_axis(-50.0, 50.0, 28)
    m = T.SplineMesh(ax)
    lev = O.Level(m)
    rng = np.random.default_rng(1234)
    pos = 8.0 * rng.standard_normal((50_000, 3))
    rho = np.zeros(m.n ** 3)
    nout = O.lib().orc_deposit_cic_host(lev.ref(), len(pos), O.pd(pos), 196 / 50_000, O.pd(rho))
    assert nout == 0
    q = O.lib().orc_total_charge(lev.ref(), O.pd(rho))
    assert abs(q - 196.0) < 1e-12 * 196
    outside = np.array([[200.0, 0, 0], [0, -300.0, 0]])
    rho2 = np.zeros(m.n ** 3)
    assert O.lib().orc_deposit_cic_host(lev.ref(), 2, O.pd(outside), 1.0, O.pd(rho2)) == 2
    assert np.all(rho2 == 0)
    # S^-1 then S gives back the identity
    c = np.zeros_like(rho)
    O.lib().orc_spline_coefficients(lev.ref(), O.pd(rho), O.pd(c))
    back = c
    for _ in range(3):
        back = O.mode_product(m.cm.S, back)
    assert np.linalg.norm(back - rho) / np.linalg.norm(rho) < 1e-10


def test_smoothed_deposit_conservation_support_and_edges(O):
    # test/runtests.jl:780-847
    ax = T.uniform_axis(-50.0, 50.0, 28)
    m = T.SplineMesh(ax)
    sm = T.gaussian_smoothing(ax, nbdt=100, quadrature=100)
    lev, S = O.Level(m), O.Smoothing(sm)
    rng = np.random.default_rng(99)
    pos = 8.0 * rng.standard_normal((5000, 3))
    rho = np.zeros(m.n ** 3)
    assert O.lib().orc_deposit_smoothed_host(lev.ref(), S.ref(), 5000, O.pd(pos), 196 / 5000, O.pd(rho)) == 0
    assert abs(O.lib().orc_total_charge(lev.ref(), O.pd(rho)) - 196) < 1e-12 * 196
    one = np.array([[1.3, -0.7, 2.1]])
    r1, rt = np.zeros(m.n ** 3), np.zeros(m.n ** 3)
    O.lib().orc_deposit_smoothed_host(lev.ref(), S.ref(), 1, O.pd(one), 1.0, O.pd(r1))
    O.lib().orc_deposit_cic_host(lev.ref(), 1, O.pd(one), 1.0, O.pd(rt))
    assert np.count_nonzero(r1) == 512 and np.count_nonzero(rt) == 8
    h = ax.knots[1] - ax.knots[0]
    edge = np.array([[ax.knots[0] + h / 4, 0, 0], [0, ax.knots[-1] - h / 4, 0]])
    both = np.ascontiguousarray(np.vstack([edge, pos]))
    rb = np.zeros(m.n ** 3)
    assert O.lib().orc_deposit_smoothed_host(lev.ref(), S.ref(), len(both), O.pd(both), 196 / 5000, O.pd(rb)) == 2


def test_multipole_of_centred_gaussian(O):
    # test/runtests.jl:339-366
    ax = T.uniform_axis(-20.0, 20.0, 16)
    m = T.SplineMesh(ax)
    lev = O.Level(m)
    g = ax.colloc
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    rho = np.exp(-(x ** 2 + y ** 2 + z ** 2) / (2 * 9.0)).ravel()
    rho *= 10.0 / O.lib().orc_total_charge(lev.ref(), O.pd(rho))
    out = np.zeros(10)
    O.lib().orc_multipole(lev.ref(), O.pd(rho), O.pd(out))
    assert abs(out[0] - 10) < 1e-10 * 10
    assert np.all(np.abs(out[1:4]) < 1e-8)
    assert np.all(np.abs(out[4:]) < 1e-6)
    sh = np.exp(-((x - 4) ** 2 + y ** 2 + z ** 2) / 18.0).ravel()
    O.lib().orc_multipole(lev.ref(), O.pd(sh), O.pd(out))
    assert abs(out[1] - 4) < 1e-6 * 4 and abs(out[2]) < 1e-8


def test_poisson_convergence_and_inverse(O):
    # test/runtests.jl:249-281 (tensor solver: fourth order, err < 1e-6 at n=16)
    L_ = 2.0

    def err(n):
        m = T.SplineMesh(T.uniform_axis(0.0, L_, n))
        lev = O.Level(m)
        c = m.axis.colloc[1:-1]
        z, y, x = np.meshgrid(c, c, c, indexing="ij")
        phi = (np.sin(np.pi * x / L_) * np.sin(np.pi * y / L_) * np.sin(np.pi * z / L_)).ravel()
        out = np.zeros_like(phi)
        O.lib().orc_tensor_solve(lev.ref(), O.pd(np.ascontiguousarray(-3 * (np.pi / L_) ** 2 * phi)), O.pd(out))
        return np.linalg.norm(out - phi) / np.linalg.norm(phi)

    errs = [err(n) for n in (4, 8, 16)]
    assert errs[0] > errs[1] > errs[2]
    assert all(math.log2(errs[i] / errs[i + 1]) > 3.8 for i in range(2))
    assert errs[-1] < 1e-6
    m = T.SplineMesh(T.uniform_axis(0.0, L_, 8))
    lev = O.Level(m)
    rho = np.random.default_rng(0).standard_normal(16 ** 3)
    phi = np.zeros_like(rho)
    O.lib().orc_tensor_solve(lev.ref(), O.pd(rho), O.pd(phi))
    assert np.linalg.norm(_laplacian(O, lev, phi) - rho) / np.linalg.norm(rho) < 1e-10


def test_nested_poisson_faces_and_interior(O):
    # test/runtests.jl:368-398 and 887-931
    fine, coarse = T.uniform_axis(-10.0, 10.0, 8), T.uniform_axis(-30.0, 30.0, 8)
    mf, mc = T.SplineMesh(fine), T.SplineMesh(coarse)
    F, Cl = O.Level(mf), O.Level(mc)
    g, gc = fine.colloc, coarse.colloc
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    rhof = np.exp(-(x ** 2 + y ** 2 + z ** 2) / 2).ravel()
    z, y, x = np.meshgrid(gc, gc, gc, indexing="ij")
    rhoc = np.exp(-(x ** 2 + y ** 2 + z ** 2) / 2).ravel()
    phif, phic = np.zeros_like(rhof), np.zeros_like(rhoc)
    O.lib().orc_poisson(F.ref(), Cl.ref(), O.pd(rhof), O.pd(rhoc), O.pd(phif), O.pd(phic))
    assert np.all(np.isfinite(phif))
    coefs = np.zeros_like(phic)
    O.lib().orc_spline_coefficients(Cl.ref(), O.pd(phic), O.pd(coefs))
    n = mf.n
    for (i, j, k) in ((0, 3, 5), (n - 1, 1, 2)):
        v = C.c_double()
        assert O.lib().orc_spline_potential(Cl.ref(), O.pd(coefs), g[i], g[j], g[k], C.byref(v))
        assert abs(phif[i + n * (j + n * k)] - v.value) < 1e-12 * max(1, abs(v.value))
    # interior solves its own system with the lifted boundary
    ni = n - 2
    P = phif.reshape(n, n, n)
    inner = np.ascontiguousarray(P[1:-1, 1:-1, 1:-1]).ravel()
    D = mf.laplacian
    R = rhof.reshape(n, n, n)
    rhs = -4 * np.pi * R[1:-1, 1:-1, 1:-1]
    rhs = rhs - D[1:-1, 0][None, None, :] * P[1:-1, 1:-1, 0][:, :, None] - D[1:-1, -1][None, None, :] * P[1:-1, 1:-1, -1][:, :, None]
    rhs = rhs - D[1:-1, 0][None, :, None] * P[1:-1, 0, 1:-1][:, None, :] - D[1:-1, -1][None, :, None] * P[1:-1, -1, 1:-1][:, None, :]
    rhs = rhs - D[1:-1, 0][:, None, None] * P[0, 1:-1, 1:-1][None, :, :] - D[1:-1, -1][:, None, None] * P[-1, 1:-1, 1:-1][None, :, :]
    lap = _laplacian(O, F, inner)
    assert np.linalg.norm(lap - rhs.ravel()) / np.linalg.norm(rhs) < 1e-10


def test_electric_fields_of_a_linear_potential(O):
    # test/runtests.jl:637-695: Phi = x gives E = (-1, 0, 0)
    ax = T.uniform_axis(-50.0, 50.0, 28)
    m = T.SplineMesh(ax)
    lev = O.Level(m)
    n = m.n
    cx = np.zeros(n)
    c1 = np.zeros(n)
    for k in range(ax.nknots):
        cx[2 * k], cx[2 * k + 1] = ax.knots[k], 1.0
        c1[2 * k], c1[2 * k + 1] = 1.0, 0.0
    csol = (c1[:, None, None] * c1[None, :, None] * cx[None, None, :]).ravel()  # [k][j][i]
    for p in ((2.3, -1.7, 4.1), (-8.0, 0.5, -3.3), (11.2, 6.6, -9.9)):
        E = np.zeros(3)
        assert O.lib().orc_spline_field(lev.ref(), O.pd(csol), *p, O.pd(E))
        assert np.max(np.abs(E - (-1.0, 0.0, 0.0))) < 1e-13
    E = np.zeros(3)
    assert not O.lib().orc_spline_field(lev.ref(), O.pd(csol), 200.0, 0.0, 0.0, O.pd(E))
    # smoothed field through the host forces! path, w = 1
    sm = T.gaussian_smoothing(ax, nbdt=200, quadrature=200)
    S = O.Smoothing(sm)
    pts = np.array([(2.3, -1.7, 4.1), (-8.0, 0.5, -3.3), (11.2, 6.6, -9.9)])
    f = np.zeros((3, 3))
    O.lib().orc_forces_host(lev.ref(), lev.ref(), S.ref(), 3, O.pd(pts), O.pd(csol), O.pd(csol), 1.0, 0, O.pd(f))
    assert np.max(np.abs(f - np.array([-1.0, 0, 0]))) < 1e-4


def test_forces_three_regimes(O):
    # test/runtests.jl:697-720
    fine, coarse = T.uniform_axis(-50.0, 50.0, 28), T.uniform_axis(-150.0, 150.0, 28)
    mf, mc = T.SplineMesh(fine), T.SplineMesh(coarse)
    F, Cl = O.Level(mf), O.Level(mc)
    sm = T.gaussian_smoothing(fine, nbdt=100, quadrature=100)
    S = O.Smoothing(sm)
    csol = np.zeros(mf.n ** 3)
    pos = np.array([[0.0, 0, 0], [100.0, 0, 0], [400.0, 0, 0]])
    f = np.zeros((3, 3))
    nout = O.lib().orc_forces_host(F.ref(), Cl.ref(), S.ref(), 3, O.pd(pos), O.pd(csol), O.pd(csol), 0.01, 7,
                                   O.pd(f))
    assert nout == 2
    assert np.all(f[0] == 0) and np.all(f[1] == 0)
    assert abs(f[2, 0] - (-(0.01 ** 2) * 7 / 400 ** 2)) < 1e-18 and f[2, 1] == 0


def test_verlet_exact_free_flight_and_escape(O):
    # test/runtests.jl:400-466
    w, dt = 0.5, 0.05
    q0, v = np.array([1.0, -2.0, 0.5]), np.array([0.3, 0.1, -0.2])
    pos = q0[None, :].copy()
    prev = (q0 - dt * v)[None, :].copy()
    f = np.zeros((1, 3))
    diag = np.zeros(5)
    for _ in range(20):
        O.lib().orc_verlet_host(1, O.pd(pos), O.pd(prev), O.pd(f), dt, w, math.inf, O.pd(diag))
    assert np.allclose(pos[0], q0 + 20 * dt * v)
    assert abs(diag[0] - w * np.sum(v ** 2) / 2) < 1e-12
    three = np.array([[1.0, 0, 0], [5.0, 0, 0], [9.0, 0, 0]])
    prev3 = three - dt * v
    f3 = np.zeros((3, 3))
    O.lib().orc_verlet_host(3, O.pd(three), O.pd(prev3), O.pd(f3), dt, w, 6.0, O.pd(diag))
    assert abs(diag[1] - diag[0] / 3) < 1e-12


def test_packed_verlet_matches_plain(O, vb):
    # test/runtests.jl:543-596 in float32 offsets: free flight stays exact to the offset precision
    x0, h = -78.0, 2.4375
    w, dt = 0.5, 0.05
    start = np.array([(1.0 + 0.1 * i, 0.5 * i, -0.3 * i) for i in range(1, 51)])
    prev = start - dt * np.array([0.2, -0.1, 0.05])
    k, d = vb.pack_positions(start, x0, h)
    pk, pdl = vb.pack_positions(prev, x0, h)
    f = np.zeros((3, 50), np.float32)
    diag = np.zeros(5)
    args = (np.float32(dt * dt / w), np.float32(h), np.float32(x0), w / (2 * dt), np.float32(1e30), 1 / (2 * w))
    for _ in range(40):
        O.lib().orc_verlet_packed(50, O.pi(k), O.pf(d), O.pi(pk), O.pf(pdl), O.pf(f), *args, O.pd(diag))
    got = vb.unpack_positions(k, d, x0, h)
    want = start + 40 * dt * np.array([0.2, -0.1, 0.05])
    assert np.max(np.abs(got - want)) < 2e-5


def test_gaussian_softening_series_matches_closed_form(O):
    # test/runtests.jl:1343-1401: the series branch and the closed form agree at u = 0.5
    s = 5.0
    for u in (0.49, 0.4999999, 0.5000001, 0.51):
        r2 = (u * s) ** 2
        r = math.sqrt(r2)
        closed = (math.erf(r / (math.sqrt(2) * s)) - math.sqrt(2 / math.pi) * (r / s) * math.exp(-r2 / s ** 2 / 2)) / (r2 * r)
        assert abs(O.lib().orc_gaussian_force_kernel(r2, s) - closed) < 1e-9 * closed
    # far away it is Coulomb
    assert abs(O.lib().orc_gaussian_force_kernel(1e6, s) * 1e9 - 1) < 1e-9


def test_projectile_back_reaction_conserves_momentum(O):
    # test/runtests.jl:1403-1450: the reaction on the cloud balances the
    # electron part of the force on the projectile
    from oracle.oracle import OrcProjectile
    rng = np.random.default_rng(3)
    pos = 10 * rng.standard_normal((200, 3))
    force = np.zeros((200, 3))
    pr = OrcProjectile()
    pr.pos[0], pr.pos[1], pr.pos[2] = 3.0, 1.0, -2.0
    pr.charge, pr.mass, pr.ball_radius, pr.gauss_sigma, pr.active = 25.0, 1e5, 5.0, 5.0, 1
    F = np.zeros(3)
    ee, ej = np.zeros(1), np.zeros(1)
    O.lib().orc_projectile_forces_host(200, O.pd(pos), O.pd(force), C.byref(pr), 0.98, 0.0, 1e-3, O.pd(F),
                                       O.pd(ee), O.pd(ej))
    # outside an ion-free jellium the projectile force is the sum of the electron pulls
    assert np.allclose(F, -force.sum(axis=0), rtol=1e-12, atol=1e-14)


def test_mean_field_is_additive_in_coefficient_space(O):
    # test/runtests.jl:933-977
    ax = T.uniform_axis(-30.0, 30.0, 10)
    m = T.SplineMesh(ax)
    lev = O.Level(m)
    g = ax.colloc
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    rho = (1e-3 * np.exp(-(x ** 2 + y ** 2 + z ** 2) / 200)).ravel()
    jel = vb.Jellium.of(196.0)
    csol = np.zeros_like(rho)
    O.lib().orc_effective_potential(lev.ref(), O.pd(csol), O.pd(rho), jel.nions, jel.radius)
    c1 = csol.copy()
    O.lib().orc_effective_potential(lev.ref(), O.pd(csol), O.pd(rho), jel.nions, jel.radius)
    assert np.allclose(csol, 2 * c1, rtol=1e-12, atol=1e-15)
