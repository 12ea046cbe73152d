"""Known-answer tests of the set-up tables, restated from the reference's own
suite (test/runtests.jl) -- the oracle and the device library both consume
these tables, so they are pinned first."""
import math

import numpy as np
import pytest

from conftest import load_package

T = load_package().tables


def make_testaxis(n=8, L=1.0):
    """Non-uniform test grid (test/runtests.jl:9-21)."""
    knots = [L * (t + 0.15 * math.sin(2 * math.pi * t)) for t in np.linspace(0, 1, n + 1)]
    colloc = [knots[0]]
    for j in range(n):
        a, b = knots[j], knots[j + 1]
        colloc += [a + (b - a) / 3, a + 2 * (b - a) / 3]
    colloc.append(knots[-1])
    return T.SplineAxis(np.array(knots), np.array(colloc))


def test_hermite_basis_identities():
    # test/runtests.jl:63-88
    ax = make_testaxis()
    g = ax.knots
    for k in range(2, ax.nknots):
        v, s = 2 * (k - 1) + 1, 2 * (k - 1) + 2
        assert abs(T.evaluate(g, v, g[k - 1], 1)[0] - 1) < 1e-14
        assert abs(T.evaluate(g, s, g[k - 1], 1)[0]) < 1e-14
        assert abs(T.evaluate(g, v, g[k - 1], 1)[1]) < 1e-12
        assert abs(T.evaluate(g, s, g[k - 1], 1)[1] - 1) < 1e-12
        assert abs(T.value(g, v, g[k - 2])) < 1e-14
        assert abs(T.value(g, v, g[k])) < 1e-14
    assert T.value(g, 7, g[1]) == 0 and T.value(g, 7, g[5]) == 0


def test_reproduction_of_cubics():
    # test/runtests.jl:90-108
    ax = make_testaxis(10)
    p = lambda x: 2.0 - 0.7 * x + 1.3 * x ** 2 - 0.4 * x ** 3
    dp = lambda x: -0.7 + 2.6 * x - 1.2 * x ** 2
    for x in np.linspace(ax.knots[0], ax.knots[-1], 37):
        s = sum(p(ax.knots[k]) * T.value(ax.knots, 2 * k + 1, x) + dp(ax.knots[k]) * T.value(ax.knots, 2 * k + 2, x)
                for k in range(ax.nknots))
        assert abs(s - p(x)) < 1e-12


def test_axis_construction():
    # test/runtests.jl:110-152
    ax = T.uniform_axis(-50.0, 50.0, 28)
    assert ax.nknots == 29 and ax.nbasis == 58
    assert ax.knots[0] == -50.0 and ax.knots[-1] == 50.0
    h = ax.knots[1] - ax.knots[0]
    assert abs(ax.colloc[1] - (ax.knots[0] + h * (1 - 1 / math.sqrt(3)) / 2)) < 1e-13
    h1, L, n = 50.0 / 6, 100.0, 8
    a = T.stretch_ratio(h1, L, n)
    assert a > 1 and abs(L * (1 - a) / (1 - a ** n) - h1) < 1e-13
    axs = T.stretched_axis(50.0, 150.0, 7, 8)
    assert axs.nknots == 29
    assert abs(axs.knots[0] + 150) < 1e-9 and abs(axs.knots[-1] - 150) < 1e-9
    assert abs(axs.knots[14]) < 1e-12
    assert np.allclose(axs.knots, -axs.knots[::-1])
    assert abs(np.diff(axs.knots)[7] - h1) < 1e-9 * h1
    assert np.all(np.diff(axs.knots) > 0)


@pytest.mark.parametrize("axis", ["uniform", "stretched", "test"])
def test_moments_exact_on_cubics(axis):
    # test/runtests.jl:154-184
    ax = {"uniform": lambda: T.uniform_axis(-2.0, 3.0, 9), "stretched": lambda: T.stretched_axis(1.0, 4.0, 5, 6),
          "test": lambda: make_testaxis(11)}[axis]()
    c = (2.0, -0.7, 1.3, -0.4)
    p = lambda x: sum(cj * x ** j for j, cj in enumerate(c))
    dp = lambda x: sum(j * cj * x ** (j - 1) for j, cj in enumerate(c) if j)
    x0, xn = ax.knots[0], ax.knots[-1]
    for k in range(3):
        m = T.moments(ax, k)
        got = sum(p(g) * m[2 * i] + dp(g) * m[2 * i + 1] for i, g in enumerate(ax.knots))
        exact = sum(cj * (xn ** (j + k + 1) - x0 ** (j + k + 1)) / (j + k + 1) for j, cj in enumerate(c))
        assert abs(got - exact) <= 1e-11 * abs(exact)


def test_collocation_matrices_and_operator():
    # test/runtests.jl:186-247
    ax = make_testaxis(12)
    cm = T.collocation_matrices(ax)
    m = ax.nbasis
    i, j = np.indices((m, m))
    assert np.all(cm.S[np.abs(i - j) > 2] == 0)
    assert not np.allclose(cm.S, cm.S.T)
    D = T.laplacian1d_full(cm)
    assert np.linalg.norm(D @ cm.S - cm.S2) / np.linalg.norm(cm.S2) < 1e-12
    lam = np.linalg.eigvals(D[1:-1, 1:-1])
    assert np.max(np.abs(lam.imag)) < 1e-10 * np.max(np.abs(lam.real))
    assert np.all(lam.real < 0)
    # D f = f'' exactly on a cubic, interior rows
    ax = T.uniform_axis(-2.0, 3.0, 10)
    Df = T.laplacian1d_full(T.collocation_matrices(ax))
    f = lambda x: 2.0 - 0.7 * x + 1.3 * x ** 2 - 0.4 * x ** 3
    got = Df @ f(ax.colloc)
    assert np.max(np.abs(got[1:-1] - (2.6 - 2.4 * ax.colloc[1:-1]))) < 1e-11


def test_lookup_table_equals_bisection():
    # test/runtests.jl:722-743 (locate, src/deposition.jl:42-47)
    for ax in (T.uniform_axis(-10.0, 10.0, 8), T.stretched_axis(50.0, 150.0, 7, 8), make_testaxis(9, L=3.0)):
        tbl = T.LocateTable.of(ax)
        gt = ax.colloc

        def bis(x):
            if x < gt[0] or x > gt[-1]:
                return None
            c = max(1, int(np.searchsorted(gt, x, side="left")))
            return c, (gt[c] - x) / (gt[c] - gt[c - 1])

        def tab(x):
            if x < gt[0] or x > gt[-1]:
                return None
            b = min(math.floor((x - tbl.x0) * tbl.invwidth) + 1, len(tbl.cell))
            c = int(tbl.cell[b - 1])
            while c < len(gt) - 1 and gt[c] < x:
                c += 1
            return c, (gt[c] - x) / (gt[c] - gt[c - 1])

        for u in np.linspace(gt[0], gt[-1], 997):
            assert tab(u) == bis(u)
        assert tab(gt[0] - 1e-9) is None and tab(gt[-1] + 1e-9) is None
        assert len(tbl.cell) >= len(gt)


def test_smoothing_tables_match_closed_form():
    # test/runtests.jl:468-501, and the documented 5.4e-11 / 4.9e-10 agreement
    ax = T.uniform_axis(-78.0, 78.0, 110)
    sm = T.gaussian_smoothing(ax)
    h = ax.knots[1] - ax.knots[0]
    eo = eg = 0.0
    for i in range(0, sm.nbdt + 1, 50):
        d = (i / sm.nbdt) * h - h / 2
        ov, gr = T.smoothing_columns(d, h)
        eo = max(eo, np.max(np.abs(np.array(ov) - sm.overlap[:, i])))
        eg = max(eg, np.max(np.abs(np.array(gr) - sm.gradient[:, i])))
    assert eo < 1e-9 and eg < 1e-8
    assert np.max(np.abs(sm.overlap)) > 0.5 and np.max(np.abs(sm.gradient)) > 0.5
    assert abs(sm.sigma - h / 3) < 1e-15


def test_smoothing_kernel_normalisation():
    # test/runtests.jl:688-694
    ax = T.uniform_axis(-50.0, 50.0, 28)
    sm = T.gaussian_smoothing(ax, nbdt=200, quadrature=200)
    cst = np.array([1.0 if a % 2 == 1 else 0.0 for a in range(1, 11)])
    assert np.max(np.abs(cst @ sm.overlap - 1)) < 1e-5
    assert np.max(np.abs(cst @ sm.gradient)) < 1e-4


def test_nested_meshes_of_the_xenon_run():
    # scripts/xenon.jl:162-167, src/simulation.jl:175-178
    assert T.grids(64) == (32, 32) and T.grids(28) == (14, 14) and T.grids(48) == (24, 24)
    m = T.build_meshes(64, 32, 32, 78.0, 235.0)
    assert m.fine.n == 130 and m.coarse.n == 130
    assert m.fine.axis.knots[1] - m.fine.axis.knots[0] == 2.4375
    assert abs(m.coarse.axis.knots[0] + 235) < 1e-9 and abs(m.coarse.axis.knots[-1] - 235) < 1e-9
    assert np.all(m.fine.op.lam < 0) and np.all(m.coarse.op.lam < 0)
    with pytest.raises(ValueError):
        T.NestedMeshes(m.coarse, m.fine)
