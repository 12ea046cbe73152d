"""Setup tables of the two nested spline meshes and of the Gaussian smoothing.

Everything here runs once per simulation, on the host, in float64, and hands
the resulting tables to the device library (``vlb_create``).  It restates the
reference's set-up chain:

* Hermite basis and axes ............ src/splines.jl:74-287
* collocation matrices, S^-1, D ..... src/collocation.jl:34-94
* eigen-factorisation, 1/sum(lambda)  src/tensorsolver.jl:128-168
* SplineMesh and dual moments ....... src/mesh.jl:367-382
* dual lengths of the CIC deposit ... src/deposition.jl:23-33
* LocateTable ....................... src/splines.jl:362-396
* GaussianSmoothing (trapezoid) ..... src/fields.jl:162-217
* closed-form smoothing columns ..... src/fields.jl:79-160 (used to check the tables)

All axes of one mesh level are identical (the reference builds both levels
from one axis repeated three times, src/simulation.jl:175-178).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from fractions import Fraction

import numpy as np

VALUE, SLOPE = 0, 1
GAUSS2_NODES = ((1 - 1 / math.sqrt(3)) / 2, (1 + 1 / math.sqrt(3)) / 2)
GAUSS3_NODES = (-math.sqrt(3 / 5), 0.0, math.sqrt(3 / 5))
GAUSS3_WEIGHTS = (5 / 9, 8 / 9, 5 / 9)
# knot-index bounds of the 10 window basis functions (src/fields.jl:60-61)
SMOOTHING_SUPPORTS = ((1, 2), (1, 2), (1, 3), (1, 3), (2, 4),
                      (2, 4), (3, 5), (3, 5), (4, 5), (4, 5))


# --------------------------------------------------------------------------
# Hermite basis (src/splines.jl:24-147).  `lin` is the 1-based linear index
# 2(knot-1) + kind + 1, knots are 1-based as in the reference.
# --------------------------------------------------------------------------
def basis_of(lin: int) -> tuple[int, int]:
    q, r = divmod(lin - 1, 2)
    return q + 1, r


def hermite(kind, a, h, s):
    return 3 * (a * a) - 2 * (a * a * a) if kind == VALUE else h * (a * a - a * a * a) * s


def hermite1(kind, a, h, s):
    return -6 * (a - a * a) * s / h if kind == VALUE else -2 * a + 3 * (a * a)


def hermite2(kind, a, h, s):
    return 6 * (1 - 2 * a) / (h * h) if kind == VALUE else (2 - 6 * a) * s / h


def localcoords(g, knot, x):
    """src/splines.jl:110-122 (knot is 1-based)."""
    n, k = len(g), knot
    if k > 1 and x <= g[k - 1]:
        if x < g[k - 2]:
            return None
        h = g[k - 1] - g[k - 2]
        return ((x - g[k - 2]) / h, h, -1.0)
    elif k < n and x >= g[k - 1]:
        if x > g[k]:
            return None
        h = g[k] - g[k - 1]
        return ((g[k] - x) / h, h, 1.0)
    return None


def evaluate(g, lin, x, nder=0):
    """Value and derivatives of basis `lin` at `x` (src/splines.jl:130-139)."""
    knot, kind = basis_of(lin)
    loc = localcoords(g, knot, x)
    if loc is None:
        return (0.0,) * (nder + 1)
    a, h, s = loc
    out = [hermite(kind, a, h, s)]
    if nder >= 1:
        out.append(hermite1(kind, a, h, s))
    if nder >= 2:
        out.append(hermite2(kind, a, h, s))
    return tuple(out)


def value(g, lin, x):
    return evaluate(g, lin, x, 0)[0]


# --------------------------------------------------------------------------
# Axes (src/splines.jl:170-287)
# --------------------------------------------------------------------------
@dataclass
class SplineAxis:
    knots: np.ndarray
    colloc: np.ndarray

    def __post_init__(self):
        self.knots = np.asarray(self.knots, dtype=np.float64)
        self.colloc = np.asarray(self.colloc, dtype=np.float64)
        if np.any(np.diff(self.knots) < 0):
            raise ValueError("knots must be increasing")
        if len(self.colloc) != 2 * len(self.knots):
            raise ValueError("2 collocation points per knot are required")

    @property
    def nknots(self):
        return len(self.knots)

    @property
    def nbasis(self):
        return 2 * len(self.knots)


def collocation_points(knots) -> np.ndarray:
    out = [knots[0]]
    for j in range(len(knots) - 1):
        for u in GAUSS2_NODES:
            out.append(knots[j] + (knots[j + 1] - knots[j]) * u)
    out.append(knots[-1])
    return np.array(out, dtype=np.float64)


def _exact_range(x0: float, xn: float, length: int) -> list[float]:
    """`range(x0, xn; length)` of Float64: every element the correctly rounded
    x0 + (xn-x0)*i/(length-1), which is what the reference's TwicePrecision
    range yields."""
    a, b = Fraction(x0), Fraction(xn)
    m = length - 1
    return [float(a + (b - a) * i / m) for i in range(length)]


def uniform_axis(x0: float, xn: float, nintervals: int) -> SplineAxis:
    """src/splines.jl:219-222"""
    knots = np.array(_exact_range(x0, xn, nintervals + 1))
    return SplineAxis(knots, collocation_points(knots))


def stretch_ratio(h1: float, L: float, n: int) -> float:
    """Bisection to the last float (src/splines.jl:239-253)."""
    def f(a):
        return L * (1 - a) / (1 - a ** n) - h1
    lo, hi = math.nextafter(1.0, 2.0), 10.0
    flo = f(lo)
    if math.copysign(1, flo) == math.copysign(1, f(hi)):
        raise ValueError(f"no geometric ratio in ]1, 10] for h1={h1}, L={L}, n={n}")
    while math.nextafter(lo, math.inf) < hi:
        mid = (lo + hi) / 2
        if mid == lo or mid == hi:
            break
        if math.copysign(1, f(mid)) == math.copysign(1, flo):
            lo = mid
        else:
            hi = mid
    return (lo + hi) / 2


def stretched_axis(xinner: float, xouter: float, n_inner: int, n_outer: int) -> SplineAxis:
    """src/splines.jl:272-287"""
    h1 = xinner / (n_inner - 1)
    L = xouter - xinner
    a = stretch_ratio(h1, L, n_outer)
    step = L * (1 - a) / (1 - a ** n_outer)
    half = _exact_range(0.0, xinner, n_inner)
    acc = 0.0
    for k in range(n_outer):
        acc += step * (a ** k if k else 1.0)
        half.append(xinner + acc)
    knots = [-v for v in reversed(half[1:])] + half
    knots = np.array(knots, dtype=np.float64)
    return SplineAxis(knots, collocation_points(knots))


# --------------------------------------------------------------------------
# Moments (src/splines.jl:302-340)
# --------------------------------------------------------------------------
def _gauss3(g, lin, a, c, k):
    mid, half = (a + c) / 2, (c - a) / 2
    terms = []
    for xi, w in zip(GAUSS3_NODES, GAUSS3_WEIGHTS):
        x = mid + half * xi
        xk = 1.0 if k == 0 else (x if k == 1 else x * x)
        terms.append(w * xk * value(g, lin, x))
    return half * ((terms[0] + terms[1]) + terms[2])


def moment(g, lin, k):
    n = len(g)
    kn, _ = basis_of(lin)
    total = 0.0
    if kn > 1:
        total += _gauss3(g, lin, g[kn - 2], g[kn - 1], k)
    if kn < n:
        total += _gauss3(g, lin, g[kn - 1], g[kn], k)
    return total


def moments(ax: SplineAxis, k: int) -> np.ndarray:
    return np.array([moment(ax.knots, lin, k) for lin in range(1, ax.nbasis + 1)])


# --------------------------------------------------------------------------
# Collocation matrices and the 1-D operator (src/collocation.jl:34-94)
# --------------------------------------------------------------------------
@dataclass
class CollocationMatrices:
    axis: SplineAxis
    S: np.ndarray
    S1: np.ndarray
    S2: np.ndarray
    Sinv: np.ndarray


def collocation_matrices(ax: SplineAxis) -> CollocationMatrices:
    m = ax.nbasis
    S, S1, S2 = (np.zeros((m, m)) for _ in range(3))
    g, gt = ax.knots, ax.colloc
    for j in range(1, ax.nknots):
        for lin in range(2 * j - 1, 2 * j + 3):
            for k in (2 * j, 2 * j + 1):
                S[k - 1, lin - 1], S1[k - 1, lin - 1], S2[k - 1, lin - 1] = \
                    evaluate(g, lin, gt[k - 1], 2)
    S[0, 0], S1[0, 0], S2[0, 0] = evaluate(g, 1, gt[0], 2)
    S[m - 1, m - 2], S1[m - 1, m - 2], S2[m - 1, m - 2] = evaluate(g, m - 1, gt[m - 1], 2)
    return CollocationMatrices(ax, S, S1, S2, np.linalg.inv(S))


def laplacian1d_full(cm: CollocationMatrices) -> np.ndarray:
    """D = S'' S^-1 by an LU right-division (src/collocation.jl:94)."""
    return np.linalg.solve(cm.S.T, cm.S2.T).T


def dual_moments(cm: CollocationMatrices):
    """S^-T m for orders 0,1,2 (src/mesh.jl:367-368)."""
    return tuple(cm.Sinv.T @ moments(cm.axis, k) for k in range(3))


def dual_lengths(ax: SplineAxis) -> np.ndarray:
    """src/deposition.jl:23-33"""
    gt, g = ax.colloc, ax.knots
    m = len(gt)
    out = np.empty(m)
    for j in range(1, m + 1):
        if j == 1:
            out[0] = (gt[1] - g[0]) / 2
        elif j == 2:
            out[1] = (gt[2] - g[0]) / 2
        elif j == m:
            out[m - 1] = (g[-1] - gt[m - 2]) / 2
        elif j == m - 1:
            out[m - 2] = (g[-1] - gt[m - 3]) / 2
        else:
            out[j - 1] = (gt[j] - gt[j - 2]) / 2
    return out


@dataclass
class DiagonalizedOperator:
    """Real eigen-factorisation of a 1-D operator (src/tensorsolver.jl:123-138)."""
    M: np.ndarray
    Minv: np.ndarray
    lam: np.ndarray

    @staticmethod
    def of(D: np.ndarray, atol: float = 1e-10) -> "DiagonalizedOperator":
        vals, vecs = np.linalg.eig(D)
        imagmax = np.max(np.abs(vals.imag))
        scale = np.max(np.abs(vals.real))
        if imagmax > atol * max(scale, 1.0):
            raise ValueError(f"non-real spectrum (max|Im lambda| = {imagmax})")
        M = np.ascontiguousarray(vecs.real)
        return DiagonalizedOperator(M, np.linalg.inv(M), np.ascontiguousarray(vals.real))


def inv_lambda_sum(lx, ly, lz) -> np.ndarray:
    """1/(lx[i]+ly[j]+lz[k]) stored with i fastest (src/tensorsolver.jl:157-168)."""
    s = (lx[None, None, :] + ly[None, :, None]) + lz[:, None, None]
    if np.any(s == 0):
        raise ValueError("eigenvalue sum vanishes: singular operator")
    return 1.0 / s


@dataclass
class LocateTable:
    """Uniform bins over the collocation points (src/splines.jl:362-376).
    `cell` holds 1-based cell indices, as the reference does."""
    x0: float
    invwidth: float
    cell: np.ndarray

    @staticmethod
    def of(ax: SplineAxis) -> "LocateTable":
        gt = ax.colloc
        n = len(gt)
        width = np.min(np.diff(gt)) / 2
        nbin = math.ceil((gt[-1] - gt[0]) / width) + 2
        xs = np.array([gt[0] + b * width for b in range(nbin)])
        cell = np.clip(np.searchsorted(gt, xs, side="right"), 1, n - 1).astype(np.int32)
        return LocateTable(float(gt[0]), 1.0 / width, cell)


@dataclass
class SplineMesh:
    """One cubic mesh level: everything the Poisson chain draws from it
    (src/mesh.jl:327-382).  The three axes are identical."""
    axis: SplineAxis
    cm: CollocationMatrices = field(init=False)
    laplacian: np.ndarray = field(init=False)
    op: DiagonalizedOperator = field(init=False)
    duals: tuple = field(init=False)
    dlen: np.ndarray = field(init=False)
    invlsum: np.ndarray = field(init=False)
    locator: LocateTable = field(init=False)

    def __post_init__(self):
        self.cm = collocation_matrices(self.axis)
        self.laplacian = laplacian1d_full(self.cm)
        self.op = DiagonalizedOperator.of(self.laplacian[1:-1, 1:-1])
        self.duals = dual_moments(self.cm)
        self.dlen = dual_lengths(self.axis)
        lam = self.op.lam
        self.invlsum = inv_lambda_sum(lam, lam, lam)
        self.locator = LocateTable.of(self.axis)

    @property
    def n(self):
        return self.axis.nbasis

    @property
    def interior(self):
        return self.axis.nbasis - 2


# --------------------------------------------------------------------------
# Gaussian smoothing tables (src/fields.jl:162-217)
# --------------------------------------------------------------------------
@dataclass
class GaussianSmoothing:
    sigma: float
    spacing: float
    nbdt: int
    overlap: np.ndarray   # (10, nbdt+1)
    gradient: np.ndarray  # (10, nbdt+1)
    nodes: np.ndarray     # (8, nbdt+1)


def _trapezoid_rows(fvals_of_x, xs, step):
    """Trapezoid over the accumulated abscissae, one row per table column.
    `fvals_of_x(k)` returns f(xs[k]) for every column at once."""
    total = np.zeros_like(fvals_of_x(0))
    fx = fvals_of_x(0)
    for k in range(1, len(xs)):
        fnext = fvals_of_x(k)
        total += (fx + fnext) * step / 2
        fx = fnext
    return total


def gaussian_smoothing(ax: SplineAxis, nbdt: int = 1000, quadrature: int = 1000) -> GaussianSmoothing:
    g = ax.knots
    h = g[1] - g[0]
    sigma = h / 3
    norm1d = 1.0 / (math.sqrt(2 * math.pi) * sigma)
    rmin, rmax = (g[2] + g[1]) / 2, (g[3] + g[2]) / 2
    r = np.array([rmin + i * (rmax - rmin) / nbdt for i in range(nbdt + 1)])
    two_s2 = 2 * sigma ** 2
    s2 = sigma ** 2
    overlap = np.empty((10, nbdt + 1))
    gradient = np.empty((10, nbdt + 1))
    nodes = np.empty((8, nbdt + 1))
    for a in range(1, 11):
        lo, hi = SMOOTHING_SUPPORTS[a - 1]
        a0, b0 = g[lo - 1], g[hi - 1]
        step = (b0 - a0) / quadrature
        xs = [a0]
        for _ in range(quadrature):
            xs.append(xs[-1] + step)
        vs = [value(g, a, x) for x in xs]

        def f_ov(k):
            gauss = norm1d * np.exp(-((r - xs[k]) ** 2) / two_s2)
            return vs[k] * gauss

        def f_gr(k):
            gauss = norm1d * np.exp(-((r - xs[k]) ** 2) / two_s2)
            return (-(r - xs[k])) / s2 * vs[k] * gauss

        overlap[a - 1] = _trapezoid_rows(f_ov, xs, step)
        gradient[a - 1] = _trapezoid_rows(f_gr, xs, step)
    for a in range(1, 9):
        nodes[a - 1] = norm1d * np.exp(-((r - ax.colloc[a]) ** 2) / two_s2)
    return GaussianSmoothing(sigma, h, nbdt, overlap, gradient, nodes)


def _smoothing_moments(u):
    e = math.exp(-u * u / 2)
    s = math.sqrt(math.pi / 2) * math.erf(u / math.sqrt(2))
    return (s, -e, s - u * e, -(u * u + 2) * e, 3 * s - (u * u * u + 3 * u) * e)


def smoothing_columns(delta: float, h: float):
    """Exact overlap/gradient columns at offset delta (src/fields.jl:124-160)."""
    t = 3 * delta / h
    M = [_smoothing_moments(3 * (j - 3) - t) for j in range(1, 6)]
    ov, gr = [0.0] * 10, [0.0] * 10
    third = 1 / 3
    for a in range(1, 11):
        k, kind = basis_of(a)
        lo, hi = SMOOTHING_SUPPORTS[a - 1]
        o = dg = 0.0
        for j, direc in ((k - 1, 1), (k, -1)):
            if not (1 <= j <= 4 and j >= lo and j + 1 <= hi):
                continue
            d = [M[j][n] - M[j - 1][n] for n in range(5)]
            al = -(3 * (j - 3) - t) * third if direc > 0 else (3 * (j - 2) - t) * third
            be = third if direc > 0 else -third
            q2 = al * al * d[0] + 2 * al * be * d[1] + be * be * d[2]
            q3 = al ** 3 * d[0] + 3 * al ** 2 * be * d[1] + 3 * al * be ** 2 * d[2] + be ** 3 * d[3]
            r2 = al * al * d[1] + 2 * al * be * d[2] + be * be * d[3]
            r3 = al ** 3 * d[1] + 3 * al ** 2 * be * d[2] + 3 * al * be ** 2 * d[3] + be ** 3 * d[4]
            sgn = -1.0 if direc > 0 else 1.0
            cv, cs = (3.0, -2.0) if kind == VALUE else (sgn, -sgn)
            sc = 1.0 if kind == VALUE else h
            o += sc * (cv * q2 + cs * q3)
            dg += sc * (cv * r2 + cs * r3)
        ov[a - 1], gr[a - 1] = o, dg
    sigma = h / 3
    norm = 1 / (math.sqrt(2 * math.pi) * sigma)
    return [norm * sigma * v for v in ov], [norm * v for v in gr]


# --------------------------------------------------------------------------
# The nested pair (src/simulation.jl:175-178, scripts/xenon.jl:162-167)
# --------------------------------------------------------------------------
def grids(nfine: int):
    """Coarse subdivision derived from the fine one (scripts/xenon.jl:162-167)."""
    if nfine % 2:
        raise ValueError(f"nfine must be even (got {nfine})")
    m = nfine // 2 + 1
    n1 = m // 2
    return 2 * n1, 2 * (m - n1) - 2


@dataclass
class NestedMeshes:
    fine: SplineMesh
    coarse: SplineMesh

    def __post_init__(self):
        fi, co = self.fine.axis.knots, self.coarse.axis.knots
        if not (co[0] <= fi[0] and fi[-1] <= co[-1]):
            raise ValueError("the fine level sticks out of the coarse level")


def build_meshes(nfine: int, ninner: int, nouter: int, rcluster: float, rbox: float) -> NestedMeshes:
    fine = uniform_axis(-rcluster, rcluster, nfine)
    coarse = stretched_axis(rcluster, rbox, ninner // 2, (nouter + 2) // 2)
    return NestedMeshes(SplineMesh(fine), SplineMesh(coarse))
