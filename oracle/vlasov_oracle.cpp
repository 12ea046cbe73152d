// ORACLE -- test infrastructure only.
//
// A float64 CPU restatement of LaurentPlagne/Vlasov.jl's per-step
// pseudo-particle loop, used as the checker of the CUDA library.  Only the
// tests, the smoke check and bench.py's CPU-baseline / reference arms load
// it; the product path never does.
//
// Two semantics are restated:
//
//  * the reference's CPU path (src/simulation.jl:309-352): float64 positions,
//    host deposit_smoothed!/deposit!, host forces! with its margin test, host
//    projectile_forces! with ball softening, host Verlet;
//  * the reference's device path (src/simulation.jl:472-531): the packed
//    (k int32, delta float32) cloud, the stable counting sort, the FP32
//    discrete choices of the kernels (table columns, stencil fit, CIC cell
//    lookup, Verlet integer update) replicated bit for bit, and every
//    continuous quantity (density, potential, forces, projectile) in float64.
//
// Parity anchors: the reference's known-answer tests (test/runtests.jl) are
// restated in tests/; no Fortran dumps ship with the reference, so the
// float64 arithmetic here is pinned by those tests and by analytic cases.
//
// Build: g++ -O3 -march=native -fopenmp -ffp-contract=off -shared -fPIC.
// -ffp-contract=off keeps a*b+c as two roundings, which the FP32 discrete
// replicas below depend on.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

extern "C" {

struct orc_level {
  int32_t nk;             // knots per axis
  int32_t n;              // collocation points per axis = 2 nk
  const double* knots;    // [nk]
  const double* colloc;   // [n]
  const double* sinv;     // [n*n] row-major S^-1
  const double* lap;      // [n*n] row-major full laplacian D = S'' S^-1
  const double* M;        // [(n-2)^2] row-major eigenvectors
  const double* Minv;     // [(n-2)^2] row-major inverse
  const double* invlsum;  // [(n-2)^3] 1/(lx+ly+lz), i fastest
  const double* dual;     // [3*n] dual moments, orders 0,1,2
  const double* dlen;     // [n] dual lengths
  double loc_x0, loc_invw;
  int32_t loc_ncell;
  const int32_t* loc_cells;  // [loc_ncell], 1-based cells
};

struct orc_smoothing {
  int32_t nbdt;
  double spacing;
  const double* overlap;   // [(nbdt+1)*10]  column-major: [col][a]
  const double* gradient;  // [(nbdt+1)*10]
  const double* nodes;     // [(nbdt+1)*8]
};

// Projectile scalars.  `gauss_sigma` is the width of the Gaussian kernel of
// the fused device path (scale(softening), src/accelerator.jl:632);
// `ball_radius` the ball of the host paths (src/projectile.jl:79-80).
struct orc_projectile {
  double pos[3], prev[3], vel[3];
  double charge, mass, gauss_sigma, ball_radius;
  int32_t active;
  int32_t softening;  // 0: the device path's (Gaussian in the stencil, ball in the tail); 1: the ball everywhere
};

}  // extern "C"

namespace {

constexpr double PI = 3.14159265358979323846;

// ---------------------------------------------------------------- splines
// src/splines.jl:74-139
inline double hermite(int kind, double a, double h, double s) {
  return kind == 0 ? 3 * (a * a) - 2 * (a * a * a) : h * (a * a - a * a * a) * s;
}
inline double hermite1(int kind, double a, double h, double s) {
  return kind == 0 ? -6 * (a - a * a) * s / h : -2 * a + 3 * (a * a);
}
// value and first derivative of basis `lin` (1-based) at x
inline void eval_basis(const double* g, int nk, int lin, double x, double* v, double* d) {
  int knot = (lin - 1) / 2 + 1, kind = (lin - 1) % 2;
  int k = knot;
  double a, h, s;
  if (k > 1 && x <= g[k - 1]) {
    if (x < g[k - 2]) { *v = 0; *d = 0; return; }
    h = g[k - 1] - g[k - 2]; a = (x - g[k - 2]) / h; s = -1.0;
  } else if (k < nk && x >= g[k - 1]) {
    if (x > g[k]) { *v = 0; *d = 0; return; }
    h = g[k] - g[k - 1]; a = (g[k] - x) / h; s = 1.0;
  } else { *v = 0; *d = 0; return; }
  *v = hermite(kind, a, h, s);
  if (d) *d = hermite1(kind, a, h, s);
}

// 1-based cell of x on the knots, 0 outside (src/fields.jl:235-238)
inline int cell_index(const double* g, int nk, double x) {
  if (x < g[0] || x > g[nk - 1]) return 0;
  int idx0 = int(std::lower_bound(g, g + nk, x) - g);  // 0-based first >= x
  return std::max(1, idx0);  // searchsortedfirst - 1, 1-based
}

// 1-based nearest knot (src/fields.jl:224-227)
inline int nearest_knot(const double* g, int nk, double x) {
  int last = int(std::upper_bound(g, g + nk, x) - g);  // searchsortedlast
  int i = std::min(std::max(last, 1), nk - 1);
  return (g[i] - x) < (x - g[i - 1]) ? i + 1 : i;
}

// spline_potential (src/fields.jl:440-469); returns false outside
bool spline_potential(const double* g, int nk, const double* c, int n,
                      double px, double py, double pz, double* out) {
  int cx = cell_index(g, nk, px), cy = cell_index(g, nk, py), cz = cell_index(g, nk, pz);
  if (!cx || !cy || !cz) return false;
  double vx[4], vy[4], vz[4], dd;
  for (int a = 0; a < 4; ++a) {
    eval_basis(g, nk, 2 * (cx - 1) + a + 1, px, &vx[a], &dd);
    eval_basis(g, nk, 2 * (cy - 1) + a + 1, py, &vy[a], &dd);
    eval_basis(g, nk, 2 * (cz - 1) + a + 1, pz, &vz[a], &dd);
  }
  double phi = 0;
  for (int ak = 0; ak < 4; ++ak) {
    int k = 2 * (cz - 1) + ak;
    for (int aj = 0; aj < 4; ++aj) {
      int j = 2 * (cy - 1) + aj;
      double w = vy[aj] * vz[ak];
      for (int ai = 0; ai < 4; ++ai) {
        int i = 2 * (cx - 1) + ai;
        phi += c[i + (size_t)n * (j + (size_t)n * k)] * vx[ai] * w;
      }
    }
  }
  *out = phi;
  return true;
}

// spline_field (src/fields.jl:358-393): -grad of the interpolant
bool spline_field(const double* g, int nk, const double* c, int n,
                  double px, double py, double pz, double E[3]) {
  int cx = cell_index(g, nk, px), cy = cell_index(g, nk, py), cz = cell_index(g, nk, pz);
  if (!cx || !cy || !cz) return false;
  double vx[4], vy[4], vz[4], dx[4], dy[4], dz[4];
  for (int a = 0; a < 4; ++a) {
    eval_basis(g, nk, 2 * (cx - 1) + a + 1, px, &vx[a], &dx[a]);
    eval_basis(g, nk, 2 * (cy - 1) + a + 1, py, &vy[a], &dy[a]);
    eval_basis(g, nk, 2 * (cz - 1) + a + 1, pz, &vz[a], &dz[a]);
  }
  double ex = 0, ey = 0, ez = 0;
  for (int ak = 0; ak < 4; ++ak) {
    int k = 2 * (cz - 1) + ak;
    for (int aj = 0; aj < 4; ++aj) {
      int j = 2 * (cy - 1) + aj;
      for (int ai = 0; ai < 4; ++ai) {
        int i = 2 * (cx - 1) + ai;
        double cc = c[i + (size_t)n * (j + (size_t)n * k)];
        ex -= cc * dx[ai] * vy[aj] * vz[ak];
        ey -= cc * vx[ai] * dy[aj] * vz[ak];
        ez -= cc * vx[ai] * vy[aj] * dz[ak];
      }
    }
  }
  E[0] = ex; E[1] = ey; E[2] = ez;
  return true;
}

// ------------------------------------------------------------ tensor chain
// dest[p + m i'] = sum_i A[i'][i] src[i + n p]   (src/tensorsolver.jl:217-223)
// Blocked over 16 columns p so that each output row segment is contiguous
// (the reference does it as one BLAS GEMM, C = X^T A^T).
void mode_product(double* dest, const double* A, const double* src, int n, size_t m) {
  constexpr int PB = 16;
  const long long nblk = (long long)((m + PB - 1) / PB);
#pragma omp parallel
  {
    std::vector<double> xt((size_t)n * PB);
#pragma omp for schedule(static)
    for (long long b = 0; b < nblk; ++b) {
      const size_t p0 = (size_t)b * PB;
      const int cnt = (int)std::min<size_t>(PB, m - p0);
      for (int pp = 0; pp < PB; ++pp)
        for (int i = 0; i < n; ++i) xt[(size_t)i * PB + pp] = pp < cnt ? src[(p0 + pp) * n + i] : 0.0;
      for (int r = 0; r < n; ++r) {
        const double* a = A + (size_t)r * n;
        double acc[PB] = {0};
        for (int i = 0; i < n; ++i) {
          const double ai = a[i];
          const double* x = &xt[(size_t)i * PB];
          for (int pp = 0; pp < PB; ++pp) acc[pp] += ai * x[pp];
        }
        double* out = dest + p0 + m * r;
        for (int pp = 0; pp < cnt; ++pp) out[pp] = acc[pp];
      }
    }
  }
}

// three rotations, dest/work alternating on the parity of the remaining
// steps (src/tensorsolver.jl:243-254)
void apply_all_rotating(double* dest, const double* A, const double* src, double* work, int n) {
  size_t m = (size_t)n * n;
  mode_product(dest, A, src, n, m);
  mode_product(work, A, dest, n, m);
  mode_product(dest, A, work, n, m);
}

// X = (M (x) M (x) M) diag(invlsum) (Minv (x) Minv (x) Minv) B  (src/tensorsolver.jl:267-296)
void tensor_solve(double* X, const double* B, const orc_level& L, double* w1, double* w2) {
  int ni = L.n - 2;
  size_t tot = (size_t)ni * ni * ni;
  apply_all_rotating(w1, L.Minv, B, w2, ni);
  for (size_t t = 0; t < tot; ++t) w1[t] *= L.invlsum[t];
  apply_all_rotating(X, L.M, w1, w2, ni);
}

struct Multipole { double q, c[3], quad[6]; };

// all_moments + _multipole (src/poisson.jl:55-189)
Multipole multipole(const double* rho, const orc_level& L) {
  int n = L.n;
  const double *p0 = L.dual, *p1 = L.dual + n, *p2 = L.dual + 2 * n;
  double tot[10] = {0};
  std::vector<double> part((size_t)n * n * 10);
#pragma omp parallel for schedule(static)
  for (int t = 0; t < n * n; ++t) {
    int j = t % n, k = t / n;
    double a = p0[j] * p0[k], b = p1[j] * p0[k], cc = p0[j] * p1[k];
    double d = p2[j] * p0[k], e = p0[j] * p2[k], f = p1[j] * p1[k];
    double s0 = 0, s1 = 0, s2 = 0;
    const double* col = rho + (size_t)n * t;
    for (int i = 0; i < n; ++i) { double v = col[i]; s0 += v * p0[i]; s1 += v * p1[i]; s2 += v * p2[i]; }
    double* P = &part[(size_t)t * 10];
    P[0] = s0 * a; P[1] = s1 * a; P[2] = s0 * b; P[3] = s0 * cc; P[4] = s2 * a;
    P[5] = s0 * d; P[6] = s0 * e; P[7] = s1 * b; P[8] = s1 * cc; P[9] = s0 * f;
  }
  for (int t = 0; t < n * n; ++t)
    for (int r = 0; r < 10; ++r) tot[r] += part[(size_t)t * 10 + r];
  Multipole mp;
  double q = tot[0];
  mp.q = q;
  for (int d = 0; d < 3; ++d) mp.c[d] = (q == 0) ? 0.0 : tot[1 + d] / q;
  double m200 = tot[4], m020 = tot[5], m002 = tot[6], mxy = tot[7], mxz = tot[8], myz = tot[9];
  double quad[6] = {2 * m200 - m020 - m002, 2 * m020 - m200 - m002, 2 * m002 - m200 - m020,
                    3 * mxy, 3 * mxz, 3 * myz};
  double bx = mp.c[0], by = mp.c[1], bz = mp.c[2];
  double b2 = bx * bx + by * by + bz * bz;
  double shift[6] = {q * (3 * bx * bx - b2), q * (3 * by * by - b2), q * (3 * bz * bz - b2),
                     3 * q * bx * by, 3 * q * bx * bz, 3 * q * by * bz};
  for (int r = 0; r < 6; ++r) mp.quad[r] = quad[r] - shift[r];
  return mp;
}

// potential(mp, x, y, z) (src/poisson.jl:198-206)
inline double mp_potential(const Multipole& mp, double x, double y, double z) {
  double px = x - mp.c[0], py = y - mp.c[1], pz = z - mp.c[2];
  double r2 = px * px + py * py + pz * pz;
  double invr = 1.0 / std::sqrt(r2);
  double quad = mp.quad[0] * px * px + mp.quad[1] * py * py + mp.quad[2] * pz * pz +
                2 * (mp.quad[3] * px * py + mp.quad[4] * px * pz + mp.quad[5] * py * pz);
  double i5 = invr * invr * invr * invr * invr;
  return mp.q * invr + quad * i5 / 2;
}

inline bool on_face(int i, int j, int k, int n) {
  return i == 0 || j == 0 || k == 0 || i == n - 1 || j == n - 1 || k == n - 1;
}

// solve_interior! (src/poisson.jl:366-372, rhs 275-294)
void solve_interior(double* phi, const double* rho, const orc_level& L) {
  int n = L.n, ni = n - 2;
  size_t tot = (size_t)ni * ni * ni;
  std::vector<double> rhs(tot), w1(tot), w2(tot);
  const double c = -4 * PI;
  const double* D = L.lap;
#pragma omp parallel for schedule(static)
  for (int t = 0; t < ni * ni; ++t) {
    int j = t % ni, k = t / ni;
    double dyl = D[(j + 1) * n + 0], dyr = D[(j + 1) * n + n - 1];
    double dzl = D[(k + 1) * n + 0], dzr = D[(k + 1) * n + n - 1];
    for (int i = 0; i < ni; ++i) {
      auto P = [&](int a, int b, int cc) { return phi[a + (size_t)n * (b + (size_t)n * cc)]; };
      rhs[i + (size_t)ni * t] = c * rho[(i + 1) + (size_t)n * ((j + 1) + (size_t)n * (k + 1))] -
          D[(i + 1) * n + 0] * P(0, j + 1, k + 1) - D[(i + 1) * n + n - 1] * P(n - 1, j + 1, k + 1) -
          dyl * P(i + 1, 0, k + 1) - dyr * P(i + 1, n - 1, k + 1) -
          dzl * P(i + 1, j + 1, 0) - dzr * P(i + 1, j + 1, n - 1);
    }
  }
  tensor_solve(rhs.data(), rhs.data(), L, w1.data(), w2.data());
#pragma omp parallel for schedule(static)
  for (int t = 0; t < ni * ni; ++t) {
    int j = t % ni, k = t / ni;
    for (int i = 0; i < ni; ++i)
      phi[(i + 1) + (size_t)n * ((j + 1) + (size_t)n * (k + 1))] = rhs[i + (size_t)ni * t];
  }
}

void spline_coefficients(double* c, const double* f, const orc_level& L) {
  size_t tot = (size_t)L.n * L.n * L.n;
  std::vector<double> work(tot);
  apply_all_rotating(c, L.sinv, f, work.data(), L.n);
}

// nested poisson! (src/poisson.jl:427-436)
void poisson_nested(double* phif, double* phic, const double* rhof, const double* rhoc,
                    const orc_level& F, const orc_level& C) {
  int nc = C.n, nf = F.n;
  // coarse: multipole faces, interior zero (src/poisson.jl:250-260, 351-354)
  Multipole mp = multipole(rhoc, C);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nc; ++k)
    for (int j = 0; j < nc; ++j)
      for (int i = 0; i < nc; ++i) {
        size_t t = i + (size_t)nc * (j + (size_t)nc * k);
        phic[t] = on_face(i, j, k, nc) ? mp_potential(mp, C.colloc[i], C.colloc[j], C.colloc[k]) : 0.0;
      }
  solve_interior(phic, rhoc, C);
  // fine: faces from the coarse spline (src/poisson.jl:383-413)
  std::vector<double> coefs((size_t)nc * nc * nc);
  spline_coefficients(coefs.data(), phic, C);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nf; ++k)
    for (int j = 0; j < nf; ++j)
      for (int i = 0; i < nf; ++i) {
        size_t t = i + (size_t)nf * (j + (size_t)nf * k);
        double v = 0.0;
        if (on_face(i, j, k, nf) &&
            !spline_potential(C.knots, C.nk, coefs.data(), nc, F.colloc[i], F.colloc[j], F.colloc[k], &v))
          v = NAN;
        phif[t] = v;
      }
  solve_interior(phif, rhof, F);
}

// ------------------------------------------------------------- mean field
// src/meanfield.jl:61-123, 356-386
const double XC_EXCHANGE = -std::cbrt(3 / PI);
const double XC_CORRELATION = -0.0333;
const double XC_CORRELATION_SCALE = 11.4 * std::cbrt(4 * PI / 3);

inline double xc_potential(double rho) {
  double c = std::cbrt(rho);
  return XC_EXCHANGE * c + XC_CORRELATION * std::log1p(XC_CORRELATION_SCALE * c);
}
inline double sphere_potential(double Q, double R, double r) {
  return r < R ? -Q * (3 - (r / R) * (r / R)) / (2 * R) : -Q / r;
}

void effective_potential(double* csol, const double* rho, const orc_level& L, double nions, double radius) {
  int n = L.n;
  size_t tot = (size_t)n * n * n;
  std::vector<double> extra(tot), c(tot);
  const double* g = L.colloc;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        size_t t = i + (size_t)n * (j + (size_t)n * k);
        double r = std::sqrt(g[i] * g[i] + g[j] * g[j] + g[k] * g[k]);
        extra[t] = xc_potential(rho[t]) + sphere_potential(nions, radius, r);
      }
  spline_coefficients(c.data(), extra.data(), L);
  for (size_t t = 0; t < tot; ++t) csol[t] += c[t];
}

// total_charge (src/deposition.jl:213-257)
double total_charge(const double* rho, const orc_level& L) {
  int n = L.n;
  const double* p = L.dual;
  double s = 0;
  std::vector<double> part((size_t)n * n);
#pragma omp parallel for schedule(static)
  for (int t = 0; t < n * n; ++t) {
    int j = t % n, k = t / n;
    double a = 0;
    for (int i = 0; i < n; ++i) a += rho[i + (size_t)n * t] * p[i];
    part[t] = a * p[j] * p[k];
  }
  for (int t = 0; t < n * n; ++t) s += part[t];
  return s;
}

// ------------------------------------------------------------- projectile
// src/projectile.jl:79-111
const double GAUSS_SERIES[7] = {1.0 / 3, -1.0 / 10, 1.0 / 56, -1.0 / 432, 1.0 / 4224, -1.0 / 49920, 1.0 / 685440};
const double SQRT_2_OVER_PI = std::sqrt(2 / PI);

inline double gaussian_force_kernel(double r2, double sigma) {
  double u2 = r2 / (sigma * sigma);
  if (u2 <= 0.25) {
    double p = 0;
    for (int k = 6; k >= 0; --k) p = GAUSS_SERIES[k] + u2 * p;
    return SQRT_2_OVER_PI * p / (sigma * sigma * sigma);
  }
  double r = std::sqrt(r2);
  double x = r / (std::sqrt(2.0) * sigma);
  return (std::erf(x) - SQRT_2_OVER_PI * (r / sigma) * std::exp(-u2 / 2)) / (r2 * r);
}
inline double ball_force_kernel(double r2, double R) {
  return r2 > R * R ? 1.0 / (r2 * std::sqrt(r2)) : 1.0 / (R * R * R);
}

// ------------------------------------------------- FP32 discrete replicas
// These reproduce the reference kernels' Float32 arithmetic exactly: every
// operation is a separately rounded float op (no contraction).
inline int32_t round_even_i32(float x) { return (int32_t)std::nearbyintf(x); }

inline int32_t column_f32(float d, float spacing, int32_t nbdt, int32_t ncol) {
  float half = spacing * 0.5f;
  float v = (d + half) / spacing * (float)nbdt + 0.5f;
  int32_t c = (int32_t)std::floor(v) + 1;
  return std::min(std::max(c, (int32_t)1), ncol);
}

inline int32_t cell_key0(int32_t kx, int32_t ky, int32_t kz, int32_t nk) {
  kx = std::min(std::max(kx, 1), nk);
  ky = std::min(std::max(ky, 1), nk);
  kz = std::min(std::max(kz, 1), nk);
  return (kx - 1) + nk * ((ky - 1) + nk * (kz - 1));
}

// 0-based cell -> 1-based knots and stencil bases
inline void cell_knots(int32_t cell, int32_t nk, int32_t* kx, int32_t* ky, int32_t* kz) {
  *kx = cell % nk + 1; cell /= nk;
  *ky = cell % nk + 1; cell /= nk;
  *kz = cell + 1;
}

// stencil of the field kernel fits (src/kernels.jl:375-377)
inline bool field_fits(int32_t kx, int32_t ky, int32_t kz, int32_t n) {
  int32_t bx = 2 * kx - 5, by = 2 * ky - 5, bz = 2 * kz - 5;
  return bx >= 1 && by >= 1 && bz >= 1 && bx + 9 <= n && by + 9 <= n && bz + 9 <= n;
}
// stencil of the deposit fits (src/kernels.jl:106-117)
inline bool deposit_fits(int32_t kx, int32_t ky, int32_t kz, int32_t n) {
  int32_t bx = 2 * kx - 5, by = 2 * ky - 5, bz = 2 * kz - 5;
  return bx >= 0 && by >= 0 && bz >= 0 && bx + 8 <= n && by + 8 <= n && bz + 8 <= n;
}

// _locate_cell in float (src/kernels.jl:1069-1081); returns 1-based cell, 0 outside
inline int32_t locate_f32(const float* gt, int32_t ng, float x0, float invw,
                          const int32_t* cells, int32_t ncells, float x, float* w) {
  if (x < gt[0] || x > gt[ng - 1]) { *w = 0; return 0; }
  int32_t b = std::min((int32_t)std::floor((x - x0) * invw) + 1, ncells);
  int32_t c = cells[b - 1];
  int32_t lastc = ng - 1;
  while (c < lastc && gt[c] < x) ++c;
  *w = (gt[c] - x) / (gt[c] - gt[c - 1]);
  return c;
}

}  // namespace

extern "C" {

int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

// ---------------------------------------------------------------- tables
void orc_mode_product(double* dest, const double* A, const double* src, int n, long long m) {
  mode_product(dest, A, src, n, (size_t)m);
}
void orc_spline_coefficients(const orc_level* L, const double* f, double* c) { spline_coefficients(c, f, *L); }
double orc_total_charge(const orc_level* L, const double* rho) { return total_charge(rho, *L); }
void orc_tensor_solve(const orc_level* L, const double* B, double* X) {
  int ni = L->n - 2;
  size_t tot = (size_t)ni * ni * ni;
  std::vector<double> w1(tot), w2(tot);
  tensor_solve(X, B, *L, w1.data(), w2.data());
}
void orc_multipole(const orc_level* L, const double* rho, double out[10]) {
  Multipole mp = multipole(rho, *L);
  out[0] = mp.q;
  for (int d = 0; d < 3; ++d) out[1 + d] = mp.c[d];
  for (int r = 0; r < 6; ++r) out[4 + r] = mp.quad[r];
}
void orc_poisson(const orc_level* F, const orc_level* C, const double* rhof, const double* rhoc,
                 double* phif, double* phic) {
  poisson_nested(phif, phic, rhof, rhoc, *F, *C);
}
void orc_effective_potential(const orc_level* L, double* csol, const double* rho, double nions, double radius) {
  effective_potential(csol, rho, *L, nions, radius);
}
int orc_spline_field(const orc_level* L, const double* c, double px, double py, double pz, double E[3]) {
  return spline_field(L->knots, L->nk, c, L->n, px, py, pz, E) ? 1 : 0;
}
int orc_spline_potential(const orc_level* L, const double* c, double px, double py, double pz, double* v) {
  return spline_potential(L->knots, L->nk, c, L->n, px, py, pz, v) ? 1 : 0;
}
double orc_gaussian_force_kernel(double r2, double sigma) { return gaussian_force_kernel(r2, sigma); }

// ------------------------------------------------------------------ sort
// cellsort! (src/sorting.jl:163-204): stable counting sort on the clamped
// cell of (k).  perm[s] is the 0-based index of the s-th sorted particle;
// occupied holds 0-based cells in increasing order; bounds[0]=0..bounds[nocc]=N.
int orc_cellsort(long long N, const int32_t* knode, int32_t nk, int32_t* keys, int32_t* perm,
                 int32_t* occupied, int32_t* bounds) {
  size_t ncell = (size_t)nk * nk * nk;
  const int32_t *kx = knode, *ky = knode + N, *kz = knode + 2 * N;
  std::vector<int32_t> cnt(ncell, 0);
  for (long long i = 0; i < N; ++i) {
    keys[i] = cell_key0(kx[i], ky[i], kz[i], nk);
    cnt[keys[i]]++;
  }
  std::vector<int32_t> off(ncell);
  int32_t a = 0, g = 0;
  bounds[0] = 0;
  for (size_t c = 0; c < ncell; ++c) {
    off[c] = a;
    if (!cnt[c]) continue;
    occupied[g++] = (int32_t)c;
    a += cnt[c];
    bounds[g] = a;
  }
  for (long long i = 0; i < N; ++i) perm[off[keys[i]]++] = (int32_t)i;
  return g;
}

// Out-of-stencil list over sorted slots (src/kernels.jl:1041-1058), in
// increasing slot order.
long long orc_outside(long long N, const int32_t* knode, int32_t n, int32_t* outlist) {
  long long c = 0;
  for (long long s = 0; s < N; ++s)
    if (!field_fits(knode[s], knode[N + s], knode[2 * N + s], n)) outlist[c++] = (int32_t)s;
  return c;
}

// _columns_kernel! (src/kernels.jl:754-779) in exact Float32.  Returns nout.
long long orc_columns(long long N, const int32_t* knode, const float* delta, float x0, float h,
                      float lo, float hi, float spacing, int32_t nbdt, int32_t ncol, int32_t* cols) {
  long long nout = 0;
  for (long long s = 0; s < N; ++s) {
    bool inside = true;
    for (int d = 0; d < 3; ++d) {
      float p = x0 + (float)(knode[d * N + s] - 1) * h + delta[d * N + s];
      inside = inside && (lo <= p) && (p <= hi);
    }
    if (inside) {
      for (int d = 0; d < 3; ++d) cols[d * N + s] = column_f32(delta[d * N + s], spacing, nbdt, ncol);
    } else {
      cols[s] = cols[N + s] = cols[2 * N + s] = 1;
      ++nout;
    }
  }
  return nout;
}

// _deposit_sorted_kernel! (src/kernels.jl:601-726) accumulated in float64,
// then the renormalisation of deposit_smoothed!(..., acc) (src/accelerator.jl:554-557).
// Returns the charge before scaling.
// The same deposit without the renormalisation (the raw density, which the
// shards of a sharded step sum); returns its total charge.
double orc_deposit_sorted_raw(const orc_level* F, const orc_smoothing* sm, long long N,
                              const int32_t* cols, const int32_t* occupied, const int32_t* bounds,
                              int32_t nocc, double* rho);

double orc_deposit_sorted(const orc_level* F, const orc_smoothing* sm, long long N,
                          const int32_t* cols, const int32_t* occupied, const int32_t* bounds,
                          int32_t nocc, long long nout, double charge, double* rho) {
  double q = orc_deposit_sorted_raw(F, sm, N, cols, occupied, bounds, nocc, rho);
  const size_t tot = (size_t)F->n * F->n * F->n;
  double scale = (double)(N - nout) * charge / q;
  for (size_t t = 0; t < tot; ++t) rho[t] *= scale;
  return q;
}

double orc_deposit_sorted_raw(const orc_level* F, const orc_smoothing* sm, long long N,
                              const int32_t* cols, const int32_t* occupied, const int32_t* bounds,
                              int32_t nocc, double* rho) {
  int n = F->n, nk = F->nk;
  size_t tot = (size_t)n * n * n;
  std::fill(rho, rho + tot, 0.0);
  const double* nodes = sm->nodes;
  for (int g = 0; g < nocc; ++g) {
    int32_t kx, ky, kz;
    cell_knots(occupied[g], nk, &kx, &ky, &kz);
    if (!deposit_fits(kx, ky, kz, n)) continue;
    int32_t bx = 2 * kx - 5, by = 2 * ky - 5, bz = 2 * kz - 5;
    double acc[512] = {0};
    for (int32_t s = bounds[g]; s < bounds[g + 1]; ++s) {
      const double* vx = nodes + 8 * (size_t)(cols[s] - 1);
      const double* vy = nodes + 8 * (size_t)(cols[N + s] - 1);
      const double* vz = nodes + 8 * (size_t)(cols[2 * N + s] - 1);
      for (int c = 0; c < 8; ++c)
        for (int b = 0; b < 8; ++b) {
          double w = vy[b] * vz[c];
          for (int a = 0; a < 8; ++a) acc[a + 8 * (b + 8 * c)] += vx[a] * w;
        }
    }
    for (int c = 0; c < 8; ++c)
      for (int b = 0; b < 8; ++b)
        for (int a = 0; a < 8; ++a)
          rho[(bx + a) + (size_t)n * ((by + b) + (size_t)n * (bz + c))] += acc[a + 8 * (b + 8 * c)];
  }
  return total_charge(rho, *F);
}

// Coarse CIC deposit of the device path (src/kernels.jl:1207-1273,
// src/devicemesh.jl:93-106): position and cell in Float32 as the kernel,
// weights and sums in float64.
void orc_deposit_cic_device(const orc_level* C, long long N, const int32_t* knode, const float* delta,
                            float x0f, float hf, double charge, double* rho) {
  int n = C->n;
  size_t tot = (size_t)n * n * n;
  std::fill(rho, rho + tot, 0.0);
  std::vector<float> gt(n);
  for (int i = 0; i < n; ++i) gt[i] = (float)C->colloc[i];
  float lx0 = (float)C->loc_x0, linv = (float)C->loc_invw;
  for (long long s = 0; s < N; ++s) {
    int32_t ii[3]; float w[3];
    bool ok = true;
    for (int d = 0; d < 3; ++d) {
      float p = x0f + (float)(knode[d * N + s] - 1) * hf + delta[d * N + s];
      ii[d] = locate_f32(gt.data(), n, lx0, linv, C->loc_cells, C->loc_ncell, p, &w[d]);
      ok = ok && ii[d] > 0;
    }
    if (!ok) continue;
    double ax = w[0], ay = w[1], az = w[2];
    double bx = 1.0f - w[0], by = 1.0f - w[1], bz = 1.0f - w[2];
    int i = ii[0] - 1, j = ii[1] - 1, k = ii[2] - 1;
    auto R = [&](int a, int b, int c) -> double& { return rho[a + (size_t)n * (b + (size_t)n * c)]; };
    R(i, j, k) += ax * ay * az;         R(i, j, k + 1) += ax * ay * bz;
    R(i, j + 1, k) += ax * by * az;     R(i, j + 1, k + 1) += ax * by * bz;
    R(i + 1, j, k) += bx * ay * az;     R(i + 1, j, k + 1) += bx * ay * bz;
    R(i + 1, j + 1, k) += bx * by * az; R(i + 1, j + 1, k + 1) += bx * by * bz;
  }
  const double* dl = C->dlen;
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) rho[i + (size_t)n * (j + (size_t)n * k)] *= charge / (dl[i] * dl[j] * dl[k]);
}

// Forces of the device path over a sorted packed cloud
// (src/kernels.jl:339-470 + the host tail src/accelerator.jl:679-733),
// continuous arithmetic in float64.  force is SoA [3N].  red[4] receives the
// projectile sums.  Returns the out-of-stencil count.
long long orc_forces_device(const orc_level* F, const orc_level* C, const orc_smoothing* sm,
                            long long N, const int32_t* knode, const float* delta,
                            const int32_t* occupied, const int32_t* bounds, int32_t nocc,
                            const double* csolf, const double* csolc, double w,
                            double x0, double h, const orc_projectile* pr, double* force, double red[4]) {
  int n = F->n, nk = F->nk, nc = C->n;
  float spf = (float)sm->spacing;
  int32_t nbdt = sm->nbdt, ncol = nbdt + 1;
  const double *ov = sm->overlap, *gr = sm->gradient;
  double coef = pr && pr->active ? -w * pr->charge : 0.0;
  double sig = pr ? pr->gauss_sigma : 1.0;
  // the CPU path's softening, projectile_forces! with BallSoftening
  // (src/projectile.jl:203-232): the ball for every particle, both ways
  const bool ball = pr && pr->softening == 1;
  double rx = 0, ry = 0, rz = 0, re = 0;
  long long nouts = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : rx, ry, rz, re, nouts)
  for (int g = 0; g < nocc; ++g) {
    int32_t kx, ky, kz;
    cell_knots(occupied[g], nk, &kx, &ky, &kz);
    bool ok = field_fits(kx, ky, kz, n);
    int32_t bx = 2 * kx - 5, by = 2 * ky - 5, bz = 2 * kz - 5;  // 1-based
    for (int32_t s = bounds[g]; s < bounds[g + 1]; ++s) {
      double fx = 0, fy = 0, fz = 0;
      float d0 = delta[s], d1 = delta[N + s], d2 = delta[2 * N + s];
      if (ok) {
        int32_t cx = column_f32(d0, spf, nbdt, ncol), cy = column_f32(d1, spf, nbdt, ncol),
                cz = column_f32(d2, spf, nbdt, ncol);
        const double *ox = ov + 10 * (size_t)(cx - 1), *gx = gr + 10 * (size_t)(cx - 1);
        const double *oy = ov + 10 * (size_t)(cy - 1), *gy = gr + 10 * (size_t)(cy - 1);
        const double *oz = ov + 10 * (size_t)(cz - 1), *gz = gr + 10 * (size_t)(cz - 1);
        double sx = 0, sy = 0, sz = 0;
        for (int kk = 0; kk < 10; ++kk) {
          for (int jj = 0; jj < 10; ++jj) {
            const double* col = csolf + (size_t)(bx - 1) + (size_t)n * ((by - 1 + jj) + (size_t)n * (bz - 1 + kk));
            double dxp = 0, val = 0;
            for (int ii = 0; ii < 10; ++ii) { dxp = std::fma(col[ii], gx[ii], dxp); val = std::fma(col[ii], ox[ii], val); }
            sx = std::fma(oy[jj] * oz[kk], dxp, sx);
            sy = std::fma(gy[jj] * oz[kk], val, sy);
            sz = std::fma(oy[jj] * gz[kk], val, sz);
          }
        }
        fx = -w * sx; fy = -w * sy; fz = -w * sz;
      } else {
        // host tail: coarse spline field (escaped = 0 outside both grids)
        ++nouts;
        double px = x0 + (double)(knode[s] - 1) * h + (double)d0;
        double py = x0 + (double)(knode[N + s] - 1) * h + (double)d1;
        double pz = x0 + (double)(knode[2 * N + s] - 1) * h + (double)d2;
        double E[3];
        if (spline_field(C->knots, C->nk, csolc, nc, px, py, pz, E)) { fx = w * E[0]; fy = w * E[1]; fz = w * E[2]; }
        if (coef != 0) {
          double dx = pr->pos[0] - px, dy = pr->pos[1] - py, dz = pr->pos[2] - pz;
          double m = -w * pr->charge * ball_force_kernel(dx * dx + dy * dy + dz * dz, pr->ball_radius);
          fx -= m * dx; fy -= m * dy; fz -= m * dz;
        }
      }
      if (coef != 0 && ball) {
        // the particle's own position (the cell's, when the stencil fits)
        double px = x0 + (double)(knode[s] - 1) * h + (double)d0;
        double py = x0 + (double)(knode[N + s] - 1) * h + (double)d1;
        double pz = x0 + (double)(knode[2 * N + s] - 1) * h + (double)d2;
        double dx = pr->pos[0] - px, dy = pr->pos[1] - py, dz = pr->pos[2] - pz;
        double d2s = dx * dx + dy * dy + dz * dz;
        double mm = coef * ball_force_kernel(d2s, pr->ball_radius);
        if (ok) { fx -= mm * dx; fy -= mm * dy; fz -= mm * dz; }  // the tail took its own above
        rx += mm * dx; ry += mm * dy; rz += mm * dz;
        re += sphere_potential(1.0, pr->ball_radius, std::sqrt(d2s));
      } else if (coef != 0) {
        // fused projectile, position rebuilt from the (clamped) cell
        double px = x0 + (double)(kx - 1) * h + (double)d0;
        double py = x0 + (double)(ky - 1) * h + (double)d1;
        double pz = x0 + (double)(kz - 1) * h + (double)d2;
        double dx = pr->pos[0] - px, dy = pr->pos[1] - py, dz = pr->pos[2] - pz;
        double d2s = dx * dx + dy * dy + dz * dz;
        double mm = coef * gaussian_force_kernel(d2s, sig);
        if (ok) { fx -= mm * dx; fy -= mm * dy; fz -= mm * dz; }
        rx += mm * dx; ry += mm * dy; rz += mm * dz;
        double r = std::sqrt(d2s);
        re += r < 1.0e-4 * sig ? 0.7978845608 / sig : std::erf(r / 1.4142135624 / sig) / r;
      }
      force[s] = fx; force[N + s] = fy; force[2 * N + s] = fz;
    }
  }
  red[0] = rx; red[1] = ry; red[2] = rz; red[3] = re;
  return nouts;
}

// projectile_forces!(cloud, acc, proj, jel) (src/accelerator.jl:746-756)
void orc_projectile_force_device(const orc_projectile* pr, double w, double nions, double jel_radius,
                                 const double red[4], double F[3], double* e_el, double* e_jel) {
  double r2 = pr->pos[0] * pr->pos[0] + pr->pos[1] * pr->pos[1] + pr->pos[2] * pr->pos[2];
  double q = pr->charge;
  double modf = r2 > jel_radius * jel_radius ? nions * q / std::pow(r2, 1.5) : q / 64.0;
  for (int d = 0; d < 3; ++d) F[d] = modf * pr->pos[d] + red[d];
  *e_el = w * q * red[3];
  *e_jel = q * sphere_potential(nions, jel_radius, std::sqrt(r2));
}

// step!(proj, force, dt) (src/projectile.jl:298-304)
void orc_projectile_step(orc_projectile* pr, const double F[3], double dt) {
  for (int d = 0; d < 3; ++d) {
    double nw = 2 * pr->pos[d] - pr->prev[d] + (dt * dt / pr->mass) * F[d];
    pr->vel[d] = (nw - pr->prev[d]) / (2 * dt);
    pr->prev[d] = pr->pos[d];
    pr->pos[d] = nw;
  }
}

// _verlet_packed_kernel! (src/kernels.jl:985-1025) with the Float32 state
// update replicated exactly; diagnostics in float64.
void orc_verlet_packed(long long N, int32_t* k, float* d, int32_t* pk, float* pd, const float* force,
                       float a, float h, float x0, double pfac, float r2max, double inv2M, double diag[5]) {
  double ek = 0, eo = 0, lx = 0, ly = 0, lz = 0;
#pragma omp parallel for schedule(static) reduction(+ : ek, eo, lx, ly, lz)
  for (long long i = 0; i < N; ++i) {
    float q[3], pm[3];
    int32_t kn[3]; float dn[3];
    for (int c = 0; c < 3; ++c) {
      int32_t kq = k[c * N + i], ok = pk[c * N + i];
      float dq = d[c * N + i], od = pd[c * N + i], f = force[c * N + i];
      int32_t kk = 2 * kq - ok;
      float t1 = 2.0f * dq - od;
      float t2 = a * f;
      float dd = t1 + t2;
      int32_t m = round_even_i32(dd / h);
      kk += m;
      float mh = (float)m * h;
      dd = dd - mh;
      float gap = (float)(kk - ok) * h + (dd - od);
      kn[c] = kk; dn[c] = dd;
      pm[c] = gap;
      float qa = x0 + (float)(kq - 1) * h;
      q[c] = qa + dq;
    }
    double px = (double)pm[0] * pfac, py = (double)pm[1] * pfac, pz = (double)pm[2] * pfac;
    double e = (px * px + py * py + pz * pz) * inv2M;
    ek += e;
    float r2 = q[0] * q[0] + q[1] * q[1];
    r2 = r2 + q[2] * q[2];
    if (r2 > r2max) eo += e;
    lx += q[1] * pz - q[2] * py;
    ly += q[2] * px - q[0] * pz;
    lz += q[0] * py - q[1] * px;
    for (int c = 0; c < 3; ++c) {
      pk[c * N + i] = k[c * N + i];
      pd[c * N + i] = d[c * N + i];
      k[c * N + i] = kn[c];
      d[c * N + i] = dn[c];
    }
  }
  diag[0] = ek; diag[1] = eo; diag[2] = lx; diag[3] = ly; diag[4] = lz;
}

// enclosed_charge (src/projectile.jl:243-247) on a packed cloud
double orc_enclosed_charge_packed(long long N, const int32_t* k, const float* d, double x0, double h,
                                  double w, const double P[3], double radius) {
  long long cnt = 0;
  double r2 = radius * radius;
#pragma omp parallel for schedule(static) reduction(+ : cnt)
  for (long long i = 0; i < N; ++i) {
    double s = 0;
    for (int c = 0; c < 3; ++c) {
      double p = x0 + (double)(k[c * N + i] - 1) * h + (double)d[c * N + i];
      double dd = p - P[c];
      s += dd * dd;
    }
    if (s < r2) ++cnt;
  }
  return w * (double)cnt;
}

// ==================================================== reference CPU path
// deposit_smoothed! (src/fields.jl:264-297) with per-thread buffers
// (src/deposition.jl:59-133).  positions AoS [3N].  Returns nout.
long long orc_deposit_smoothed_host(const orc_level* F, const orc_smoothing* sm, long long N,
                                    const double* pos, double charge, double* rho) {
  int n = F->n, nk = F->nk;
  size_t tot = (size_t)n * n * n;
  const double* g = F->knots;
  double half = sm->spacing / 2;
  double blo = g[1] + half, bhi = g[nk - 2] - half;
  int nt = omp_get_max_threads();
  nt = (int)std::max<long long>(1, std::min<long long>(nt, N));
  std::vector<std::vector<double>> buf(nt, std::vector<double>(tot, 0.0));
  std::vector<long long> nouts(nt, 0);
#pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    long long base = N / nt, rem = N % nt;
    long long start = t * base + std::min<long long>(t, rem);
    long long stop = start + base + (t < rem ? 1 : 0);
    double* dest = buf[t].data();
    for (long long i = start; i < stop; ++i) {
      const double* p = pos + 3 * i;
      bool in = true;
      for (int d = 0; d < 3; ++d) in = in && blo <= p[d] && p[d] <= bhi;
      if (!in) { nouts[t]++; continue; }
      int ci[3], col[3], base_[3];
      for (int d = 0; d < 3; ++d) {
        ci[d] = nearest_knot(g, nk, p[d]);
        col[d] = (int)std::floor((p[d] - g[ci[d] - 1] + sm->spacing / 2) / sm->spacing * sm->nbdt + 0.5) + 1;
        base_[d] = 2 * ci[d] - 5;
      }
      const double* gx = sm->nodes + 8 * (size_t)(col[0] - 1);
      const double* gy = sm->nodes + 8 * (size_t)(col[1] - 1);
      const double* gz = sm->nodes + 8 * (size_t)(col[2] - 1);
      for (int kk = 0; kk < 8; ++kk)
        for (int jj = 0; jj < 8; ++jj) {
          double c = gy[jj] * gz[kk];
          size_t row = (size_t)n * ((base_[1] + jj) + (size_t)n * (base_[2] + kk));
          for (int ii = 0; ii < 8; ++ii) dest[base_[0] + ii + row] += gx[ii] * c;
        }
    }
  }
  std::copy(buf[0].begin(), buf[0].end(), rho);
  for (int t = 1; t < nt; ++t)
    for (size_t e = 0; e < tot; ++e) rho[e] += buf[t][e];
  long long nout = 0;
  for (int t = 0; t < nt; ++t) nout += nouts[t];
  for (size_t e = 0; e < tot; ++e) rho[e] *= charge;
  double q = total_charge(rho, *F);
  double scale = (double)(N - nout) * charge / q;
  for (size_t e = 0; e < tot; ++e) rho[e] *= scale;
  return nout;
}

// deposit! (src/deposition.jl:146-184), LocateTable lookup in float64.
long long orc_deposit_cic_host(const orc_level* C, long long N, const double* pos, double charge, double* rho) {
  int n = C->n;
  size_t tot = (size_t)n * n * n;
  const double* gt = C->colloc;
  int nt = omp_get_max_threads();
  nt = (int)std::max<long long>(1, std::min<long long>(nt, N));
  std::vector<std::vector<double>> buf(nt, std::vector<double>(tot, 0.0));
  std::vector<long long> nouts(nt, 0);
  auto locate = [&](double x, double* w) -> int {
    if (x < gt[0] || x > gt[n - 1]) return 0;
    int b = std::min((int)std::floor((x - C->loc_x0) * C->loc_invw) + 1, (int)C->loc_ncell);
    int c = C->loc_cells[b - 1];
    while (c < n - 1 && gt[c] < x) ++c;
    *w = (gt[c] - x) / (gt[c] - gt[c - 1]);
    return c;
  };
#pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    long long base = N / nt, rem = N % nt;
    long long start = t * base + std::min<long long>(t, rem);
    long long stop = start + base + (t < rem ? 1 : 0);
    double* dest = buf[t].data();
    for (long long s = start; s < stop; ++s) {
      double w[3]; int ii[3];
      bool ok = true;
      for (int d = 0; d < 3; ++d) { ii[d] = locate(pos[3 * s + d], &w[d]); ok = ok && ii[d] > 0; }
      if (!ok) { nouts[t]++; continue; }
      double ax = w[0], ay = w[1], az = w[2], bx = 1 - ax, by = 1 - ay, bz = 1 - az;
      int i = ii[0] - 1, j = ii[1] - 1, k = ii[2] - 1;
      auto R = [&](int a, int b, int c) -> double& { return dest[a + (size_t)n * (b + (size_t)n * c)]; };
      R(i, j, k) += ax * ay * az;         R(i, j, k + 1) += ax * ay * bz;
      R(i, j + 1, k) += ax * by * az;     R(i, j + 1, k + 1) += ax * by * bz;
      R(i + 1, j, k) += bx * ay * az;     R(i + 1, j, k + 1) += bx * ay * bz;
      R(i + 1, j + 1, k) += bx * by * az; R(i + 1, j + 1, k + 1) += bx * by * bz;
    }
  }
  std::copy(buf[0].begin(), buf[0].end(), rho);
  for (int t = 1; t < nt; ++t)
    for (size_t e = 0; e < tot; ++e) rho[e] += buf[t][e];
  const double* dl = C->dlen;
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) rho[i + (size_t)n * (j + (size_t)n * k)] *= charge / (dl[i] * dl[j] * dl[k]);
  long long nout = 0;
  for (int t = 0; t < nt; ++t) nout += nouts[t];
  return nout;
}

// forces! host (src/fields.jl:490-524).  pos/force AoS [3N].  Returns n outside the margin.
long long orc_forces_host(const orc_level* F, const orc_level* C, const orc_smoothing* sm, long long N,
                          const double* pos, const double* csolf, const double* csolc, double w,
                          long long escaped, double* force) {
  int n = F->n, nk = F->nk;
  const double* g = F->knots;
  double lo = g[2], hi = g[nk - 3];
  double w2 = w * w;
  long long nout = 0;
#pragma omp parallel for schedule(static) reduction(+ : nout)
  for (long long i = 0; i < N; ++i) {
    const double* p = pos + 3 * i;
    double* f = force + 3 * i;
    bool in = true;
    for (int d = 0; d < 3; ++d) in = in && lo < p[d] && p[d] < hi;
    if (in) {
      int ci[3], col[3], b[3];
      for (int d = 0; d < 3; ++d) {
        ci[d] = nearest_knot(g, nk, p[d]);
        b[d] = 2 * ci[d] - 5;
        col[d] = (int)std::floor((p[d] - g[ci[d] - 1] + sm->spacing / 2) / sm->spacing * sm->nbdt + 0.5) + 1;
      }
      const double *ox = sm->overlap + 10 * (size_t)(col[0] - 1), *gx = sm->gradient + 10 * (size_t)(col[0] - 1);
      const double *oy = sm->overlap + 10 * (size_t)(col[1] - 1), *gy = sm->gradient + 10 * (size_t)(col[1] - 1);
      const double *oz = sm->overlap + 10 * (size_t)(col[2] - 1), *gz = sm->gradient + 10 * (size_t)(col[2] - 1);
      double fx = 0, fy = 0, fz = 0;
      for (int kk = 0; kk < 10; ++kk) {
        int k = b[2] + kk - 1;
        for (int jj = 0; jj < 10; ++jj) {
          int j = b[1] + jj - 1;
          const double* col_ = csolf + (size_t)(b[0] - 1) + (size_t)n * (j + (size_t)n * k);
          double dxp = 0, val = 0;
          for (int ii = 0; ii < 10; ++ii) { dxp = std::fma(col_[ii], gx[ii], dxp); val = std::fma(col_[ii], ox[ii], val); }
          fx = std::fma(oy[jj] * oz[kk], dxp, fx);
          fy = std::fma(gy[jj] * oz[kk], val, fy);
          fz = std::fma(oy[jj] * gz[kk], val, fz);
        }
      }
      f[0] = w * -fx; f[1] = w * -fy; f[2] = w * -fz;
    } else {
      ++nout;
      double E[3];
      if (spline_field(C->knots, C->nk, csolc, C->n, p[0], p[1], p[2], E)) {
        f[0] = w * E[0]; f[1] = w * E[1]; f[2] = w * E[2];
      } else {
        double r3 = std::pow(p[0] * p[0] + p[1] * p[1] + p[2] * p[2], 1.5);
        double m = -w2 * (double)escaped / r3;
        f[0] = m * p[0]; f[1] = m * p[1]; f[2] = m * p[2];
      }
    }
  }
  return nout;
}

// smoothed_potential (src/fields.jl:405-429): the 10^3 overlap-weighted sum
// of csol around p's nearest knots.
double smoothed_potential(const orc_level* F, const orc_smoothing* sm, const double* csolf, const double* p) {
  const double* g = F->knots;
  const int n = F->n, nk = F->nk;
  int b[3], col[3];
  for (int d = 0; d < 3; ++d) {
    const int ci = nearest_knot(g, nk, p[d]);
    b[d] = 2 * ci - 5;
    col[d] = (int)std::floor((p[d] - g[ci - 1] + sm->spacing / 2) / sm->spacing * sm->nbdt + 0.5) + 1;
  }
  const double* ox = sm->overlap + 10 * (size_t)(col[0] - 1);
  const double* oy = sm->overlap + 10 * (size_t)(col[1] - 1);
  const double* oz = sm->overlap + 10 * (size_t)(col[2] - 1);
  double phi = 0;
  for (int kk = 0; kk < 10; ++kk) {
    const int k = b[2] + kk - 1;
    for (int jj = 0; jj < 10; ++jj) {
      const int j = b[1] + jj - 1;
      const double wyz = oy[jj] * oz[kk];
      const double* row = csolf + (size_t)(b[0] - 1) + (size_t)n * (j + (size_t)n * k);
      double s = 0;
      for (int ii = 0; ii < 10; ++ii) s += row[ii] * ox[ii];
      phi += s * wyz;
    }
  }
  return phi;
}

extern "C" {

// interaction_energy (src/energy.jl:19-43): sum of w phi(p) over the
// particles, phi the smoothed fine potential inside the host margin, the
// coarse spline outside it, enclosed / r outside both.  pos AoS [3N].
double orc_interaction_energy(const orc_level* F, const orc_level* C, const orc_smoothing* sm, long long N,
                              const double* pos, const double* csolf, const double* csolc, double w,
                              double enclosed) {
  const double* g = F->knots;
  const double lo = g[2], hi = g[F->nk - 3];
  double total = 0;
#pragma omp parallel for schedule(static) reduction(+ : total)
  for (long long i = 0; i < N; ++i) {
    const double* p = pos + 3 * i;
    bool in = true;
    for (int d = 0; d < 3; ++d) in = in && lo < p[d] && p[d] < hi;
    double phi;
    if (in) {
      phi = smoothed_potential(F, sm, csolf, p);
    } else if (!spline_potential(C->knots, C->nk, csolc, C->n, p[0], p[1], p[2], &phi)) {
      phi = enclosed / std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    }
    total += w * phi;
  }
  return total;
}

}  // extern "C"

// projectile_forces! host (src/projectile.jl:203-232), ball softening, serial.
void orc_projectile_forces_host(long long N, const double* pos, double* force, const orc_projectile* pr,
                                double w, double nions, double jel_radius, double F[3], double* e_el, double* e_jel) {
  const double* P = pr->pos;
  double q = pr->charge, R = pr->ball_radius;
  double r2 = P[0] * P[0] + P[1] * P[1] + P[2] * P[2];
  double modf = r2 > jel_radius * jel_radius ? nions * q / std::pow(r2, 1.5) : q / 64.0;
  double fx = modf * P[0], fy = modf * P[1], fz = modf * P[2];
  *e_jel = q * sphere_potential(nions, jel_radius, std::sqrt(r2));
  double coef = -w * q, ee = 0;
  for (long long i = 0; i < N; ++i) {
    double dx = P[0] - pos[3 * i], dy = P[1] - pos[3 * i + 1], dz = P[2] - pos[3 * i + 2];
    double d2 = dx * dx + dy * dy + dz * dz;
    double m = coef * ball_force_kernel(d2, R);
    double f0 = m * dx, f1 = m * dy, f2 = m * dz;
    fx += f0; fy += f1; fz += f2;
    force[3 * i] -= f0; force[3 * i + 1] -= f1; force[3 * i + 2] -= f2;
    ee += w * sphere_potential(q, R, std::sqrt(d2));
  }
  F[0] = fx; F[1] = fy; F[2] = fz;
  *e_el = ee;
}

// step!(cloud, dt; rcmax) (src/particles.jl:205-250), chunked threads
void orc_verlet_host(long long N, double* pos, double* prev, const double* force, double dt, double M,
                     double rcmax, double diag[5]) {
  double acc = dt * dt / M, pfac = M / (2 * dt), r2max = rcmax * rcmax;
  int nt = omp_get_max_threads();
  nt = (int)std::max<long long>(1, std::min<long long>(nt, N));
  std::vector<double> part((size_t)nt * 5, 0.0);
#pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    long long base = N / nt, rem = N % nt;
    long long start = t * base + std::min<long long>(t, rem);
    long long stop = start + base + (t < rem ? 1 : 0);
    double ek = 0, eo = 0, a0 = 0, a1 = 0, a2 = 0;
    for (long long i = start; i < stop; ++i) {
      double* q = pos + 3 * i;
      double* o = prev + 3 * i;
      const double* f = force + 3 * i;
      double qn[3], p[3];
      for (int c = 0; c < 3; ++c) { qn[c] = 2 * q[c] - o[c] + acc * f[c]; p[c] = pfac * (qn[c] - o[c]); }
      double e = (p[0] * p[0] + p[1] * p[1] + p[2] * p[2]) / (2 * M);
      ek += e;
      if (q[0] * q[0] + q[1] * q[1] + q[2] * q[2] > r2max) eo += e;
      a0 += q[1] * p[2] - q[2] * p[1];
      a1 += q[2] * p[0] - q[0] * p[2];
      a2 += q[0] * p[1] - q[1] * p[0];
      for (int c = 0; c < 3; ++c) { o[c] = q[c]; q[c] = qn[c]; }
    }
    double* P = &part[(size_t)t * 5];
    P[0] = ek; P[1] = eo; P[2] = a0; P[3] = a1; P[4] = a2;
  }
  for (int r = 0; r < 5; ++r) diag[r] = 0;
  for (int t = 0; t < nt; ++t)
    for (int r = 0; r < 5; ++r) diag[r] += part[(size_t)t * 5 + r];
}

double orc_enclosed_charge_host(long long N, const double* pos, double w, const double P[3], double radius) {
  long long cnt = 0;
  double r2 = radius * radius;
#pragma omp parallel for schedule(static) reduction(+ : cnt)
  for (long long i = 0; i < N; ++i) {
    double dx = pos[3 * i] - P[0], dy = pos[3 * i + 1] - P[1], dz = pos[3 * i + 2] - P[2];
    if (dx * dx + dy * dy + dz * dz < r2) ++cnt;
  }
  return w * (double)cnt;
}

}  // extern "C"

// ------------------------------------------------------------- sampling
// The seeded initial cloud, so that the CPU baseline needs nothing of the
// product.  ran2 as the thesis has it (src/random.jl:31-90): L'Ecuyer's
// two multiplicative congruential generators combined through a 32-entry
// Bays-Durham table; IQ1 = 3668 (53668 when `consistent`), so that the
// Schrage product k*IR1 wraps round 32 bits as the Fortran's does.
namespace {

struct OrcRan2 {
  static constexpr int32_t M1 = 2147483563, M2 = 2147483399;
  int32_t q1, s1, s2, last, table[32];

  static int32_t wrap(int64_t v) { return (int32_t)(uint32_t)(uint64_t)v; }
  // a*x mod m by Schrage's factorisation, in wrapping 32-bit arithmetic
  static int32_t lcg(int32_t x, int32_t a, int32_t q, int32_t r, int32_t m) {
    const int32_t k = x / q;
    int32_t y = wrap((int64_t)wrap((int64_t)a * wrap((int64_t)x - (int64_t)k * q)) - (int64_t)wrap((int64_t)k * r));
    return y < 0 ? wrap((int64_t)y + m) : y;
  }
  OrcRan2(int32_t seed, bool consistent) {
    q1 = consistent ? 53668 : 3668;
    s1 = seed < 0 ? -seed : 1;
    if (s1 < 1) s1 = 1;
    s2 = s1;
    for (int j = 40; j >= 1; --j) {  // 8 warm-up draws, then the table from the top
      s1 = lcg(s1, 40014, q1, 12211, M1);
      if (j <= 32) table[j - 1] = s1;
    }
    last = table[0];
  }
  float uniform() {
    s1 = lcg(s1, 40014, q1, 12211, M1);
    s2 = lcg(s2, 40692, 52774, 3791, M2);
    const int32_t slot = last / (1 + (M1 - 2) / 32);
    last = wrap((int64_t)table[slot] - s2);
    table[slot] = s1;
    if (last < 1) last = wrap((int64_t)last + (M1 - 1));
    const float v = (1.0f / (float)M1) * (float)last;
    const float top = 1.0f - 1.2e-7f;
    return v < top ? v : top;
  }
};

// linear interpolation on [0, 1] sampled at n regular points (src/initial.jl:161-168)
double regular_interp(const double* v, int n, double u) {
  const int j = std::min((int)std::floor(u * (n - 1)) + 1, n - 1);
  const double a = (double)(j - 1) / (n - 1), b = (double)j / (n - 1);
  return v[j - 1] + (v[j] - v[j - 1]) * (u - a) / (b - a);
}

// a vector of length r in the direction (phi = 2 pi u1, cos theta = 2 u2 - 1) (src/initial.jl:323-328)
void sphere_point(double r, double u1, double u2, double* out) {
  const double c = 2 * u2 - 1, s = std::sqrt(1 - c * c), ph = 2 * PI * u1;
  out[0] = r * std::cos(ph) * s;
  out[1] = r * std::sin(ph) * s;
  out[2] = r * c;
}

}  // namespace

extern "C" {

// sample_thomas_fermi (src/initial.jl:94-113, 184-203): per particle six
// uniforms -- the radius from the quantile table, its direction, the Fermi
// momentum p_F(r) = (3 pi^2 rho(r))^(1/3) times cbrt(u) (uniform in the
// Fermi ball), its direction -- momenta times the weight.  AoS 3*npart.
void orc_sample_thomas_fermi(const double* quantiles, int32_t nq, const double* density, int32_t nr, double rmax,
                             long long npart, double weight, int32_t seed, int32_t consistent, double* pos,
                             double* mom) {
  OrcRan2 g(seed, consistent != 0);
  const double kf = std::cbrt(3 * (PI * PI));
  for (long long i = 0; i < npart; ++i) {
    double u[6];
    for (int j = 0; j < 6; ++j) u[j] = (double)g.uniform();
    const double r = regular_interp(quantiles, nq, u[0]);
    sphere_point(r, u[1], u[2], pos + 3 * i);
    const double rho = regular_interp(density, nr, r / rmax);
    const double p = std::cbrt(u[3]) * kf * std::cbrt(rho);
    sphere_point(p * weight, u[4], u[5], mom + 3 * i);
  }
}

}  // extern "C"
