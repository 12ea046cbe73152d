// The nested tensor-product Poisson solve and the spline-coefficient
// conversions, on the device.
//
// Every product of the chain is the reference's rotating mode product
// (src/tensorsolver.jl:217-223):
//
//     dest[p + m*i'] = sum_i A[i', i] * src[i + n*p],    m = n^2,
//
// which applies A along the first axis and leaves the axes rotated, so three
// of them restore the order.  One FP32 kernel does all of them; the stages
// around the products are fused into its load or its store:
//
//   load  : plain | Poisson right-hand side with the Dirichlet lifting
//           (src/poisson.jl:275-294) | phi + V_xc(rho) + V_jel(r) (the mean
//           field, src/meanfield.jl:116-123, folded into the S^-1 of the
//           total potential: S^-1 phi + S^-1 extra = S^-1 (phi + extra))
//   store : plain | times 1/(lx+ly+lz) (src/tensorsolver.jl:291) | into the
//           interior of phi (src/kernels.jl:804-813)
//
// plus the multipole moments, the multipole faces of the coarse level
// (src/poisson.jl:55-206, src/kernels.jl:868-873) and the fine faces read
// from the coarse spline (src/kernels.jl:888-898).

#include "vlb_internal.cuh"

namespace vlb {

int grid_for(const Ctx& c, int64_t n, int threads, int per_sm);

namespace {

constexpr int kPT = 64;  // p columns per CTA

enum { EPI_PLAIN = 0, EPI_INVL = 1, EPI_PHI = 2 };

struct ProductArgs {
  float* dest;
  const float* AT;     // [n][npad]  A transposed, zero padded
  const float* src;
  int n, npad;
  long long m;
  const float* invl;   // EPI_INVL
};

// row stride of the staged src tile: >= n, 16-byte rows, and == 4 (mod 8)
// so that the 8 column groups of a warp read 8 different banks
__host__ __device__ __forceinline__ int tile_lds(int n) {
  int l = (n + 3) / 4 * 4;
  if (l % 8 == 0) l += 4;
  return l;
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// One CTA: all output rows i' (n padded to npad) for kPT consecutive columns
// p.  A^T and the src tile are staged with asynchronous copies (every copy in
// flight at once), then each thread accumulates an 8 x 8 block in registers.
template <int EPI>
__global__ void __launch_bounds__(256) k_mode_product(ProductArgs a) {
  extern __shared__ __align__(16) float sm[];
  const int n = a.n, npad = a.npad;
  const int lds = tile_lds(n);
  float* As = sm;                       // [n][npad]
  float* Ss = sm + (size_t)n * npad;    // [kPT][lds]
  const int tid = threadIdx.x, nth = blockDim.x;
  const int tx = tid & 7, ty = tid >> 3;
  const long long p0 = (long long)blockIdx.x * kPT;
  const int cnt = (int)min((long long)kPT, a.m - p0);
  {
    const int tot4 = n * npad / 4;
    for (int e = tid; e < tot4; e += nth) cp_async16(As + 4 * e, a.AT + 4 * e);
    const int half = n / 2;  // n is even: 8-byte pieces
    const float* base = a.src + p0 * n;
    const int tot2 = cnt * half;
    for (int e = tid; e < tot2; e += nth) {
      const int pr = e / half, i2 = e - pr * half;
      cp_async8(Ss + pr * lds + 2 * i2, base + (size_t)pr * n + 2 * i2);
    }
    for (int e = cnt * lds + tid; e < kPT * lds; e += nth) Ss[e] = 0.f;
    cp_async_wait_all();
  }
  __syncthreads();
  float acc[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[r][c] = 0.f;
  const float* arow = As + ty * 8;
  const float* bcol = Ss + tx * lds;
#pragma unroll 2
  for (int kk = 0; kk < n; ++kk) {
    const float4 a0 = *reinterpret_cast<const float4*>(arow + (size_t)kk * npad);
    const float4 a1 = *reinterpret_cast<const float4*>(arow + (size_t)kk * npad + 4);
    const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
    float bv[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) bv[c] = bcol[c * 8 * lds + kk];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[r][c] = fmaf(av[r], bv[c], acc[r][c]);
  }
  if (EPI == EPI_INVL) {
    // every factor in flight before the first store (dest and invl could
    // alias as far as the compiler knows)
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int row = ty * 8 + r;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int pc = tx + 8 * c;
        const bool in = row < n && pc < cnt;
        acc[r][c] *= in ? __ldg(a.invl + (p0 + pc) + a.m * row) : 0.f;
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int row = ty * 8 + r;
    if (row >= n) continue;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int pc = tx + 8 * c;
      if (pc >= cnt) continue;
      const long long p = p0 + pc;
      const long long o = p + a.m * row;
      float v = acc[r][c];
      if (EPI != EPI_PHI) {
        a.dest[o] = v;
      } else {
        const int N = n + 2;
        const int i = (int)(p % n), j = (int)(p / n);
        a.dest[(size_t)(i + 1) + (size_t)N * ((j + 1) + (size_t)N * (row + 1))] = v;
      }
    }
  }
}

size_t product_smem(int n, int npad) { return ((size_t)n * npad + (size_t)kPT * tile_lds(n)) * sizeof(float); }

template <int EPI>
void product(Ctx& c, const ProductArgs& a) {
  const size_t smem = product_smem(a.n, a.npad);
  static bool attr_set = false;
  if (!attr_set) {
    VLB_CUDA(cudaFuncSetAttribute(k_mode_product<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(227 * 1024)));
    attr_set = true;
  }
  const unsigned grid = (unsigned)((a.m + kPT - 1) / kPT);
  k_mode_product<EPI><<<grid, a.npad, smem, c.stream>>>(a);
  VLB_LAUNCHED(c);
}

__device__ __forceinline__ float xc_potential(float rho) {
  // src/meanfield.jl:371-386
  const float XC_EXCHANGE = -0.9847450218426966f;          // -cbrt(3/pi)
  const float XC_CORRELATION = -0.0333f;
  const float XC_CORRELATION_SCALE = 18.376708275787752f;  // 11.4 cbrt(4pi/3)
  float c = cbrtf(rho);
  return XC_EXCHANGE * c + XC_CORRELATION * log1pf(XC_CORRELATION_SCALE * c);
}
__device__ __forceinline__ float sphere_potential(float Q, float R, float r) {
  return r < R ? -Q * (3.f - (r / R) * (r / R)) / (2.f * R) : -Q / r;
}

// Right-hand side of the interior with the Dirichlet lifting
// (src/poisson.jl:275-294), one thread per interior point, i fastest: a
// grid-stride loop over the n^3 interior points (n^3 < 2^31).
__global__ void __launch_bounds__(256) k_rhs(float* __restrict__ rhs, const float* __restrict__ rho,
                                             const float* __restrict__ P, const float* __restrict__ D, int n) {
  const int N = n + 2;
  const size_t sj = N, sk = (size_t)N * N;
  const unsigned un = (unsigned)n, tot = un * un * un;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
    const unsigned jk = t / un, i = t - jk * un;
    const unsigned k = jk / un, j = jk - k * un;
    const size_t row = sj * (j + 1) + sk * (k + 1);
    const size_t c = (size_t)(i + 1) + row;
    float v = fmul(-12.566370614359172f, rho[c]);
    v = fsub(v, fmul(D[(i + 1) * N], P[row]));
    v = fsub(v, fmul(D[(i + 1) * N + N - 1], P[row + N - 1]));
    v = fsub(v, fmul(D[(j + 1) * N], P[(i + 1) + sk * (k + 1)]));
    v = fsub(v, fmul(D[(j + 1) * N + N - 1], P[(i + 1) + sj * (N - 1) + sk * (k + 1)]));
    v = fsub(v, fmul(D[(k + 1) * N], P[(i + 1) + sj * (j + 1)]));
    v = fsub(v, fmul(D[(k + 1) * N + N - 1], P[(i + 1) + sj * (j + 1) + sk * (N - 1)]));
    rhs[t] = v;
  }
}

// phi + V_xc(rho) + V_jel(r) at the collocation points (phi may be null):
// a grid-stride loop over the n^3 points, i fastest (n^3 < 2^31).
__global__ void __launch_bounds__(256) k_meanfield_src(float* __restrict__ out, const float* __restrict__ phi,
                                                       const float* __restrict__ rho, const float* __restrict__ g,
                                                       int n, float nions, float radius) {
  const unsigned un = (unsigned)n, tot = un * un * un;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
    const unsigned jk = t / un, i = t - jk * un;
    const unsigned k = jk / un, j = jk - k * un;
    const float r = sqrtf(g[i] * g[i] + g[j] * g[j] + g[k] * g[k]);
    const float extra = xc_potential(rho[t]) + sphere_potential(nions, radius, r);
    out[t] = phi ? phi[t] + extra : extra;
  }
}

// ---------------------------------------------------------------- moments
constexpr int kMomBlocks = 256;   // block partials of the ten moments

// Ten moments of the density (src/poisson.jl:55-93), float64: one warp per
// (j,k) column at a time (coalesced along i), summed per warp, then per
// block in a fixed order into partial[r * kMomBlocks + block].
__global__ void __launch_bounds__(256) k_moments(const float* __restrict__ rho, const double* __restrict__ dual,
                                                 int n, double* __restrict__ partial) {
  __shared__ double sh[10][8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int m = n * n;
  const double *p0 = dual, *p1 = dual + n, *p2 = dual + 2 * n;
  double acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int t = blockIdx.x * 8 + w; t < m; t += gridDim.x * 8) {
    const float* col = rho + (size_t)n * t;
    double s0 = 0, s1 = 0, s2 = 0;
    for (int i = lane; i < n; i += 32) {
      const double v = col[i];
      s0 += v * p0[i];
      s1 += v * p1[i];
      s2 += v * p2[i];
    }
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    const int j = t % n, k = t / n;
    const double a = p0[j] * p0[k], b = p1[j] * p0[k], cc = p0[j] * p1[k];
    const double d = p2[j] * p0[k], e = p0[j] * p2[k], f = p1[j] * p1[k];
    acc[0] += s0 * a;
    acc[1] += s1 * a;
    acc[2] += s0 * b;
    acc[3] += s0 * cc;
    acc[4] += s2 * a;
    acc[5] += s0 * d;
    acc[6] += s0 * e;
    acc[7] += s1 * b;
    acc[8] += s1 * cc;
    acc[9] += s0 * f;
  }
  if (lane == 0)
    for (int r = 0; r < 10; ++r) sh[r][w] = acc[r];
  __syncthreads();
  if (threadIdx.x < 10) {
    double s = 0;
    for (int ww = 0; ww < 8; ++ww) s += sh[threadIdx.x][ww];
    partial[(size_t)threadIdx.x * kMomBlocks + blockIdx.x] = s;
  }
}

// Block r: the sum of moment r over the block partials, in a fixed order.
__global__ void __launch_bounds__(256) k_moment_sums(const double* __restrict__ partial, DeviceScalars* dsc) {
  __shared__ double sh[256];
  const int r = blockIdx.x;
  sh[threadIdx.x] = threadIdx.x < kMomBlocks ? partial[(size_t)r * kMomBlocks + threadIdx.x] : 0.0;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) dsc->moments[r] = sh[0];
}

// Monopole, barycentre and traceless quadrupole in the barycentre frame
// (src/poisson.jl:168-189) from the ten moments.
__device__ __forceinline__ void multipole_of(const double* tot, double* mp) {
  const double q = tot[0];
  const double cx = q == 0 ? 0 : tot[1] / q, cy = q == 0 ? 0 : tot[2] / q, cz = q == 0 ? 0 : tot[3] / q;
  const double m200 = tot[4], m020 = tot[5], m002 = tot[6], mxy = tot[7], mxz = tot[8], myz = tot[9];
  const double b2 = cx * cx + cy * cy + cz * cz;
  mp[0] = q;
  mp[1] = cx; mp[2] = cy; mp[3] = cz;
  mp[4] = (2 * m200 - m020 - m002) - q * (3 * cx * cx - b2);
  mp[5] = (2 * m020 - m200 - m002) - q * (3 * cy * cy - b2);
  mp[6] = (2 * m002 - m200 - m020) - q * (3 * cz * cz - b2);
  mp[7] = 3 * mxy - 3 * q * cx * cy;
  mp[8] = 3 * mxz - 3 * q * cx * cz;
  mp[9] = 3 * myz - 3 * q * cy * cz;
}

// t-th surface point of an n^3 grid, 0-based (src/kernels.jl:836-859)
__device__ __forceinline__ void face_point(int t, int n, int& i, int& j, int& k) {
  const int cap = n * n;
  if (t < cap) { i = t % n; j = t / n; k = 0; return; }
  t -= cap;
  if (t < cap) { i = t % n; j = t / n; k = n - 1; return; }
  t -= cap;
  const int ring = 2 * n + 2 * (n - 2);
  k = t / ring + 1;
  const int r = t % ring;
  if (r < n) { i = r; j = 0; }
  else if (r < 2 * n) { i = r - n; j = n - 1; }
  else if (r < 2 * n + (n - 2)) { i = 0; j = r - 2 * n + 1; }
  else { i = n - 1; j = r - 2 * n - (n - 2) + 1; }
}

// Multipole potential on the faces (src/poisson.jl:198-206)
__global__ void k_faces_multipole(float* __restrict__ phi, const float* __restrict__ g, int n,
                                  DeviceScalars* dsc) {
  const int nf = 2 * n * n + (n - 2) * (4 * n - 4);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double mp[10];
  multipole_of(dsc->moments, mp);
  if (t == 0)
    for (int r = 0; r < 10; ++r) dsc->multipole[r] = mp[r];
  if (t >= nf) return;
  int i, j, k;
  face_point(t, n, i, j, k);
  const double px = (double)g[i] - mp[1], py = (double)g[j] - mp[2], pz = (double)g[k] - mp[3];
  const double r2 = px * px + py * py + pz * pz;
  const double invr = 1.0 / sqrt(r2);
  const double quad = mp[4] * px * px + mp[5] * py * py + mp[6] * pz * pz +
                      2 * (mp[7] * px * py + mp[8] * px * pz + mp[9] * py * pz);
  const double i5 = invr * invr * invr * invr * invr;
  phi[(size_t)i + (size_t)n * (j + (size_t)n * k)] = (float)(mp[0] * invr + quad * i5 / 2);
}

// Hermite basis value in float (src/splines.jl:74-122)
__device__ __forceinline__ float basis_value(const float* g, int nk, int lin, float x) {
  const int knot = (lin - 1) / 2 + 1, kind = (lin - 1) & 1;
  float a, h, s;
  if (knot > 1 && x <= g[knot - 1]) {
    if (x < g[knot - 2]) return 0.f;
    h = g[knot - 1] - g[knot - 2]; a = (x - g[knot - 2]) / h; s = -1.f;
  } else if (knot < nk && x >= g[knot - 1]) {
    if (x > g[knot]) return 0.f;
    h = g[knot] - g[knot - 1]; a = (g[knot] - x) / h; s = 1.f;
  } else {
    return 0.f;
  }
  return kind == 0 ? 3.f * (a * a) - 2.f * (a * a * a) : h * (a * a - a * a * a) * s;
}

__device__ __forceinline__ int cell_index_f(const float* g, int nk, float x) {
  if (x < g[0] || x > g[nk - 1]) return 0;
  int lo = 0, hi = nk;  // first index with g[idx] >= x
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (g[mid] < x) lo = mid + 1; else hi = mid;
  }
  return max(1, lo);
}

// Fine faces from the coarse spline (src/kernels.jl:888-898, src/fields.jl:440-469)
__global__ void k_faces_from_coarse(float* __restrict__ phi, const float* __restrict__ gf, int n,
                                    const float* __restrict__ kc, int nkc, const float* __restrict__ csol, int nc) {
  const int nf = 2 * n * n + (n - 2) * (4 * n - 4);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nf) return;
  int i, j, k;
  face_point(t, n, i, j, k);
  const float px = gf[i], py = gf[j], pz = gf[k];
  const int cx = cell_index_f(kc, nkc, px), cy = cell_index_f(kc, nkc, py), cz = cell_index_f(kc, nkc, pz);
  float v;
  if (!cx || !cy || !cz) {
    v = __int_as_float(0x7fc00000);
  } else {
    float vx[4], vy[4], vz[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      vx[a] = basis_value(kc, nkc, 2 * (cx - 1) + a + 1, px);
      vy[a] = basis_value(kc, nkc, 2 * (cy - 1) + a + 1, py);
      vz[a] = basis_value(kc, nkc, 2 * (cz - 1) + a + 1, pz);
    }
    v = 0.f;
    for (int ak = 0; ak < 4; ++ak)
      for (int aj = 0; aj < 4; ++aj) {
        const float w = vy[aj] * vz[ak];
        const float* row = csol + (size_t)2 * (cx - 1) + (size_t)nc * ((2 * (cy - 1) + aj) + (size_t)nc * (2 * (cz - 1) + ak));
#pragma unroll
        for (int ai = 0; ai < 4; ++ai) v += row[ai] * vx[ai] * w;
      }
  }
  phi[(size_t)i + (size_t)n * (j + (size_t)n * k)] = v;
}

__global__ void k_add(float* __restrict__ a, const float* __restrict__ b, size_t n) {
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
    a[t] += b[t];
}

ProductArgs base_args(const Level& L, bool interior) {
  ProductArgs a{};
  a.n = interior ? L.ni : L.n;
  a.npad = interior ? L.nipad : L.npad;
  a.m = (long long)a.n * a.n;
  return a;
}

// solve_interior! with the faces already in phi (src/devicemesh.jl:133-146)
void solve_interior(Ctx& c, Level& L) {
  const int ni = L.ni;
  k_rhs<<<grid_for(c, (int64_t)ni * ni * ni, 256, 8), 256, 0, c.stream>>>(c.work[2], L.rho, L.phi, L.lap, ni);
  VLB_LAUNCHED(c);
  ProductArgs a = base_args(L, true);
  if (c.mode_precision != VLB_POISSON_FP32) {
    // two chains of three products on the tensor cores
    const float* s1[3] = {c.work[2], c.work[0], c.work[1]};
    float* d1[3] = {c.work[0], c.work[1], c.work[0]};
    const int e1[3] = {EPI_PLAIN, EPI_PLAIN, EPI_INVL};
    launch_mode_chain_tc(c, L.tc_Minv, 3, s1, d1, e1, a.m, L.invlsum);
    const float* s2[3] = {c.work[0], c.work[1], c.work[0]};
    float* d2[3] = {c.work[1], c.work[0], L.phi};
    const int e2[3] = {EPI_PLAIN, EPI_PLAIN, EPI_PHI};
    launch_mode_chain_tc(c, L.tc_M, 3, s2, d2, e2, a.m, nullptr);
    return;
  }
  // forward: into the eigenbasis
  a.AT = L.MinvT;
  a.src = c.work[2]; a.dest = c.work[0];
  product<EPI_PLAIN>(c, a);
  a.src = c.work[0]; a.dest = c.work[1];
  product<EPI_PLAIN>(c, a);
  a.src = c.work[1]; a.dest = c.work[0]; a.invl = L.invlsum;
  product<EPI_INVL>(c, a);
  // back
  a.AT = L.MT;
  a.src = c.work[0]; a.dest = c.work[1];
  product<EPI_PLAIN>(c, a);
  a.src = c.work[1]; a.dest = c.work[0];
  product<EPI_PLAIN>(c, a);
  a.src = c.work[0]; a.dest = L.phi;
  product<EPI_PHI>(c, a);
}

// three S^-1 rotations: src -> w0 -> w1 -> dst
void coefficients(Ctx& c, Level& L, const float* src, float* w0, float* w1, float* dst) {
  ProductArgs a = base_args(L, false);
  if (c.mode_precision != VLB_POISSON_FP32) {
    const float* s[3] = {src, w0, w1};
    float* d[3] = {w0, w1, dst};
    const int e[3] = {EPI_PLAIN, EPI_PLAIN, EPI_PLAIN};
    launch_mode_chain_tc(c, L.tc_sinv, 3, s, d, e, a.m, nullptr);
    return;
  }
  a.AT = L.sinvT;
  a.src = src; a.dest = w0;
  product<EPI_PLAIN>(c, a);
  a.src = w0; a.dest = w1;
  product<EPI_PLAIN>(c, a);
  a.src = w1; a.dest = dst;
  product<EPI_PLAIN>(c, a);
}

}  // namespace

void launch_coefficients(Ctx& c, Level& L, const float* src, float* dst) {
  coefficients(c, L, src, c.work[0], c.work[1], dst);
}

// csol = S^-1 (phi + V_xc(rho) + V_jel(r)): the Hartree coefficients and the
// mean field of effective_potential! (src/devicemesh.jl:171-183) in one pass
void launch_mean_field_coefficients(Ctx& c, Level& L, const float* phi, float* csol, double nions,
                                    double radius) {
  k_meanfield_src<<<grid_for(c, (int64_t)L.n * L.n * L.n, 256, 8), 256, 0, c.stream>>>(
      c.work[2], phi, L.rho, L.colloc, L.n, (float)nions, (float)radius);
  VLB_LAUNCHED(c);
  coefficients(c, L, c.work[2], c.work[0], c.work[1], csol);
}

// csol += S^-1 [V_xc(rho) + V_jel(r)] (src/devicemesh.jl:171-183)
void launch_mean_field_add(Ctx& c, Level& L, double nions, double radius) {
  const size_t tot = (size_t)L.n * L.n * L.n;
  k_meanfield_src<<<grid_for(c, (int64_t)L.n * L.n * L.n, 256, 8), 256, 0, c.stream>>>(
      c.work[2], nullptr, L.rho, L.colloc, L.n, (float)nions, (float)radius);
  VLB_LAUNCHED(c);
  coefficients(c, L, c.work[2], c.work[0], c.work[1], c.work[2]);
  k_add<<<grid_for(c, (int64_t)tot, 256, 8), 256, 0, c.stream>>>(L.csol, c.work[2], tot);
  VLB_LAUNCHED(c);
}

void launch_poisson(Ctx& c) {
  Level& F = c.fine;
  Level& C = c.coarse;
  // coarse: multipole faces + solve (src/poisson.jl:351-354)
  const int mc = C.n * C.n;
  (void)mc;
  k_moments<<<kMomBlocks, 256, 0, c.stream>>>(C.rho, C.dual_d, C.n, c.partials);
  VLB_LAUNCHED(c);
  k_moment_sums<<<10, 256, 0, c.stream>>>(c.partials, c.dsc);
  VLB_LAUNCHED(c);
  const int nfc = 2 * C.n * C.n + (C.n - 2) * (4 * C.n - 4);
  k_faces_multipole<<<(nfc + 255) / 256, 256, 0, c.stream>>>(C.phi, C.colloc, C.n, c.dsc);
  VLB_LAUNCHED(c);
  solve_interior(c, C);
  // fine faces from the coarse Hartree coefficients, then the fine solve
  launch_coefficients(c, C, C.phi, C.csol_hartree);
  const int nff = 2 * F.n * F.n + (F.n - 2) * (4 * F.n - 4);
  k_faces_from_coarse<<<(nff + 255) / 256, 256, 0, c.stream>>>(F.phi, F.colloc, F.n, C.knots, C.nk,
                                                               C.csol_hartree, C.n);
  VLB_LAUNCHED(c);
  solve_interior(c, F);
}

}  // namespace vlb
