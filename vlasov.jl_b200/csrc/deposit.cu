// Charge deposits of the sorted cloud.
//
// Fine grid (src/accelerator.jl:531-565, src/kernels.jl:601-779): for every
// occupied cell, the 8^3 Gaussian-smoothed stencil of its particles is summed
// in registers and written once, either with float32 atomics (as the
// reference) or as int64 fixed point (charge scaled by 2^40), which is
// bit-identical from run to run and independent of the order in which cells
// finish.  The table columns and the window test are the reference's Float32
// arithmetic (src/kernels.jl:754-779); particles outside the window keep
// column 1 and are counted in nout, exactly as the reference does.  The
// charge is then renormalised to (N - nout) * w (src/accelerator.jl:554-557)
// with a deterministic reduction of sum rho m0x m0y m0z
// (src/deposition.jl:213-245).
//
// Coarse grid (src/kernels.jl:1207-1273, src/devicemesh.jl:93-106):
// trilinear cloud-in-cell on the stretched collocation points, each thread
// walking a block of consecutive sorted particles into a private window of
// shared memory that is added to the grid once.  The cell lookup is the
// reference's Float32 LocateTable walk.

#include "vlb_internal.cuh"

namespace vlb {

int grid_for(const Ctx& c, int64_t n, int threads, int per_sm);

namespace {

constexpr int kDepThreads = 256;
constexpr int kDepLanes = 16;      // particle lanes per CTA
constexpr int kDepStage = 256;     // particles whose columns are staged at once
constexpr double kFixedScale = 1099511627776.0;        // 2^40
constexpr double kFixedInv = 1.0 / 1099511627776.0;

__global__ void __launch_bounds__(kDepThreads) k_deposit_fine(
    const int32_t* __restrict__ occupied, const int32_t* __restrict__ bounds, DeviceScalars* dsc,
    int64_t Npad, const int32_t* __restrict__ k, const float* __restrict__ d, const float* __restrict__ nodes,
    int nk, int n, float x0, float h, float lo, float hi, float spacing, int nbdt, int ncol, float* rho,
    unsigned long long* rho_fixed, int mode) {
  extern __shared__ __align__(16) unsigned char smem[];
  float* nodes_s = reinterpret_cast<float*>(smem);                      // [ncol][8]
  int* cols_s = reinterpret_cast<int*>(nodes_s + (size_t)ncol * 8);      // [3][kDepStage]
  float* red_s = reinterpret_cast<float*>(cols_s + 3 * kDepStage);       // [kDepLanes][512]
  __shared__ int s_g;
  __shared__ int s_nout;
  const int tid = threadIdx.x;
  for (int e = tid; e < ncol * 8; e += kDepThreads) nodes_s[e] = nodes[e];
  if (tid == 0) s_nout = 0;
  const int nocc = dsc->noccupied;
  const int pl = tid / 16, q = tid % 16;
  const int j0 = 2 * (q % 4), k0 = 2 * (q / 4);
  int my_nout = 0;
  __syncthreads();
  for (;;) {
    if (tid == 0) s_g = (int)atomicAdd(&dsc->work_deposit, 1ull);
    __syncthreads();
    const int g = s_g;
    if (g >= nocc) break;
    const int cell = occupied[g];
    const int sl = bounds[g], sh = bounds[g + 1];
    int kx, ky, kz;
    cell_knots((uint32_t)cell, nk, kx, ky, kz);
    const bool fits = deposit_fits(kx, ky, kz, n);
    float acc[32];
#pragma unroll
    for (int a = 0; a < 32; ++a) acc[a] = 0.f;
    for (int base = sl; base < sh; base += kDepStage) {
      const int s = base + tid;
      if (s < sh) {
        bool inside = true;
        int cc[3];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          const int kk = k[ax * Npad + s];
          const float dd = d[ax * Npad + s];
          const float p = fadd(fadd(x0, fmul((float)(kk - 1), h)), dd);
          inside = inside && (lo <= p) && (p <= hi);
          cc[ax] = table_column(dd, spacing, nbdt, ncol);
        }
        if (!inside) { cc[0] = cc[1] = cc[2] = 1; ++my_nout; }
        cols_s[tid] = cc[0];
        cols_s[kDepStage + tid] = cc[1];
        cols_s[2 * kDepStage + tid] = cc[2];
      }
      __syncthreads();
      if (fits) {
        const int cnt = min(kDepStage, sh - base);
        for (int t = pl; t < cnt; t += kDepLanes) {
          const float* vx = nodes_s + (size_t)(cols_s[t] - 1) * 8;
          const float* vy = nodes_s + (size_t)(cols_s[kDepStage + t] - 1) * 8;
          const float* vz = nodes_s + (size_t)(cols_s[2 * kDepStage + t] - 1) * 8;
          const float4 xa = *reinterpret_cast<const float4*>(vx);
          const float4 xb = *reinterpret_cast<const float4*>(vx + 4);
          const float2 y = *reinterpret_cast<const float2*>(vy + j0);
          const float2 z = *reinterpret_cast<const float2*>(vz + k0);
          const float x[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
          const float w[4] = {y.x * z.x, y.y * z.x, y.x * z.y, y.y * z.y};
#pragma unroll
          for (int m = 0; m < 4; ++m)
#pragma unroll
            for (int a = 0; a < 8; ++a) acc[8 * m + a] = fmaf(x[a], w[m], acc[8 * m + a]);
        }
      }
      __syncthreads();
    }
    if (fits) {
      // lane partials -> shared, then a fixed-order sum over the 16 lanes
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int jj = j0 + (m & 1), kk = k0 + (m >> 1);
#pragma unroll
        for (int a = 0; a < 8; ++a) red_s[pl * 512 + a + 8 * (jj + 8 * kk)] = acc[8 * m + a];
      }
      __syncthreads();
      const int bx = 2 * kx - 5, by = 2 * ky - 5, bz = 2 * kz - 5;
      for (int o = tid; o < 512; o += kDepThreads) {
        float v = 0.f;
#pragma unroll
        for (int l = 0; l < kDepLanes; ++l) v += red_s[l * 512 + o];
        const int a = o & 7, jj = (o >> 3) & 7, kk = o >> 6;
        const size_t addr = (size_t)(bx + a) + (size_t)n * ((by + jj) + (size_t)n * (bz + kk));
        if (mode == VLB_DEPOSIT_FIXED64) {
          const long long iv = llrint((double)v * kFixedScale);
          if (iv) atomicAdd(&rho_fixed[addr], (unsigned long long)iv);
        } else if (v != 0.f) {
          atomicAdd(&rho[addr], v);
        }
      }
    }
    __syncthreads();
  }
  atomicAdd(&s_nout, my_nout);
  __syncthreads();
  if (tid == 0 && s_nout) atomicAdd(&dsc->nout, s_nout);
}

// Per (j,k) column: sum_i rho[i,j,k] m0[i], times m0[j] m0[k].
__global__ void k_charge_columns(const float* __restrict__ rho, const unsigned long long* __restrict__ fixed,
                                 const double* __restrict__ m0, int n, double* __restrict__ partial) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * n) return;
  const int j = t % n, kq = t / n;
  double s = 0;
  if (fixed) {
    for (int i = 0; i < n; ++i) s += (double)(long long)fixed[(size_t)t * n + i] * kFixedInv * m0[i];
  } else {
    for (int i = 0; i < n; ++i) s += (double)rho[(size_t)t * n + i] * m0[i];
  }
  partial[t] = s * m0[j] * m0[kq];
}

// One block: the fixed-order sum of the column partials.
__global__ void __launch_bounds__(1024) k_charge_total(const double* __restrict__ partial, int m, double* out) {
  __shared__ double sh[1024];
  double s = 0;
  for (int t = threadIdx.x; t < m; t += 1024) s += partial[t];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// rho *= (N - nout) w / q, converting from fixed point when needed.
__global__ void k_charge_scale(float* __restrict__ rho, const unsigned long long* __restrict__ fixed, size_t tot,
                               const DeviceScalars* dsc, int64_t N, double w) {
  const double q = dsc->charge_raw;
  const float sc = (float)((double)(N - dsc->nout) * w / q);
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (size_t)gridDim.x * blockDim.x) {
    const float v = fixed ? (float)((double)(long long)fixed[t] * kFixedInv) : rho[t];
    rho[t] = v * sc;
  }
}

// --------------------------------------------------------------- coarse
constexpr int kCicThreads = 256;
constexpr int kCicBlock = 64;   // consecutive sorted particles per thread
constexpr int kCicT = 4;        // private window: 4^3 coarse points
constexpr int kCicT3 = kCicT * kCicT * kCicT;

// Cell of x on the stretched collocation points (src/kernels.jl:1069-1081):
// the Float32 LocateTable walk, tables in shared memory; 0 outside.  w is the
// weight of the left point, with the division replaced by the interval's
// reciprocal.
__device__ __forceinline__ int locate_cell(const float* __restrict__ gt, const float* __restrict__ igap, int ng,
                                           float lx0, float linvw, const int32_t* __restrict__ cells, int ncells,
                                           float x, float& w) {
  if (x < gt[0] || x > gt[ng - 1]) { w = 0.f; return 0; }
  int b = min((int)floorf(fmul(fsub(x, lx0), linvw)) + 1, ncells);
  int c = cells[b - 1];
  const int lastc = ng - 1;
  while (c < lastc && gt[c] < x) ++c;
  w = fsub(gt[c], x) * igap[c];
  return c;
}

// Each thread walks kCicBlock consecutive sorted particles -- a handful of
// neighbouring fine cells -- into a private 4^3 window of shared memory
// anchored one point before its first particle, and adds the window to the
// grid once; particles that miss the window use global atomics (the
// reference's design, src/kernels.jl:1083-1273).  Loads are 16-byte vectors of
// four particles.  Contributions carry charge / (wx wy wz)
// (src/devicemesh.jl:104).
__global__ void __launch_bounds__(kCicThreads) k_deposit_cic(
    int64_t N, int64_t Npad, const int32_t* __restrict__ k, const float* __restrict__ d,
    const float* __restrict__ gt_g, int ng, float lx0, float linvw, const int32_t* __restrict__ cells_g, int ncells,
    const float* __restrict__ dl_g, float x0f, float hf, float charge, float* rho, int64_t nblock) {
  extern __shared__ __align__(16) unsigned char smem[];
  float* tile = reinterpret_cast<float*>(smem);                 // [kCicT3][kCicThreads]
  float* gt = tile + kCicT3 * kCicThreads;                      // [ng]
  float* igap = gt + ng;                                        // [ng] 1 / (gt[c] - gt[c-1])
  float* idl = igap + ng;                                       // [ng] 1 / dual length
  int32_t* cells = reinterpret_cast<int32_t*>(idl + ng);        // [ncells]
  for (int e = threadIdx.x; e < ng; e += kCicThreads) {
    gt[e] = gt_g[e];
    igap[e] = e > 0 ? 1.f / (gt_g[e] - gt_g[e - 1]) : 0.f;
    idl[e] = 1.f / dl_g[e];
  }
  for (int e = threadIdx.x; e < ncells; e += kCicThreads) cells[e] = cells_g[e];
  __syncthreads();
  const int t = threadIdx.x;
  const size_t n = ng, nn = n * n;
  for (int64_t blk = (int64_t)blockIdx.x * kCicThreads + t; blk < nblock; blk += (int64_t)gridDim.x * kCicThreads) {
#pragma unroll
    for (int p = 0; p < kCicT3; ++p) tile[p * kCicThreads + t] = 0.f;
    const int64_t lo = blk * kCicBlock;
    const int64_t hi = min(lo + kCicBlock, N);
    int ox = 0, oy = 0, oz = 0;
    bool anchored = false;
    for (int64_t q = lo; q < hi; q += 4) {
      // four particles per 16-byte load; Npad and lo are multiples of 4
      const int4 kx4 = *reinterpret_cast<const int4*>(k + q);
      const int4 ky4 = *reinterpret_cast<const int4*>(k + Npad + q);
      const int4 kz4 = *reinterpret_cast<const int4*>(k + 2 * Npad + q);
      const float4 dx4 = *reinterpret_cast<const float4*>(d + q);
      const float4 dy4 = *reinterpret_cast<const float4*>(d + Npad + q);
      const float4 dz4 = *reinterpret_cast<const float4*>(d + 2 * Npad + q);
      const int kxs[4] = {kx4.x, kx4.y, kx4.z, kx4.w}, kys[4] = {ky4.x, ky4.y, ky4.z, ky4.w},
                kzs[4] = {kz4.x, kz4.y, kz4.z, kz4.w};
      const float dxs[4] = {dx4.x, dx4.y, dx4.z, dx4.w}, dys[4] = {dy4.x, dy4.y, dy4.z, dy4.w},
                  dzs[4] = {dz4.x, dz4.y, dz4.z, dz4.w};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (q + u >= hi) break;
        const float px = fadd(fadd(x0f, fmul((float)(kxs[u] - 1), hf)), dxs[u]);
        const float py = fadd(fadd(x0f, fmul((float)(kys[u] - 1), hf)), dys[u]);
        const float pz = fadd(fadd(x0f, fmul((float)(kzs[u] - 1), hf)), dzs[u]);
        float ax, ay, az;
        const int ix = locate_cell(gt, igap, ng, lx0, linvw, cells, ncells, px, ax);
        const int iy = locate_cell(gt, igap, ng, lx0, linvw, cells, ncells, py, ay);
        const int iz = locate_cell(gt, igap, ng, lx0, linvw, cells, ncells, pz, az);
        if (!(ix > 0 && iy > 0 && iz > 0)) continue;
        const int i0 = ix - 1, j0 = iy - 1, k0 = iz - 1;  // 0-based left points
        if (!anchored) { ox = i0 - 1; oy = j0 - 1; oz = k0 - 1; anchored = true; }
        const float wx0 = ax * idl[i0], wx1 = (1.f - ax) * idl[i0 + 1];
        const float wy0 = ay * idl[j0], wy1 = (1.f - ay) * idl[j0 + 1];
        const float wz0 = charge * az * idl[k0], wz1 = charge * (1.f - az) * idl[k0 + 1];
        const int lx = i0 - ox, ly = j0 - oy, lz = k0 - oz;
        if (lx >= 0 && ly >= 0 && lz >= 0 && lx + 1 < kCicT && ly + 1 < kCicT && lz + 1 < kCicT) {
          float* b = tile + (lx + kCicT * (ly + kCicT * lz)) * kCicThreads + t;
          constexpr int SY = kCicT * kCicThreads, SZ = kCicT * kCicT * kCicThreads, SX = kCicThreads;
          b[0] += wx0 * wy0 * wz0;
          b[SZ] += wx0 * wy0 * wz1;
          b[SY] += wx0 * wy1 * wz0;
          b[SY + SZ] += wx0 * wy1 * wz1;
          b[SX] += wx1 * wy0 * wz0;
          b[SX + SZ] += wx1 * wy0 * wz1;
          b[SX + SY] += wx1 * wy1 * wz0;
          b[SX + SY + SZ] += wx1 * wy1 * wz1;
        } else {
          float* b = rho + (size_t)i0 + n * j0 + nn * k0;
          atomicAdd(b, wx0 * wy0 * wz0);
          atomicAdd(b + nn, wx0 * wy0 * wz1);
          atomicAdd(b + n, wx0 * wy1 * wz0);
          atomicAdd(b + n + nn, wx0 * wy1 * wz1);
          atomicAdd(b + 1, wx1 * wy0 * wz0);
          atomicAdd(b + 1 + nn, wx1 * wy0 * wz1);
          atomicAdd(b + 1 + n, wx1 * wy1 * wz0);
          atomicAdd(b + 1 + n + nn, wx1 * wy1 * wz1);
        }
      }
    }
    if (anchored) {
#pragma unroll 4
      for (int p = 0; p < kCicT3; ++p) {
        const float v = tile[p * kCicThreads + t];
        if (v != 0.f) {
          const int lx = p % kCicT, ly = (p / kCicT) % kCicT, lz = p / (kCicT * kCicT);
          atomicAdd(&rho[(size_t)(ox + lx) + n * (oy + ly) + nn * (oz + lz)], v);
        }
      }
    }
  }
}

}  // namespace

size_t deposit_fine_smem(const Ctx& c) {
  return (size_t)c.ncol * 8 * sizeof(float) + 3 * kDepStage * sizeof(int) + (size_t)kDepLanes * 512 * sizeof(float);
}

size_t cic_smem(const Ctx& c);

void deposit_setup(Ctx& c) {
  VLB_CUDA(cudaFuncSetAttribute(k_deposit_fine, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)deposit_fine_smem(c)));
  VLB_CUDA(cudaFuncSetAttribute(k_deposit_cic, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cic_smem(c)));
}

void launch_deposit_fine(Ctx& c, double charge, int mode) {
  Level& F = c.fine;
  const size_t tot = (size_t)F.n * F.n * F.n;
  Particles& P = c.part[c.cur];
  if (mode == VLB_DEPOSIT_FIXED64)
    VLB_CUDA(cudaMemsetAsync(c.rho_fixed, 0, tot * sizeof(unsigned long long), c.stream));
  else
    VLB_CUDA(cudaMemsetAsync(F.rho, 0, tot * sizeof(float), c.stream));
  VLB_CUDA(cudaMemsetAsync(&c.dsc->work_deposit, 0, sizeof(unsigned long long), c.stream));
  VLB_CUDA(cudaMemsetAsync(&c.dsc->nout, 0, sizeof(int32_t), c.stream));
  const int grid = c.num_sms * 3;
  k_deposit_fine<<<grid, kDepThreads, deposit_fine_smem(c), c.stream>>>(
      c.occupied, c.bounds, c.dsc, c.Npad, P.k, P.d, c.nodes, F.nk, F.n, c.x0f, c.hf, c.lo_f, c.hi_f, c.spacing_f,
      c.nbdt, c.ncol, F.rho, c.rho_fixed, mode);
  VLB_LAUNCHED(c);
  const unsigned long long* fx = mode == VLB_DEPOSIT_FIXED64 ? c.rho_fixed : nullptr;
  const int cols = F.n * F.n;
  k_charge_columns<<<(cols + 127) / 128, 128, 0, c.stream>>>(F.rho, fx, F.dual_d, F.n, c.partials);
  VLB_LAUNCHED(c);
  k_charge_total<<<1, 1024, 0, c.stream>>>(c.partials, cols, &c.dsc->charge_raw);
  VLB_LAUNCHED(c);
  k_charge_scale<<<grid_for(c, (int64_t)tot, 256, 8), 256, 0, c.stream>>>(F.rho, fx, tot, c.dsc, c.N, charge);
  VLB_LAUNCHED(c);
}

size_t cic_smem(const Ctx& c) {
  return (size_t)kCicT3 * kCicThreads * sizeof(float) + 3 * (size_t)c.coarse.n * sizeof(float) +
         (size_t)c.coarse.loc_ncell * sizeof(int32_t);
}

void launch_deposit_coarse(Ctx& c, double charge) {
  Level& C = c.coarse;
  const size_t tot = (size_t)C.n * C.n * C.n;
  Particles& P = c.part[c.cur];
  VLB_CUDA(cudaMemsetAsync(C.rho, 0, tot * sizeof(float), c.stream));
  const int64_t nblock = (c.N + kCicBlock - 1) / kCicBlock;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((nblock + kCicThreads - 1) / kCicThreads,
                                                               (int64_t)c.num_sms * 3));
  k_deposit_cic<<<grid, kCicThreads, cic_smem(c), c.stream>>>(c.N, c.Npad, P.k, P.d, C.colloc, C.n, C.loc_x0,
                                                              C.loc_invw, C.loc_cells, C.loc_ncell, C.dlen, c.x0f,
                                                              c.hf, (float)charge, C.rho, nblock);
  VLB_LAUNCHED(c);
}

}  // namespace vlb
