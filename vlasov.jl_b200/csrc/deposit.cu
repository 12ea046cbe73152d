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
// walking a block of consecutive sorted particles into a private 4^3 window
// of shared memory and flushing it once.

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
constexpr int kCicBlock = 64;
constexpr int kCicTile = 4;
constexpr int kCicThreads = 128;

// Cell of x on the stretched collocation points (src/kernels.jl:1069-1081),
// Float32; 0 outside.  w is the weight of the left point.
__device__ __forceinline__ int locate_cell(const float* __restrict__ gt, int ng, float lx0, float linvw,
                                           const int32_t* __restrict__ cells, int ncells, float x, float& w) {
  if (x < gt[0] || x > gt[ng - 1]) { w = 0.f; return 0; }
  int b = min((int)floorf(fmul(fsub(x, lx0), linvw)) + 1, ncells);
  int c = cells[b - 1];
  const int lastc = ng - 1;
  while (c < lastc && gt[c] < x) ++c;
  w = fdiv(fsub(gt[c], x), fsub(gt[c], gt[c - 1]));
  return c;
}

__global__ void __launch_bounds__(kCicThreads) k_deposit_cic(
    int64_t N, int64_t Npad, const int32_t* __restrict__ k, const float* __restrict__ d,
    const float* __restrict__ gt, int ng, float lx0, float linvw, const int32_t* __restrict__ cells, int ncells,
    float x0f, float hf, float* rho, int64_t nblock) {
  constexpr int T = kCicTile, T3 = T * T * T;
  __shared__ float tile[T3 * kCicThreads];
  const int t = threadIdx.x;
  const int n = ng;
  for (int64_t blk = (int64_t)blockIdx.x * kCicThreads + t;; blk += (int64_t)gridDim.x * kCicThreads) {
    // uniform trip count across the CTA is not needed: no barrier inside
    if (blk >= nblock) break;
#pragma unroll 4
    for (int p = 0; p < T3; ++p) tile[p * kCicThreads + t] = 0.f;
    const int64_t lo = blk * kCicBlock;
    const int64_t hi = min(lo + kCicBlock, N);
    int ox = 0, oy = 0, oz = 0;
    bool anchored = false;
    for (int64_t i = lo; i < hi; ++i) {
      const float px = fadd(fadd(x0f, fmul((float)(k[i] - 1), hf)), d[i]);
      const float py = fadd(fadd(x0f, fmul((float)(k[Npad + i] - 1), hf)), d[Npad + i]);
      const float pz = fadd(fadd(x0f, fmul((float)(k[2 * Npad + i] - 1), hf)), d[2 * Npad + i]);
      float ax, ay, az;
      const int ix = locate_cell(gt, ng, lx0, linvw, cells, ncells, px, ax);
      const int iy = locate_cell(gt, ng, lx0, linvw, cells, ncells, py, ay);
      const int iz = locate_cell(gt, ng, lx0, linvw, cells, ncells, pz, az);
      if (!(ix > 0 && iy > 0 && iz > 0)) continue;
      if (!anchored) { ox = ix - 2; oy = iy - 2; oz = iz - 2; anchored = true; }
      const float bx = 1.f - ax, by = 1.f - ay, bz = 1.f - az;
      const int dx = ix - ox, dy = iy - oy, dz = iz - oz;
      if (dx >= 1 && dx <= T - 1 && dy >= 1 && dy <= T - 1 && dz >= 1 && dz <= T - 1) {
        const int b = (dz - 1) * T * T + (dy - 1) * T + (dx - 1);
        tile[(b)*kCicThreads + t] += ax * ay * az;
        tile[(b + T * T) * kCicThreads + t] += ax * ay * bz;
        tile[(b + T) * kCicThreads + t] += ax * by * az;
        tile[(b + T + T * T) * kCicThreads + t] += ax * by * bz;
        tile[(b + 1) * kCicThreads + t] += bx * ay * az;
        tile[(b + 1 + T * T) * kCicThreads + t] += bx * ay * bz;
        tile[(b + 1 + T) * kCicThreads + t] += bx * by * az;
        tile[(b + 1 + T + T * T) * kCicThreads + t] += bx * by * bz;
      } else {
        const size_t i0 = (size_t)(ix - 1) + (size_t)n * ((iy - 1) + (size_t)n * (iz - 1));
        const size_t sj = n, sk = (size_t)n * n;
        atomicAdd(&rho[i0], ax * ay * az);
        atomicAdd(&rho[i0 + sk], ax * ay * bz);
        atomicAdd(&rho[i0 + sj], ax * by * az);
        atomicAdd(&rho[i0 + sj + sk], ax * by * bz);
        atomicAdd(&rho[i0 + 1], bx * ay * az);
        atomicAdd(&rho[i0 + 1 + sk], bx * ay * bz);
        atomicAdd(&rho[i0 + 1 + sj], bx * by * az);
        atomicAdd(&rho[i0 + 1 + sj + sk], bx * by * bz);
      }
    }
    if (anchored) {
      for (int dz = 0; dz < T; ++dz)
        for (int dy = 0; dy < T; ++dy)
          for (int dx = 0; dx < T; ++dx) {
            const float v = tile[(dz * T * T + dy * T + dx) * kCicThreads + t];
            if (v != 0.f)
              atomicAdd(&rho[(size_t)(ox + dx) + (size_t)n * ((oy + dy) + (size_t)n * (oz + dz))], v);
          }
    }
  }
}

// rho[i,j,k] *= charge / (wx[i] wy[j] wz[k])   (src/devicemesh.jl:104)
__global__ void k_cic_scale(float* __restrict__ rho, const float* __restrict__ dl, int n, float charge) {
  const size_t tot = (size_t)n * n * n;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % n), j = (int)((t / n) % n), kq = (int)(t / ((size_t)n * n));
    rho[t] = rho[t] * fdiv(charge, fmul(fmul(dl[i], dl[j]), dl[kq]));
  }
}

}  // namespace

size_t deposit_fine_smem(const Ctx& c) {
  return (size_t)c.ncol * 8 * sizeof(float) + 3 * kDepStage * sizeof(int) + (size_t)kDepLanes * 512 * sizeof(float);
}

void deposit_setup(Ctx& c) {
  VLB_CUDA(cudaFuncSetAttribute(k_deposit_fine, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)deposit_fine_smem(c)));
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

void launch_deposit_coarse(Ctx& c, double charge) {
  Level& C = c.coarse;
  const size_t tot = (size_t)C.n * C.n * C.n;
  Particles& P = c.part[c.cur];
  VLB_CUDA(cudaMemsetAsync(C.rho, 0, tot * sizeof(float), c.stream));
  const int64_t nblock = (c.N + kCicBlock - 1) / kCicBlock;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((nblock + kCicThreads - 1) / kCicThreads,
                                                               (int64_t)c.num_sms * 4));
  k_deposit_cic<<<grid, kCicThreads, 0, c.stream>>>(c.N, c.Npad, P.k, P.d, C.colloc, C.n, C.loc_x0, C.loc_invw,
                                                    C.loc_cells, C.loc_ncell, c.x0f, c.hf, C.rho, nblock);
  VLB_LAUNCHED(c);
  k_cic_scale<<<grid_for(c, (int64_t)tot, 256, 8), 256, 0, c.stream>>>(C.rho, C.dlen, C.n, (float)charge);
  VLB_LAUNCHED(c);
}

}  // namespace vlb
