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
// trilinear cloud-in-cell on the stretched collocation points, a warp on a
// run of the sort's work items, each lane adding its particles into its
// column of the warp's window in shared memory, which is summed and added to
// the grid once per cell of the run.  The cell lookup is the reference's
// Float32 LocateTable walk.

#include "vlb_internal.cuh"

namespace vlb {

int grid_for(const Ctx& c, int64_t n, int threads, int per_sm);

namespace {

constexpr int kDepThreads = 256;
constexpr int kDepLanes = 32;      // particle lanes per CTA, 8 threads (one z row each) per lane
constexpr int kDepStageMax = 1024;  // particles whose columns are staged at once: 1024 packed, 512 computed
constexpr int kDepRow = 68;        // floats per (lane, z row) in the reduction buffer: 64 + 4 against bank conflicts
constexpr double kFixedScale = 1099511627776.0;        // 2^40
constexpr double kFixedInv = 1.0 / 1099511627776.0;

// One CTA per occupied cell at a time (dynamic counter); a cell of the
// headline cloud holds about a thousand particles.  The cell's particles go
// in stages of 1024 (512 when computed): each thread puts the three table
// columns and the window test of four (two) particles into one int4 each of
// a double-buffered stage in shared memory while the CTA adds the previous
// stage, and the loads of the stage after are in flight meanwhile; one CTA
// barrier per stage (the columns stored as the offsets of their node rows).  With kPacked the
// columns and the window flag come packed from the sort's record move (four
// bytes a particle); otherwise the thread computes them from k and delta.  Thread
// (lane, q) owns the z row q of its lane's 8^3 sum: 64 float32
// accumulators as float2 pairs along x, so one packed FMA covers two outputs.
// At the cell's end the lane partials are summed over the lanes in a fixed
// order (in shared memory that the stages used) and added to the grid.
template <bool kPacked>
__global__ void __launch_bounds__(kDepThreads, 2) k_deposit_fine(
    const int32_t* __restrict__ occupied, const int32_t* __restrict__ bounds, DeviceScalars* dsc,
    int64_t Npad, const int32_t* __restrict__ k, const float* __restrict__ d, const uint32_t* __restrict__ cols,
    const float* __restrict__ nodes, int nk, int n, float x0, float h, float lo, float hi, float spacing, int nbdt,
    int ncol, float* rho, unsigned long long* rho_fixed, int mode) {
  extern __shared__ __align__(16) unsigned char smem[];
  float* nodes_s = reinterpret_cast<float*>(smem);                      // [ncol][8]
  unsigned char* work = smem + (((size_t)ncol * 8 * sizeof(float) + 15) & ~(size_t)15);
  constexpr int kPer = kPacked ? 4 : 2;  // particles a thread stages
  constexpr int kDepStage = kPer * kDepThreads;
  int4* cols_s = reinterpret_cast<int4*>(work);                         // [2][kDepStage]
  float* red_s = reinterpret_cast<float*>(work);                        // [kDepLanes][8][kDepRow], after the stages
  __shared__ int s_g, s_q;
  __shared__ int s_nout;
  const int tid = threadIdx.x;
  for (int e = tid; e < ncol * 8; e += kDepThreads) nodes_s[e] = nodes[e];
  if (tid == 0) s_nout = 0;
  const int nocc = dsc->noccupied;
  const int pl = tid / 8, q = tid % 8;
  int my_nout = 0;
  __syncthreads();
  // the columns of particle s (inside the cell) into the stage slot: from
  // the sort's packed columns (kPacked, in kk[0]) or from k and delta
  auto stage_one = [&](int s, int sh, const int (&kk)[3], const float (&dd)[3], int4* slot) {
    if (s >= sh) return;
    if (kPacked) {
      uint32_t pc = (uint32_t)kk[0];
      if (pc & kColsOutside) {
        pc = 0;  // column 1 on every axis
        ++my_nout;
      }
      // the node rows' offsets in the shared table (8 floats a column)
      *slot = make_int4((int)(pc & 1023u) * 8, (int)((pc >> 10) & 1023u) * 8, (int)((pc >> 20) & 1023u) * 8, 0);
      return;
    }
    bool inside = true;
    int cc[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const float p = fadd(fadd(x0, fmul((float)(kk[ax] - 1), h)), dd[ax]);
      inside = inside && (lo <= p) && (p <= hi);
      cc[ax] = table_column(dd[ax], spacing, nbdt, ncol);
    }
    if (!inside) { cc[0] = cc[1] = cc[2] = 1; ++my_nout; }
    // the node rows' offsets in the shared table (8 floats a column)
    *slot = make_int4((cc[0] - 1) * 8, (cc[1] - 1) * 8, (cc[2] - 1) * 8, 0);
  };
  auto load_one = [&](int s, int sh, int (&kk)[3], float (&dd)[3]) {
    if (s >= sh) return;
    if (kPacked) {
      kk[0] = (int)cols[s];
      return;
    }
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      kk[ax] = k[ax * Npad + s];
      dd[ax] = d[ax * Npad + s];
    }
  };
  // Cells go through a queue two deep: while cell g is added, the next cell
  // gn is known (with its bounds) and the one after is being claimed, so the
  // loads of gn's first stage go out during g's last stage.
  if (tid == 0) {
    s_g = (int)atomicAdd(&dsc->work_deposit, 1ull);
    s_q = (int)atomicAdd(&dsc->work_deposit, 1ull);
  }
  __syncthreads();
  int g = s_g, gn = s_q;
  int sl = 0, sh = 0, sln = 0, shn = 0;
  if (g < nocc) { sl = bounds[g]; sh = bounds[g + 1]; }
  if (gn < nocc) { sln = bounds[gn]; shn = bounds[gn + 1]; }
  int kr[kPer][3];
  float dr[kPer][3];
#pragma unroll
  for (int u = 0; u < kPer; ++u)
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      kr[u][ax] = 0;
      dr[u][ax] = 0.f;
    }
  // the loads of a cell's first stage, or of the next stage of this cell
  auto load_stage = [&](int base, int end) {
#pragma unroll
    for (int u = 0; u < kPer; ++u) load_one(base + u * kDepThreads + tid, end, kr[u], dr[u]);
  };
  // the loaded stage's columns into a stage buffer
  auto put_stage = [&](int base, int end, int4* dst) {
#pragma unroll
    for (int u = 0; u < kPer; ++u) stage_one(base + u * kDepThreads + tid, end, kr[u], dr[u], &dst[u * kDepThreads + tid]);
  };
  if (g < nocc) load_stage(sl, sh);
  while (g < nocc) {
    __syncthreads();  // every thread holds gn: the queue slot is free
    if (tid == 0) s_q = (int)atomicAdd(&dsc->work_deposit, 1ull);
    const int cell = occupied[g];
    int kx, ky, kz;
    cell_knots((uint32_t)cell, nk, kx, ky, kz);
    const bool fits = deposit_fits(kx, ky, kz, n);
    float2 acc[32];
#pragma unroll
    for (int a = 0; a < 32; ++a) acc[a] = make_float2(0.f, 0.f);
    // stage 0 from the registers, then the loads of the next stage to come
    put_stage(sl, sh, cols_s);
    if (sl + kDepStage < sh)
      load_stage(sl + kDepStage, sh);
    else if (gn < nocc)
      load_stage(sln, shn);
    __syncthreads();
    const int gnn = s_q;
    int slnn = 0, shnn = 0;
    if (gnn < nocc) { slnn = bounds[gnn]; shnn = bounds[gnn + 1]; }
    int buf = 0;
    for (int base = sl; base < sh; base += kDepStage) {
      // the next stage into the other buffer (its last readers passed the
      // barrier that ended the previous stage), and the loads of the one after
      const int nb = base + kDepStage;
      if (nb < sh) {
        put_stage(nb, sh, cols_s + (buf ^ 1) * kDepStage);
        if (nb + kDepStage < sh)
          load_stage(nb + kDepStage, sh);
        else if (gn < nocc)
          load_stage(sln, shn);
      }
      if (fits) {
        const int4* cur = cols_s + buf * kDepStage;
        const int cnt = min(kDepStage, sh - base);
        for (int t = pl; t < cnt; t += kDepLanes) {
          const int4 cc = cur[t];
          const float* vx = nodes_s + cc.x;
          const float* vy = nodes_s + cc.y;
          const float z = nodes_s[cc.z + q];
          const float4 xa = *reinterpret_cast<const float4*>(vx);
          const float4 xb = *reinterpret_cast<const float4*>(vx + 4);
          const float4 ya = *reinterpret_cast<const float4*>(vy);
          const float4 yb = *reinterpret_cast<const float4*>(vy + 4);
          const float2 x2[4] = {make_float2(xa.x, xa.y), make_float2(xa.z, xa.w), make_float2(xb.x, xb.y),
                                make_float2(xb.z, xb.w)};
          const float y[8] = {ya.x, ya.y, ya.z, ya.w, yb.x, yb.y, yb.z, yb.w};
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const float w = y[j] * z;
            const float2 w2 = make_float2(w, w);
#pragma unroll
            for (int a = 0; a < 4; ++a) acc[4 * j + a] = __ffma2_rn(x2[a], w2, acc[4 * j + a]);
          }
        }
      }
      __syncthreads();
      buf ^= 1;
    }
    if (fits) {
      // lane partials -> shared (the stages' memory), then a fixed-order
      // sum over the lanes that received particles
      float* row = red_s + (size_t)(pl * 8 + q) * kDepRow;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        *reinterpret_cast<float4*>(row + 8 * j) = make_float4(acc[4 * j].x, acc[4 * j].y, acc[4 * j + 1].x,
                                                              acc[4 * j + 1].y);
        *reinterpret_cast<float4*>(row + 8 * j + 4) = make_float4(acc[4 * j + 2].x, acc[4 * j + 2].y,
                                                                  acc[4 * j + 3].x, acc[4 * j + 3].y);
      }
      __syncthreads();
      const int nl = min(kDepLanes, sh - sl);
      const int bx = 2 * kx - 5, by = 2 * ky - 5, bz = 2 * kz - 5;
      for (int o = tid; o < 512; o += kDepThreads) {
        const int a = o & 7, jj = (o >> 3) & 7, kq = o >> 6;
        const float* src = red_s + (size_t)kq * kDepRow + 8 * jj + a;
        float v = 0.f;
        for (int l = 0; l < nl; ++l) v += src[(size_t)l * 8 * kDepRow];
        const size_t addr = (size_t)(bx + a) + (size_t)n * ((by + jj) + (size_t)n * (bz + kq));
        if (mode == VLB_DEPOSIT_FIXED64) {
          const long long iv = llrint((double)v * kFixedScale);
          if (iv) atomicAdd(&rho_fixed[addr], (unsigned long long)iv);
        } else if (v != 0.f) {
          atomicAdd(&rho[addr], v);
        }
      }
    }
    g = gn; sl = sln; sh = shn;
    gn = gnn; sln = slnn; shn = shnn;
  }
  atomicAdd(&s_nout, my_nout);
  __syncthreads();
  if (tid == 0 && s_nout) atomicAdd(&dsc->nout, s_nout);
}

// Per (j,k) column: sum_i rho[i,j,k] m0[i], times m0[j] m0[k].  One warp
// per column: lane l sums i = l, l+32, ... in order, then the fixed
// butterfly over the lanes.
__global__ void __launch_bounds__(256) k_charge_columns(const float* __restrict__ rho,
                                                        const unsigned long long* __restrict__ fixed,
                                                        const double* __restrict__ m0, int n,
                                                        double* __restrict__ partial) {
  const int t = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (t >= n * n) return;
  const int j = t % n, kq = t / n;
  double s = 0;
  if (fixed) {
    for (int i = lane; i < n; i += 32) s += (double)(long long)fixed[(size_t)t * n + i] * kFixedInv * m0[i];
  } else {
    for (int i = lane; i < n; i += 32) s += (double)rho[(size_t)t * n + i] * m0[i];
  }
  s = warp_sum(s);
  if (lane == 0) partial[t] = s * m0[j] * m0[kq];
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
// rho = raw * (N - nout) w / q with N and nout over the whole cloud (all
// shards): nout is read from xch[0], where the deposit published its own
// count and a sharded step the sum over the shards.
__global__ void k_charge_scale(float* __restrict__ rho, const unsigned long long* __restrict__ fixed, size_t tot,
                               const DeviceScalars* dsc, int64_t N, double w) {
  const double q = dsc->charge_raw;
  const float sc = (float)(((double)N - dsc->xch[0]) * w / q);
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (size_t)gridDim.x * blockDim.x) {
    const float v = fixed ? (float)((double)(long long)fixed[t] * kFixedInv) : rho[t];
    rho[t] = v * sc;
  }
}

// --------------------------------------------------------------- coarse
constexpr int kCicThreads = 256;
constexpr int kCicW = 4;                        // window points per axis
constexpr int kCicW3 = kCicW * kCicW * kCicW;   // 64 accumulators per lane

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

// The locate of one axis for the particles of one work item.  They share a
// fine cell, so their coarse left points lie in the item's window: the
// points anc .. anc + 2 after the anchor.  The item keeps the window's four
// coordinates in registers, and a particle inside (gt[anc], gt[anc + 3]]
// finds its point with two comparisons -- the point locate_cell finds --
// then reads its inverse gap and dual lengths in one round of independent
// loads instead of a chain; the weight takes the same arithmetic.  Any
// other particle takes locate_cell.
struct CicAxis {
  bool fast;
  float g0, g1, g2, g3;        // gt[anc .. anc + 3]
};

__device__ __forceinline__ void cic_axis(CicAxis& A, int anc, int ng, const float* gt) {
  A.fast = anc >= 0 && anc + 3 <= ng - 1;
  if (!A.fast) return;
  A.g0 = gt[anc]; A.g1 = gt[anc + 1]; A.g2 = gt[anc + 2]; A.g3 = gt[anc + 3];
}

// c = the first grid index with gt[c] >= x (0: outside), its weight w, and
// the inverse dual lengths of the points c - 1 and c.
__device__ __forceinline__ int cic_locate(const CicAxis& A, int anc, float x, float& w, float& il0, float& il1,
                                          const float* gt, const float* igap, const float* idl, int ng, float lx0,
                                          float linvw, const int32_t* cells, int ncells) {
  int c;
  if (A.fast && x > A.g0 && x <= A.g3) {
    const int o = (A.g1 < x) + (A.g2 < x);
    c = anc + 1 + o;
    const float gc = o == 0 ? A.g1 : (o == 1 ? A.g2 : A.g3);
    w = fsub(gc, x) * igap[c];
  } else {
    c = locate_cell(gt, igap, ng, lx0, linvw, cells, ncells, x, w);
  }
  if (c > 0) {
    il0 = idl[c - 1];
    il1 = idl[c];
  }
  return c;
}

// The two weights of one axis spread over the window's four points: the left
// point sits at offset l in [0, 2].
__device__ __forceinline__ void window_axis(int l, float w0, float w1, float (&f)[kCicW]) {
#pragma unroll
  for (int e = 0; e < kCicW; ++e) f[e] = e == l ? w0 : (e == l + 1 ? w1 : 0.f);
}

__device__ __forceinline__ void cic_add(float* rho, unsigned long long* fixed, size_t i, float v) {
  if (fixed) {
    const long long iv = llrint((double)v * kFixedScale);
    if (iv) atomicAdd(&fixed[i], (unsigned long long)iv);
  } else {
    atomicAdd(&rho[i], v);
  }
}

// The coarse density from its fixed-point accumulator.
__global__ void k_coarse_from_fixed(float* __restrict__ rho, const unsigned long long* __restrict__ fixed, size_t tot) {
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (size_t)gridDim.x * blockDim.x)
    rho[t] = (float)((double)(long long)fixed[t] * kFixedInv);
}

// One warp at a time on a run of kCicClaim consecutive work items of the
// cell sort (each at most `chunk` particles of one fine cell; a run usually
// lies in one or two cells), claimed from a dynamic counter.  The fine cell
// is one knot spacing wide and the coarse collocation gaps are at least
// 2.19 a0 against the fine h = 2.44 a0, so a cell's particles' left coarse
// points lie within two of the anchor, the point left of the cell's lower
// edge: a 4^3 window of coarse points holds all their corners.  Each lane
// adds its particles' eight trilinear corners into its own column of the
// warp's 64-entry window in shared memory (entry e of lane l at word
// 32 e + l: every update of lane l falls in bank l, whichever entries the
// lanes' particles reach).  When the cell changes, and at the end of the
// run, the warp flushes the window: lane l sums entries l and l + 32 over
// the 32 columns, column (l + j) mod 32 at step j (distinct banks across the
// lanes), and adds them to the grid.  Particles whose left point falls outside the window
// (cells clamped at the edge of the fine grid) add their corners with
// atomics directly.  The run's particles are contiguous in slot order; the
// warp walks them an iteration (32 particles of one item) at a time, reading
// each item's slots from the sort's item records, with the loads of the next
// kCicAhead iterations in flight.  Contributions carry charge / (wx wy wz)
// (src/devicemesh.jl:104); the walk is the reference's
// (src/kernels.jl:1083-1273) with the scatter grouped by cell.  With `fixed`
// the additions go to an int64 grid in fixed point (scale 2^40): the runs
// are fixed by the sort and each window's sums are taken in a fixed order,
// so the grid does not depend on which warp takes which run.
constexpr int kCicClaim = 8;
constexpr int kCicAhead = 2;  // iterations whose loads are in flight ahead of the additions
constexpr int kCicRow = 32;  // window row: entry e, lane l at e * 32 + l
constexpr int kCicWarps = kCicThreads / 32;

struct CicWin {
  int anc[3];
  CicAxis A[3];
};

__device__ __forceinline__ void cic_cell_window(CicWin& W, int kx, int ky, int kz, const float* gt,
                                                const float* igap, int ng, float lx0, float linvw,
                                                const int32_t* cells, int ncells, float x0f, float hf) {
  const int kc[3] = {kx, ky, kz};
  const float halfh = 0.5f * hf;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    float wdummy;
    const float edge = fsub(fadd(x0f, fmul((float)(kc[ax] - 1), hf)), halfh);
    const int c = locate_cell(gt, igap, ng, lx0, linvw, cells, ncells, edge, wdummy);
    W.anc[ax] = c > 0 ? c - 1 : -1000;
    cic_axis(W.A[ax], W.anc[ax], ng, gt);
  }
}

// The corners of one particle: into the lane's window column `col` (entry e
// at col[e * kCicRow]) when they fit, else to the grid.
__device__ __forceinline__ void cic_particle(const CicWin& W, int k0, int k1, int k2, float d0, float d1, float d2,
                                             float x0f, float hf, float charge, const float* gt, const float* igap,
                                             const float* idl, int ng, float lx0, float linvw, const int32_t* cells,
                                             int ncells, float* col, float* rho, unsigned long long* fixed) {
  const size_t n = ng, nn = n * n;
  const float px = fadd(fadd(x0f, fmul((float)(k0 - 1), hf)), d0);
  const float py = fadd(fadd(x0f, fmul((float)(k1 - 1), hf)), d1);
  const float pz = fadd(fadd(x0f, fmul((float)(k2 - 1), hf)), d2);
  float ax, ay, az, ix0, ix1, iy0, iy1, iz0, iz1;
  const int ix = cic_locate(W.A[0], W.anc[0], px, ax, ix0, ix1, gt, igap, idl, ng, lx0, linvw, cells, ncells);
  const int iy = cic_locate(W.A[1], W.anc[1], py, ay, iy0, iy1, gt, igap, idl, ng, lx0, linvw, cells, ncells);
  const int iz = cic_locate(W.A[2], W.anc[2], pz, az, iz0, iz1, gt, igap, idl, ng, lx0, linvw, cells, ncells);
  if (!(ix > 0 && iy > 0 && iz > 0)) return;
  const int i0 = ix - 1, j0 = iy - 1, m0 = iz - 1;  // 0-based left points
  const float wx0 = ax * ix0, wx1 = (1.f - ax) * ix1;
  const float wy0 = ay * iy0, wy1 = (1.f - ay) * iy1;
  const float wz0 = charge * az * iz0, wz1 = charge * (1.f - az) * iz1;
  const int lx = i0 - W.anc[0], ly = j0 - W.anc[1], lz = m0 - W.anc[2];
  if ((unsigned)lx <= kCicW - 2 && (unsigned)ly <= kCicW - 2 && (unsigned)lz <= kCicW - 2) {
    float* c = col + (size_t)(lx + kCicW * (ly + kCicW * lz)) * kCicRow;
    constexpr int X = kCicRow, Y = kCicW * kCicRow, Z = kCicW * kCicW * kCicRow;
    const float a00 = wx0 * wy0, a10 = wx1 * wy0, a01 = wx0 * wy1, a11 = wx1 * wy1;
    c[0] += a00 * wz0;
    c[X] += a10 * wz0;
    c[Y] += a01 * wz0;
    c[Y + X] += a11 * wz0;
    c[Z] += a00 * wz1;
    c[Z + X] += a10 * wz1;
    c[Z + Y] += a01 * wz1;
    c[Z + Y + X] += a11 * wz1;
  } else {
    const size_t b = (size_t)i0 + n * j0 + nn * m0;
    cic_add(rho, fixed, b, wx0 * wy0 * wz0);
    cic_add(rho, fixed, b + nn, wx0 * wy0 * wz1);
    cic_add(rho, fixed, b + n, wx0 * wy1 * wz0);
    cic_add(rho, fixed, b + n + nn, wx0 * wy1 * wz1);
    cic_add(rho, fixed, b + 1, wx1 * wy0 * wz0);
    cic_add(rho, fixed, b + 1 + nn, wx1 * wy0 * wz1);
    cic_add(rho, fixed, b + 1 + n, wx1 * wy1 * wz0);
    cic_add(rho, fixed, b + 1 + n + nn, wx1 * wy1 * wz1);
  }
}

// Whether x lies in (gt[anc], gt[anc + 3]] of an axis whose window is inside
// the grid: then its left point is one of the window's first three.
__device__ __forceinline__ bool cic_in_window(const CicAxis& A, float x) {
  return A.fast && x > A.g0 && x <= A.g3;
}

// One axis of a particle inside the window: offset l of its left point, and
// the two weights, with the arithmetic of cic_locate and cic_particle.
__device__ __forceinline__ void cic_axis_window(const CicAxis& A, int anc, float x, const float* igap,
                                                const float* idl, int& l, float& a, float& il0, float& il1) {
  l = (A.g1 < x) + (A.g2 < x);
  const int c = anc + 1 + l;
  const float gc = l == 0 ? A.g1 : (l == 1 ? A.g2 : A.g3);
  a = fsub(gc, x) * igap[c];
  il0 = idl[c - 1];
  il1 = idl[c];
}

// The corners of a particle whose three axes lie inside the window (the
// common case; the warp takes it when every lane's particle does): the same
// products as cic_particle, with no locate walk, no bounds test and no
// atomics.
__device__ __forceinline__ void cic_particle_window(const CicWin& W, float px, float py, float pz, float charge,
                                                    const float* igap, const float* idl, float* col) {
  int lx, ly, lz;
  float ax, ay, az, ix0, ix1, iy0, iy1, iz0, iz1;
  cic_axis_window(W.A[0], W.anc[0], px, igap, idl, lx, ax, ix0, ix1);
  cic_axis_window(W.A[1], W.anc[1], py, igap, idl, ly, ay, iy0, iy1);
  cic_axis_window(W.A[2], W.anc[2], pz, igap, idl, lz, az, iz0, iz1);
  const float wx0 = ax * ix0, wx1 = (1.f - ax) * ix1;
  const float wy0 = ay * iy0, wy1 = (1.f - ay) * iy1;
  const float wz0 = charge * az * iz0, wz1 = charge * (1.f - az) * iz1;
  float* c = col + (size_t)(lx + kCicW * (ly + kCicW * lz)) * kCicRow;
  constexpr int X = kCicRow, Y = kCicW * kCicRow, Z = kCicW * kCicW * kCicRow;
  const float a00 = wx0 * wy0, a10 = wx1 * wy0, a01 = wx0 * wy1, a11 = wx1 * wy1;
  c[0] += a00 * wz0;
  c[X] += a10 * wz0;
  c[Y] += a01 * wz0;
  c[Y + X] += a11 * wz0;
  c[Z] += a00 * wz1;
  c[Z + X] += a10 * wz1;
  c[Z + Y] += a01 * wz1;
  c[Z + Y + X] += a11 * wz1;
}

// The warp's window to the grid, then zeroed: lane l takes entries l and l + 32.
__device__ __forceinline__ void cic_flush(float* win, int lane, const CicWin& W, size_t n, float* rho,
                                          unsigned long long* fixed) {
  __syncwarp();
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int e = lane + 32 * h;
    float* row = win + (size_t)e * kCicRow;
    float v = 0.f;
#pragma unroll 8
    for (int j = 0; j < 32; ++j) {  // lane l reads word 32 e + (l + j) mod 32: bank (l + j) mod 32
      const int col = (lane + j) & 31;
      v += row[col];
      row[col] = 0.f;
    }
    if (v != 0.f) {
      const int ex = e % kCicW, ey = (e / kCicW) % kCicW, ez = e / (kCicW * kCicW);
      cic_add(rho, fixed, (size_t)(W.anc[0] + ex) + n * (W.anc[1] + ey) + n * n * (W.anc[2] + ez), v);
    }
  }
  __syncwarp();
}

// The k and delta of one lane's particle of an iteration.
struct CicLoad {
  int k[3];
  float d[3];
};

__global__ void __launch_bounds__(kCicThreads, 3) k_deposit_cic(
    const int4* __restrict__ item_rec, DeviceScalars* dsc, int64_t Npad, const int32_t* __restrict__ k,
    const float* __restrict__ d, const float* __restrict__ gt_g, int ng, float lx0, float linvw,
    const int32_t* __restrict__ cells_g, int ncells, const float* __restrict__ dl_g, float x0f, float hf,
    float charge, float* rho, unsigned long long* fixed) {
  extern __shared__ __align__(16) unsigned char smem[];
  float* wins = reinterpret_cast<float*>(smem);                 // [kCicWarps][kCicW3][kCicRow]
  float* gt = wins + kCicWarps * kCicW3 * kCicRow;              // [ng]
  float* igap = gt + ng;                                        // [ng] 1 / (gt[c] - gt[c-1])
  float* idl = igap + ng;                                       // [ng] 1 / dual length
  int32_t* cells = reinterpret_cast<int32_t*>(idl + ng);        // [ncells]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < ng; e += kCicThreads) {
    gt[e] = gt_g[e];
    igap[e] = e > 0 ? 1.f / (gt_g[e] - gt_g[e - 1]) : 0.f;
    idl[e] = 1.f / dl_g[e];
  }
  for (int e = tid; e < ncells; e += kCicThreads) cells[e] = cells_g[e];
  float* win = wins + (size_t)warp * kCicW3 * kCicRow;
  for (int e = lane; e < kCicW3 * kCicRow; e += 32) win[e] = 0.f;
  __syncthreads();
  const int nitems = dsc->nitems;
  const size_t n = ng;
  float* col = win + lane;
  // runs of kCicClaim items at fixed boundaries (guided claims, two items at a
  // time near the end, were measured slower: 0.131 against 0.118 ms at 8e6,
  // each short run flushing its own partial window)
  for (;;) {
    int i0 = 0;
    if (lane == 0) i0 = (int)atomicAdd(&dsc->work_cic, (unsigned long long)kCicClaim);
    i0 = __shfl_sync(0xffffffffu, i0, 0);
    if (i0 >= nitems) break;
    const int i1 = min(i0 + kCicClaim, nitems);
    // The run is a sequence of iterations (an item's particles s0 + 32 j + lane);
    // the loads run kCicAhead iterations ahead of the additions, across the
    // run's item boundaries, so that each warp keeps several rounds of k and
    // delta in flight.
    int4 rc = item_rec[i0];
    int citem = i0, cs = rc.y;
    int pitem = i0, ps = rc.y, pe = rc.z;
    CicLoad q[kCicAhead];
    auto fetch = [&](CicLoad& L) {
      if (pitem < i1 && ps + lane < pe) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          L.k[a] = k[a * Npad + ps + lane];
          L.d[a] = d[a * Npad + ps + lane];
        }
      }
      ps += 32;
      if (ps >= pe && ++pitem < i1) {
        const int4 r = item_rec[pitem];
        ps = r.y;
        pe = r.z;
      }
    };
#pragma unroll
    for (int t = 0; t < kCicAhead; ++t) fetch(q[t]);
    int gcode = -1;
    CicWin W;
    while (citem < i1) {
      if (rc.x != gcode) {
        if (gcode >= 0) cic_flush(win, lane, W, n, rho, fixed);
        cic_cell_window(W, rc.w & 1023, (rc.w >> 10) & 1023, rc.w >> 20, gt, igap, ng, lx0, linvw, cells, ncells,
                        x0f, hf);
        gcode = rc.x;
      }
      const CicLoad cur = q[0];
#pragma unroll
      for (int t = 0; t + 1 < kCicAhead; ++t) q[t] = q[t + 1];
      fetch(q[kCicAhead - 1]);
      const bool valid = cs + lane < rc.z;
      const float px = fadd(fadd(x0f, fmul((float)(cur.k[0] - 1), hf)), cur.d[0]);
      const float py = fadd(fadd(x0f, fmul((float)(cur.k[1] - 1), hf)), cur.d[1]);
      const float pz = fadd(fadd(x0f, fmul((float)(cur.k[2] - 1), hf)), cur.d[2]);
      const bool inside = cic_in_window(W.A[0], px) && cic_in_window(W.A[1], py) && cic_in_window(W.A[2], pz);
      if (__all_sync(0xffffffffu, inside || !valid)) {
        if (valid) cic_particle_window(W, px, py, pz, charge, igap, idl, col);
      } else if (valid) {
        cic_particle(W, cur.k[0], cur.k[1], cur.k[2], cur.d[0], cur.d[1], cur.d[2], x0f, hf, charge, gt, igap, idl,
                     ng, lx0, linvw, cells, ncells, col, rho, fixed);
      }
      cs += 32;
      if (cs >= rc.z && ++citem < i1) {
        rc = item_rec[citem];
        cs = rc.y;
      }
    }
    if (gcode >= 0) cic_flush(win, lane, W, n, rho, fixed);
  }
}

}  // namespace

size_t deposit_fine_smem(const Ctx& c) {
  const size_t stages = (size_t)2 * kDepStageMax * sizeof(int4);
  const size_t red = (size_t)kDepLanes * 8 * kDepRow * sizeof(float);
  return (((size_t)c.ncol * 8 * sizeof(float) + 15) & ~(size_t)15) + (stages > red ? stages : red);
}

size_t cic_smem(const Ctx& c);

void deposit_setup(Ctx& c) {
  VLB_CUDA(cudaFuncSetAttribute(k_deposit_fine<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)deposit_fine_smem(c)));
  VLB_CUDA(cudaFuncSetAttribute(k_deposit_fine<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)deposit_fine_smem(c)));
  VLB_CUDA(cudaFuncSetAttribute(k_deposit_cic, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cic_smem(c)));
  // three CTAs of each per SM need the largest shared-memory split
  VLB_CUDA(cudaFuncSetAttribute(k_deposit_fine<false>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  VLB_CUDA(cudaFuncSetAttribute(k_deposit_fine<true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  VLB_CUDA(cudaFuncSetAttribute(k_deposit_cic, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
}

__global__ void k_publish_nout(DeviceScalars* dsc) { dsc->xch[0] = (double)dsc->nout; }

// The raw deposit of this context's particles (no renormalisation): the part
// of a step that the shards sum.
void launch_deposit_fine_raw(Ctx& c, int mode) {
  Level& F = c.fine;
  const size_t tot = (size_t)F.n * F.n * F.n;
  Particles& P = c.part[c.cur];
  if (mode == VLB_DEPOSIT_FIXED64)
    VLB_CUDA(cudaMemsetAsync(c.rho_fixed, 0, tot * sizeof(unsigned long long), c.stream));
  else
    VLB_CUDA(cudaMemsetAsync(F.rho, 0, tot * sizeof(float), c.stream));
  VLB_CUDA(cudaMemsetAsync(&c.dsc->work_deposit, 0, sizeof(unsigned long long), c.stream));
  VLB_CUDA(cudaMemsetAsync(&c.dsc->nout, 0, sizeof(int32_t), c.stream));
  const int grid = c.num_sms * 2;
  if (c.cols_packed)
    k_deposit_fine<true><<<grid, kDepThreads, deposit_fine_smem(c), c.stream>>>(
        c.occupied, c.bounds, c.dsc, c.Npad, P.k, P.d, c.cols, c.nodes, F.nk, F.n, c.x0f, c.hf, c.lo_f, c.hi_f,
        c.spacing_f, c.nbdt, c.ncol, F.rho, c.rho_fixed, mode);
  else
    k_deposit_fine<false><<<grid, kDepThreads, deposit_fine_smem(c), c.stream>>>(
        c.occupied, c.bounds, c.dsc, c.Npad, P.k, P.d, c.cols, c.nodes, F.nk, F.n, c.x0f, c.hf, c.lo_f, c.hi_f,
        c.spacing_f, c.nbdt, c.ncol, F.rho, c.rho_fixed, mode);
  VLB_LAUNCHED(c);
  k_publish_nout<<<1, 1, 0, c.stream>>>(c.dsc);
  VLB_LAUNCHED(c);
}

// Total charge of the (summed) raw density and the renormalisation to
// (npart_global - nout) * charge (src/accelerator.jl:554-557).
void launch_deposit_fine_normalize(Ctx& c, double charge, int mode, int64_t npart_global) {
  Level& F = c.fine;
  const size_t tot = (size_t)F.n * F.n * F.n;
  const unsigned long long* fx = mode == VLB_DEPOSIT_FIXED64 ? c.rho_fixed : nullptr;
  const int cols = F.n * F.n;
  k_charge_columns<<<(cols + 7) / 8, 256, 0, c.stream>>>(F.rho, fx, F.dual_d, F.n, c.partials);
  VLB_LAUNCHED(c);
  k_charge_total<<<1, 1024, 0, c.stream>>>(c.partials, cols, &c.dsc->charge_raw);
  VLB_LAUNCHED(c);
  k_charge_scale<<<grid_for(c, (int64_t)tot, 256, 8), 256, 0, c.stream>>>(F.rho, fx, tot, c.dsc, npart_global,
                                                                           charge);
  VLB_LAUNCHED(c);
}

// The charge sum rho m0x m0y m0z of a float32 grid of level L into *out.
void launch_grid_charge(Ctx& c, Level& L, const float* rho, double* out) {
  const int cols = L.n * L.n;
  k_charge_columns<<<(cols + 7) / 8, 256, 0, c.stream>>>(rho, nullptr, L.dual_d, L.n, c.partials);
  VLB_LAUNCHED(c);
  k_charge_total<<<1, 1024, 0, c.stream>>>(c.partials, cols, out);
  VLB_LAUNCHED(c);
}

void launch_deposit_fine(Ctx& c, double charge, int mode) {
  launch_deposit_fine_raw(c, mode);
  launch_deposit_fine_normalize(c, charge, mode, c.N);
}

size_t cic_smem(const Ctx& c) {
  return (size_t)kCicWarps * kCicW3 * kCicRow * sizeof(float) + 3 * (size_t)c.coarse.n * sizeof(float) +
         (size_t)c.coarse.loc_ncell * sizeof(int32_t);
}

// The raw coarse deposit: into rho_coarse (float32) or, in fixed point,
// into its int64 accumulator (then launch_deposit_coarse_finish).
void launch_deposit_coarse(Ctx& c, double charge, int mode) {
  Level& C = c.coarse;
  const size_t tot = (size_t)C.n * C.n * C.n;
  Particles& P = c.part[c.cur];
  const bool fixed = mode == VLB_DEPOSIT_FIXED64;
  if (fixed)
    VLB_CUDA(cudaMemsetAsync(c.rho_fixed_c, 0, tot * sizeof(unsigned long long), c.stream));
  else
    VLB_CUDA(cudaMemsetAsync(C.rho, 0, tot * sizeof(float), c.stream));
  VLB_CUDA(cudaMemsetAsync(&c.dsc->work_cic, 0, sizeof(unsigned long long), c.stream));
  k_deposit_cic<<<c.num_sms * c.cic_cps, kCicThreads, cic_smem(c), c.stream>>>(
      c.item_rec, c.dsc, c.Npad, P.k, P.d, C.colloc, C.n, C.loc_x0, C.loc_invw, C.loc_cells, C.loc_ncell, C.dlen,
      c.x0f, c.hf, (float)charge, C.rho, fixed ? c.rho_fixed_c : nullptr);
  VLB_LAUNCHED(c);
}

// Fixed point: the (summed) accumulator into rho_coarse.
void launch_deposit_coarse_finish(Ctx& c, int mode) {
  if (mode != VLB_DEPOSIT_FIXED64) return;
  Level& C = c.coarse;
  const size_t tot = (size_t)C.n * C.n * C.n;
  k_coarse_from_fixed<<<grid_for(c, (int64_t)tot, 256, 8), 256, 0, c.stream>>>(C.rho, c.rho_fixed_c, tot);
  VLB_LAUNCHED(c);
}

}  // namespace vlb
