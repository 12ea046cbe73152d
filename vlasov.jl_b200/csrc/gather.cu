// Forces on the sorted cloud: the Gaussian-smoothed field gather with the
// projectile fused in, and the out-of-stencil tail.
//
// Gather (src/kernels.jl:339-470, host reference src/fields.jl:305-347):
// the particles of one work item (at most `chunk` of one occupied cell)
// share the cell's 10^3 stencil of csol; each particle's three table
// columns come from delta with the reference's Float32 arithmetic, and
//
//     F = -w ( sum c gx oy oz, sum c ox gy oz, sum c ox oy gz ).
//
// The sum over the stencil is reassociated (y first, then x, then z)
// against the reference's order, which changes rounding only.  Two forms:
// k_field_tc (the default) computes the sums over y of a whole item as
// 3xTF32 GEMMs on the tensor cores and finishes each particle on the CUDA
// cores (its table columns read from the sort's packed columns when the
// sort wrote them, the same table_column values the deposit uses); k_field computes everything with FP32 FMAs, one warp per item.  The projectile's Gaussian force
// (src/projectile.jl:95-108) is evaluated per particle at the position
// rebuilt from the *cell's* (clamped) knots, as the reference does, its
// reaction subtracted, and the four reaction sums reduced per CTA in float64.
//
// Tail (src/accelerator.jl:679-733): the particles whose 10^3 stencil leaves
// the fine grid take the coarse spline gradient (src/fields.jl:358-393) in
// float64, or nothing outside both grids, plus the ball-softened projectile
// reaction (src/projectile.jl:79-80).  Their Gaussian reaction sums go to the
// projectile like everyone else's (the ball's, in the CPU path's softening).
// The reference runs this part on the host after a device-to-host copy; here
// it stays on the device.
//
// The softening (DeviceScalars::proj_soft) is the reference device path's
// (Gaussian for stencil particles, ball for the tail) or its CPU path's
// (the ball everywhere, src/projectile.jl:203-232).

#include "tc_util.cuh"
#include "vlb_internal.cuh"

namespace vlb {

int grid_for(const Ctx& c, int64_t n, int threads, int per_sm);

namespace {

using namespace tc;

constexpr int kGThreads = 256;

// src/projectile.jl:86-108, Float32
__device__ __forceinline__ float gaussian_force_kernel(float r2, float sigma) {
  const float u2 = r2 / (sigma * sigma);
  if (u2 <= 0.25f) {
    const float S[7] = {1.f / 3, -1.f / 10, 1.f / 56, -1.f / 432, 1.f / 4224, -1.f / 49920, 1.f / 685440};
    float p = 0.f;
#pragma unroll
    for (int k = 6; k >= 0; --k) p = S[k] + u2 * p;
    return 0.7978845608028654f * p / (sigma * sigma * sigma);
  }
  const float r = sqrtf(r2);
  const float x = r / (1.4142135623730951f * sigma);
  return (erff(x) - 0.7978845608028654f * (r / sigma) * expf(-u2 / 2.f)) / (r2 * r);
}

struct ProjF {
  float px, py, pz, coef, sigma, R;
  bool on, ball;
};

__device__ __forceinline__ ProjF load_proj(const DeviceScalars* dsc, double w) {
  ProjF p;
  p.on = dsc->proj_active != 0;
  p.px = (float)dsc->proj_pos[0];
  p.py = (float)dsc->proj_pos[1];
  p.pz = (float)dsc->proj_pos[2];
  p.coef = p.on ? (float)(-w * dsc->proj_charge) : 0.f;
  p.sigma = p.on ? (float)dsc->proj_sigma : 1.f;
  p.R = p.on ? (float)dsc->proj_ball : 1.f;
  p.ball = dsc->proj_soft == VLB_SOFTENING_BALL;
  p.on = p.on && p.coef != 0.f;
  return p;
}

// force_kernel(BallSoftening(R), r2) (src/projectile.jl:79-80)
__device__ __forceinline__ float ball_force_kernel(float r2, float R) {
  return r2 > R * R ? 1.f / (r2 * sqrtf(r2)) : 1.f / (R * R * R);
}

// The projectile's term at the position rebuilt from a cell's knots: the
// Gaussian of the reference's device path, or with P.ball the ball of its CPU
// path (src/projectile.jl:203-232).  (fx2, fy2, fz2) is the reaction the
// particle's force loses and the projectile gains; e its share of the
// electrons' energy sum: erf(r / sqrt(2) sigma) / r (Gaussian), or
// uniform_sphere_potential(1, R, r) (ball, src/meanfield.jl:52-54).
__device__ __forceinline__ void proj_term(const ProjF& P, int kx, int ky, int kz, float dx0, float dy0, float dz0,
                                          float x0, float h, float& fx2, float& fy2, float& fz2, float& e) {
  const float px = fadd(fadd(x0, fmul((float)(kx - 1), h)), dx0);
  const float py = fadd(fadd(x0, fmul((float)(ky - 1), h)), dy0);
  const float pz = fadd(fadd(x0, fmul((float)(kz - 1), h)), dz0);
  const float dx = P.px - px, dy = P.py - py, dz = P.pz - pz;
  const float d2 = dx * dx + dy * dy + dz * dz;
  const float r = sqrtf(d2);
  float mm;
  if (P.ball) {
    mm = P.coef * ball_force_kernel(d2, P.R);
    e = r < P.R ? -(3.f - (r / P.R) * (r / P.R)) / (2.f * P.R) : -1.f / r;
  } else if (d2 >= 40.5f * (P.sigma * P.sigma)) {
    // x = r / (sqrt(2) sigma) >= 4.5: 1 - erf(x) < 2e-10 and (2 / sqrt(pi)) x exp(-x^2) < 9e-9, both
    // below half an ulp of 1 (2^-25), so the kernel's numerator and erf(x) round to 1: the far field
    // 1 / r^3 and the energy share 1 / r, as the full expressions give them
    mm = P.coef * (1.f / (d2 * r));
    e = 1.f / r;
  } else {
    mm = P.coef * gaussian_force_kernel(d2, P.sigma);
    e = r < 1.0e-4f * P.sigma ? 0.7978845608f / P.sigma : erff(r / 1.4142135624f / P.sigma) / r;
  }
  fx2 = mm * dx;
  fy2 = mm * dy;
  fz2 = mm * dz;
}

__device__ __forceinline__ void load10(const float* __restrict__ tab, int col, float* v) {
  const float2* p = reinterpret_cast<const float2*>(tab + (size_t)(col - 1) * 10);
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    const float2 t = __ldg(p + a);
    v[2 * a] = t.x;
    v[2 * a + 1] = t.y;
  }
}

// The projectile's reaction sums are reduced in a fixed order, so that a
// step gives the same sums whichever CTA takes which work item: one partial
// per work item of the gather (the warp's sum over the item's particles),
// one per CTA of the tail, summed by k_red_total.

// This CTA's sums into out[4] (no atomics).
__device__ __forceinline__ void block_red(float ax, float ay, float az, float ae, double* out) {
  __shared__ double sh[4][kGThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double v[4] = {ax, ay, az, ae};
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    v[c] = warp_sum(v[c]);
    if (lane == 0) sh[c][w] = v[c];
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = 0;
    for (int ww = 0; ww < kGThreads / 32; ++ww) s += sh[threadIdx.x][ww];
    out[threadIdx.x] = s;
  }
}

// Sum of the four components over [begin, end) of a partials array, by
// one block in a fixed order (strided by thread, then a tree); thread c < 4
// returns component c.
__device__ __forceinline__ double block_sum4(const double* __restrict__ p, int begin, int end) {
  __shared__ double sh[4][256];
  const int t = threadIdx.x;
  double s[4] = {0, 0, 0, 0};
  for (int i = begin + t; i < end; i += blockDim.x)
#pragma unroll
    for (int c = 0; c < 4; ++c) s[c] += p[4 * (size_t)i + c];
#pragma unroll
  for (int c = 0; c < 4; ++c) sh[c][t] = s[c];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (t < o)
#pragma unroll
      for (int c = 0; c < 4; ++c) sh[c][t] += sh[c][t + o];
    __syncthreads();
  }
  const double r = t < 4 ? sh[t][0] : 0.0;
  __syncthreads();
  return r;
}

// First level: block b sums the work items of its contiguous share (the
// shares depend only on the item count and the grid).
__global__ void __launch_bounds__(256) k_red_blocks(const double* __restrict__ items, const DeviceScalars* dsc,
                                                    double* __restrict__ block_out) {
  const int nitems = dsc->nitems;
  const int per = (nitems + gridDim.x - 1) / gridDim.x;
  const int b0 = min(nitems, (int)blockIdx.x * per), b1 = min(nitems, b0 + per);
  const double r = block_sum4(items, b0, b1);
  if (threadIdx.x < 4) block_out[4 * blockIdx.x + threadIdx.x] = r;
}

// red[c] = the block partials, then the tail's, in a fixed order.
__global__ void __launch_bounds__(256) k_red_total(const double* __restrict__ blocks, int nblocks,
                                                   const double* __restrict__ tail, int ntail, DeviceScalars* dsc) {
  const double a = block_sum4(blocks, 0, nblocks);
  const double b = block_sum4(tail, 0, ntail);
  if (threadIdx.x < 4) dsc->red[threadIdx.x] = a + b;
}

// One warp per work item (at most `chunk` particles of one occupied cell),
// items taken from a dynamic counter.  The warp stages its cell's 10^3
// stencil in its own slice of shared memory (kept while consecutive items
// share the cell) and takes 32 particles at a time, one per lane.  No
// barrier but __syncwarp.  All sixty table values of the particle live in
// registers; every stencil row read from shared memory (a broadcast: the
// whole warp reads the same row) feeds ten independent packed FMAs.
constexpr int kRow = 12;            // padded stencil row (10 values, 16-byte aligned)
constexpr int kTile = 10 * 10 * kRow;

__global__ void __launch_bounds__(kGThreads) k_field(
    const int32_t* __restrict__ occupied, const int32_t* __restrict__ bounds,
    const int32_t* __restrict__ chunk_start, const int32_t* __restrict__ item_cell, DeviceScalars* dsc, int64_t Npad,
    const float* __restrict__ d, const float* __restrict__ csol, int n, int nk, const float* __restrict__ ov,
    const float* __restrict__ gr, int nbdt, int ncol, float spacing, float x0, float h, double w,
    float* __restrict__ force, int chunk, double* __restrict__ red_items) {
  __shared__ __align__(16) float tiles[kGThreads / 32][kTile];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  float* tile = tiles[wid];
  const int nitems = dsc->nitems;
  const ProjF P = load_proj(dsc, w);
  const float wf = (float)w;
  int cached = -1;
  for (;;) {
    int item = 0;
    if (lane == 0) item = (int)atomicAdd(&dsc->work_gather, 1ull);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= nitems) break;
    const int g = item_cell[item];
    int kx, ky, kz;
    cell_knots((uint32_t)occupied[g], nk, kx, ky, kz);
    if (!field_fits(kx, ky, kz, n)) {  // the tail takes these
      if (lane < 4) red_items[4 * (size_t)item + lane] = 0.0;
      continue;
    }
    if (g != cached) {
      __syncwarp();
      const int bx = 2 * kx - 6, by = 2 * ky - 6, bz = 2 * kz - 6;  // 0-based stencil corner
      for (int e = lane; e < 1000; e += 32) {
        const int ii = e % 10, r = e / 10;  // r = jj + 10 kk
        const int jj = r % 10, kk = r / 10;
        tile[r * kRow + ii] = csol[(size_t)(bx + ii) + (size_t)n * ((by + jj) + (size_t)n * (bz + kk))];
      }
      cached = g;
      __syncwarp();
    }
    const int s0 = bounds[g] + (item - chunk_start[g]) * chunk;
    const int s1 = min(s0 + chunk, bounds[g + 1]);
    float ax = 0.f, ay = 0.f, az = 0.f, ae = 0.f;
    for (int s = s0 + lane; s < s1; s += 32) {
      const float dx0 = d[s], dy0 = d[Npad + s], dz0 = d[2 * Npad + s];
      const int cx = table_column(dx0, spacing, nbdt, ncol);
      const int cy = table_column(dy0, spacing, nbdt, ncol);
      const int cz = table_column(dz0, spacing, nbdt, ncol);
      // x columns as pairs of neighbouring stencil points; y values as
      // broadcast pairs, for the packed FMA
      float2 ox2[5], gx2[5];
      {
        const float2* po = reinterpret_cast<const float2*>(ov + (size_t)(cx - 1) * 10);
        const float2* pg = reinterpret_cast<const float2*>(gr + (size_t)(cx - 1) * 10);
#pragma unroll
        for (int a = 0; a < 5; ++a) { ox2[a] = __ldg(po + a); gx2[a] = __ldg(pg + a); }
      }
      float2 oy2[10], gy2[10];
      {
        float oy[10], gy[10];
        load10(ov, cy, oy);
        load10(gr, cy, gy);
#pragma unroll
        for (int j = 0; j < 10; ++j) { oy2[j] = make_float2(oy[j], oy[j]); gy2[j] = make_float2(gy[j], gy[j]); }
      }
      float ozr[10], gzr[10];
      load10(ov, cz, ozr);
      load10(gr, cz, gzr);
      float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
      for (int kk = 0; kk < 10; ++kk) {
        const float oz = ozr[kk], gz = gzr[kk];
        const float* plane = tile + kk * 10 * kRow;
        // y first: Yo[a] = sum_j c[a,j] oy_j, Yg[a] = sum_j c[a,j] gy_j, ten
        // independent packed accumulators per row
        float2 yo[5], yg[5];
#pragma unroll
        for (int a = 0; a < 5; ++a) { yo[a] = make_float2(0.f, 0.f); yg[a] = make_float2(0.f, 0.f); }
#pragma unroll
        for (int jj = 0; jj < 10; ++jj) {
          const float4 c0 = *reinterpret_cast<const float4*>(plane + jj * kRow);
          const float4 c1 = *reinterpret_cast<const float4*>(plane + jj * kRow + 4);
          const float2 c2 = *reinterpret_cast<const float2*>(plane + jj * kRow + 8);
          const float2 cp[5] = {make_float2(c0.x, c0.y), make_float2(c0.z, c0.w), make_float2(c1.x, c1.y),
                                make_float2(c1.z, c1.w), c2};
#pragma unroll
          for (int a = 0; a < 5; ++a) {
            yo[a] = __ffma2_rn(cp[a], oy2[jj], yo[a]);
            yg[a] = __ffma2_rn(cp[a], gy2[jj], yg[a]);
          }
        }
        // then x: tx = sum_a gx_a Yo[a], ty = sum_a ox_a Yg[a], tz = sum_a ox_a Yo[a]
        float2 tx2 = make_float2(0.f, 0.f), ty2 = make_float2(0.f, 0.f), tz2 = make_float2(0.f, 0.f);
#pragma unroll
        for (int a = 0; a < 5; ++a) {
          tx2 = __ffma2_rn(gx2[a], yo[a], tx2);
          ty2 = __ffma2_rn(ox2[a], yg[a], ty2);
          tz2 = __ffma2_rn(ox2[a], yo[a], tz2);
        }
        sx = fmaf(oz, tx2.x + tx2.y, sx);
        sy = fmaf(oz, ty2.x + ty2.y, sy);
        sz = fmaf(gz, tz2.x + tz2.y, sz);
      }
      float fx = -wf * sx, fy = -wf * sy, fz = -wf * sz;
      if (P.on) {
        float fx2, fy2, fz2, e;
        proj_term(P, kx, ky, kz, dx0, dy0, dz0, x0, h, fx2, fy2, fz2, e);
        fx -= fx2;
        fy -= fy2;
        fz -= fz2;
        ax += fx2;
        ay += fy2;
        az += fz2;
        ae += e;
      }
      force[s] = fx;
      force[Npad + s] = fy;
      force[2 * Npad + s] = fz;
    }
    // this item's reaction sums: lane order, then a fixed butterfly
    double v[4] = {ax, ay, az, ae};
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) v[cc] = warp_sum(v[cc]);
    if (lane == 0) {
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) red_items[4 * (size_t)item + cc] = v[cc];
    }
  }
}

// ------------------------------------------------ gather on the tensor cores
// The same gather with its sums over y on the tensor cores.  For the
// particles p of one work item (at most 128: one per thread and per
// tensor-memory lane) and the cell's stencil c[kk][jj][ii] (z, y, x),
//
//     Yo[p, 10 kk + ii] = sum_jj oy_p[jj] c[kk][jj][ii],   Yg: gy_p likewise,
//
// are two GEMMs with M = 128 particles, N = 100 stencil columns (padded to
// 112) and K = 10, sharing B[n, jj] = c[kk][jj][ii].  Both run in 3xTF32 in
// one accumulation each: along K, A = [a_hi | a_lo | a_hi] and
// B = [c_hi | c_hi | c_lo] (K = 30, padded to 32), so that
// D = a_hi c_hi + a_lo c_hi + a_hi c_lo with hi = rna_tf32(x) and
// lo = rna_tf32(x - hi): the dropped a_lo c_lo and the tails' rounding are of
// order 2^-22 of the terms, FP32 accuracy.  Each thread then reads its
// particle's rows of Yo and Yg from tensor memory and finishes on the CUDA
// cores with packed FMAs: x, then z (165 FFMA2 + 30 FMA a particle in place
// of the 1,150 FFMA2 of k_field).  Two CTAs per SM, 256 tensor-memory columns
// each (Yo in [0, 112), Yg in [128, 240)).
//
// Pipeline, one iteration per item t: the loads go out first (delta of item
// t+2, cell data of t+3 (used at the end of the iteration), item_cell of
// t+4, the six tables of item t+1 as three 80-byte rows of the interleaved
// overlap/gradient table and, when its cell differs from the staged one,
// its stencil as one TMA tile copy); then the threads wait for item t's
// MMAs (issued at the end of the previous iteration), read D, finish item t
// with the tables loaded one iteration earlier, and only then split item
// t+1's y tables and stencil into the operand buffers (single: their last
// reader has completed) and hand them to the MMA.  Items go round-robin to
// the CTAs (item = blockIdx.x + t gridDim.x).  The reaction sums of an item:
// each warp's float butterfly, then the four warps in order, in float64.
// Every wait is bounded.
constexpr int kFtThreads = 128;
constexpr int kFtRows = 128;                       // the MMA's M: particles per item at most
constexpr int kFtN = 112;                          // the MMA's N: 100 stencil columns, padded
constexpr unsigned kFtA = 128u * 128u;             // one A operand: 128 rows x 32 TF32
constexpr unsigned kFtB = (unsigned)kFtN * 128u;   // the B operand: 112 rows x 32 TF32
// One A operand per sum (Yo, Yg) and one B: item t+1's rows are written only
// after item t's MMAs completed, so single buffers suffice and leave the SM's
// L1 room for the interleaved tables.
constexpr unsigned kFtStage = 2u * kFtA + kFtB;  // the raw stencil tile (1024-byte aligned)
constexpr int kFtBoxX = 20;                        // floats per staged x row: 80 bytes, 16-byte multiple
constexpr unsigned kFtStageBytes = 10u * 10u * kFtBoxX * 4u;
constexpr unsigned kFtBars = kFtStage + kFtStageBytes;
constexpr unsigned kFtSmem = kFtBars + 32u;        // + three mbarriers and the tensor-memory slot
constexpr unsigned kFtCols = 256;
constexpr unsigned kFtColG = 128;                  // first column of Yg

// Byte offset of K group kg (4 TF32) of row r in a K-major operand of 32
// TF32 per row, no swizzle: 8 x 16-byte core matrices, the 8 K groups of a
// row group contiguous (LBO 128 bytes between K neighbours, SBO 1024 bytes
// between row groups).
__device__ __forceinline__ unsigned ft_off(int r, int kg) {
  return (unsigned)((r >> 3) * 1024 + kg * 128 + (r & 7) * 16);
}

struct FtItem {
  int item;         // -1: none
  int code;         // occupied cell code
  int kx, ky, kz;   // its knots
  int s0, s1;       // particle slots
  bool has;         // the stencil fits: MMAs and forces
};

// One particle of an item: delta, slot, and the six table columns as
// neighbour pairs (ten values each).
struct FtPart {
  float dx, dy, dz;
  int s;
  bool valid;
  float2 oy[5], gy[5], ox[5], gx[5], oz[5], gz[5];
};

// An item's record as loaded (used an iteration later, so that no thread
// waits on the load): the sort writes one int4 per work item -- its cell
// code, first slot, end slot and the cell's knots packed 10 bits each.
struct FtRaw {
  int item;
  int4 rec;
};

__device__ __forceinline__ FtRaw ft_load_item(int item, int nitems, const int4* __restrict__ items) {
  FtRaw r{-1, make_int4(0, 0, 0, 0)};
  if (item >= nitems) return r;
  r.item = item;
  r.rec = items[item];
  return r;
}

__device__ __forceinline__ FtItem ft_derive(const FtRaw& r, int n) {
  FtItem it{-1, 0, 0, 0, 0, 0, 0, false};
  if (r.item < 0) return it;
  it.item = r.item;
  it.code = r.rec.x;
  it.kx = r.rec.w & 1023;
  it.ky = (r.rec.w >> 10) & 1023;
  it.kz = r.rec.w >> 20;
  it.has = field_fits(it.kx, it.ky, it.kz, n);
  it.s0 = r.rec.y;
  it.s1 = r.rec.z;
  return it;
}

// A column's overlap and gradient rows as neighbour pairs, from the
// interleaved table (80-byte rows: five 16-byte loads).
__device__ __forceinline__ void ft_load_cols(const float4* __restrict__ ovgr, int col, float2 (&o)[5],
                                             float2 (&g)[5]) {
  const float4* p = ovgr + (size_t)(col - 1) * 5;
  const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), e = __ldg(p + 3), f = __ldg(p + 4);
  o[0] = make_float2(a.x, a.y);
  o[1] = make_float2(a.z, a.w);
  o[2] = make_float2(b.x, b.y);
  o[3] = make_float2(b.z, b.w);
  o[4] = make_float2(c.x, c.y);
  g[0] = make_float2(c.z, c.w);
  g[1] = make_float2(e.x, e.y);
  g[2] = make_float2(e.z, e.w);
  g[3] = make_float2(f.x, f.y);
  g[4] = make_float2(f.z, f.w);
}

// Row r of an A operand from the ten values v: [hi | lo | hi | 0 0].
__device__ __forceinline__ void ft_store_a(unsigned char* A, int r, const float2 (&v2)[5]) {
  float hi[10], lo[10];
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    hi[2 * j] = tf32_rna(v2[j].x);
    hi[2 * j + 1] = tf32_rna(v2[j].y);
    lo[2 * j] = tf32_rna(__fsub_rn(v2[j].x, hi[2 * j]));
    lo[2 * j + 1] = tf32_rna(__fsub_rn(v2[j].y, hi[2 * j + 1]));
  }
  auto at = [&](int kg) { return reinterpret_cast<float4*>(A + ft_off(r, kg)); };
  *at(0) = make_float4(hi[0], hi[1], hi[2], hi[3]);
  *at(1) = make_float4(hi[4], hi[5], hi[6], hi[7]);
  *at(2) = make_float4(hi[8], hi[9], lo[0], lo[1]);
  *at(3) = make_float4(lo[2], lo[3], lo[4], lo[5]);
  *at(4) = make_float4(lo[6], lo[7], lo[8], lo[9]);
  *at(5) = make_float4(hi[0], hi[1], hi[2], hi[3]);
  *at(6) = make_float4(hi[4], hi[5], hi[6], hi[7]);
  *at(7) = make_float4(hi[8], hi[9], 0.f, 0.f);
}

// The cell's 10^3 stencil of the fine coefficients staged by the TMA unit:
// one box of 20 x 10 x 10 floats of the row-padded copy (pitch a multiple of
// four floats), x from the stencil's first index rounded down to a multiple
// of four (16 bytes: the box's x coordinate must be), y and z from the
// stencil's first rows, into a dense [z][y][x] tile, completing on the
// stencil's mbarrier (8,000 bytes).  Thread 0 arms the barrier and issues it.
// The 20-float rows put the tile's z planes 200 words apart, eight banks, so
// a warp's reads of one y row conflict at most two ways.
__device__ __forceinline__ void ft_stage_b(const FtItem& it, int t, const CUtensorMap* map, unsigned char* raw,
                                           unsigned bar) {
  if (t == 0) {
    mbar_expect_tx(bar, kFtStageBytes);
    tma_load_3d(smem_u32(raw), map, (2 * it.kx - 6) & ~3, 2 * it.ky - 6, 2 * it.kz - 6, bar);
  }
}

// Row t < 100 (t = 10 kk + ii) of a cell's stencil from the staged tile:
// c[jj] = coefficient (ii, jj, kk) of the stencil, at x offset
// ((2 kx - 6) & 3) + ii of the tile's row (kk, jj).
__device__ __forceinline__ void ft_read_b(const FtItem& it, int t, const unsigned char* raw, float (&c)[10]) {
  const int kk = t / 10, ii = t - 10 * kk;
  const float* rf = reinterpret_cast<const float*>(raw) + kFtBoxX * 10 * kk + ((2 * it.kx - 6) & 3) + ii;
#pragma unroll
  for (int jj = 0; jj < 10; ++jj) c[jj] = rf[kFtBoxX * jj];
}

// That row of the B operand: [hi | hi | lo | 0 0].  Rows 100..111 are never
// written: they only feed the D columns that nothing reads.
__device__ __forceinline__ void ft_store_b(unsigned char* B, int t, const float (&c)[10]) {
  float H[10], Lo[10];
#pragma unroll
  for (int jj = 0; jj < 10; ++jj) {
    H[jj] = tf32_rna(c[jj]);
    Lo[jj] = tf32_rna(__fsub_rn(c[jj], H[jj]));
  }
  auto at = [&](int kg) { return reinterpret_cast<float4*>(B + ft_off(t, kg)); };
  *at(0) = make_float4(H[0], H[1], H[2], H[3]);
  *at(1) = make_float4(H[4], H[5], H[6], H[7]);
  *at(2) = make_float4(H[8], H[9], H[0], H[1]);
  *at(3) = make_float4(H[2], H[3], H[4], H[5]);
  *at(4) = make_float4(H[6], H[7], H[8], H[9]);
  *at(5) = make_float4(Lo[0], Lo[1], Lo[2], Lo[3]);
  *at(6) = make_float4(Lo[4], Lo[5], Lo[6], Lo[7]);
  *at(7) = make_float4(Lo[8], Lo[9], 0.f, 0.f);
}

// The x and z sums of one particle from its rows of Yo and Yg at lane_base:
// for each z plane kk, packed FMAs over the x pairs (ii, ii+1) (a pair never
// straddles a plane or a 16-column group), then the plane's z weight.
__device__ __forceinline__ void ft_finish(unsigned lane_base, const FtPart& p, float& sx, float& sy, float& sz) {
  sx = sy = sz = 0.f;
  // two chains per sum: the pairs a = 0, 2, 4 and a = 1, 3
  float2 U0 = make_float2(0.f, 0.f), V0 = U0, W0 = U0, U1 = U0, V1 = U0, W1 = U0;
#pragma unroll
  for (int q = 0; q < 7; ++q) {
    unsigned yo[16], yg[16];
    tmem_ld16(lane_base + 16u * q, yo);
    tmem_ld16(lane_base + kFtColG + 16u * q, yg);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; j += 2) {
      const int nn = 16 * q + j;
      if (nn < 100) {
        const int kk = nn / 10, a = (nn % 10) / 2;
        const float2 Yo = make_float2(__uint_as_float(yo[j]), __uint_as_float(yo[j + 1]));
        const float2 Yg = make_float2(__uint_as_float(yg[j]), __uint_as_float(yg[j + 1]));
        if (a & 1) {
          U1 = __ffma2_rn(p.gx[a], Yo, U1);
          V1 = __ffma2_rn(p.ox[a], Yg, V1);
          W1 = __ffma2_rn(p.ox[a], Yo, W1);
        } else {
          U0 = __ffma2_rn(p.gx[a], Yo, U0);
          V0 = __ffma2_rn(p.ox[a], Yg, V0);
          W0 = __ffma2_rn(p.ox[a], Yo, W0);
        }
        if (a == 4) {
          const float oz = (kk & 1) ? p.oz[kk >> 1].y : p.oz[kk >> 1].x;
          const float gz = (kk & 1) ? p.gz[kk >> 1].y : p.gz[kk >> 1].x;
          sx = fmaf(oz, (U0.x + U0.y) + (U1.x + U1.y), sx);
          sy = fmaf(oz, (V0.x + V0.y) + (V1.x + V1.y), sy);
          sz = fmaf(gz, (W0.x + W0.y) + (W1.x + W1.y), sz);
          U0 = V0 = W0 = U1 = V1 = W1 = make_float2(0.f, 0.f);
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kFtThreads, 2) k_field_tc(
    const int4* __restrict__ items, DeviceScalars* dsc, int64_t Npad,
    const float* __restrict__ d, const __grid_constant__ CUtensorMap csol_map, int n, int nk,
    const float4* __restrict__ ovgr, int nbdt, int ncol, float spacing, float x0, float h, double w,
    float* __restrict__ force, int chunk, double* __restrict__ red_items, const uint32_t* __restrict__ cols) {
  extern __shared__ __align__(1024) unsigned char ftsm[];
  __shared__ double red[2][4][4];
  uint64_t* bars = reinterpret_cast<uint64_t*>(ftsm + kFtBars);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(ftsm + kFtBars + 24);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nitems = dsc->nitems;
  const ProjF P = load_proj(dsc, w);
  const float wf = (float)w;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kFtCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  unsigned char* raw = ftsm + kFtStage;
  const unsigned sbar = smem_u32(&bars[2]);
  if (tid == 0) {
    mbar_init(smem_u32(&bars[0]), 1);
    mbar_init(smem_u32(&bars[1]), 1);
    mbar_init(sbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const unsigned tmem = *tmem_slot;
  const unsigned lane_base = tmem + ((unsigned)(32 * warp) << 16);
  const unsigned sbase = smem_u32(ftsm);
  const unsigned idesc = (1u << 4)                          // D: F32
                         | (2u << 7) | (2u << 10)            // A, B: TF32, both K-major
                         | ((unsigned)(kFtN >> 3) << 17)     // N
                         | ((unsigned)(kFtRows >> 4) << 24); // M

  // delta of the particle of item `it`, and in dd[3] the sort's packed
  // table columns when they were written
  auto load_delta = [&](const FtItem& it, float (&dd)[4]) {
    if (!it.has) return;
    const int s = it.s0 + tid;
    if (s < it.s1) {
      dd[0] = d[s];
      dd[1] = d[Npad + s];
      dd[2] = d[2 * Npad + s];
      if (cols) dd[3] = __uint_as_float(cols[s]);
    }
  };

  // the loads of a particle of item `it` whose delta is dd: its six tables
  auto load_part = [&](const FtItem& it, const float (&dd)[4], FtPart& p) {
    p.valid = false;
    p.s = 0;
    if (!it.has) return;
    const int s = it.s0 + tid;
    p.s = s;
    p.valid = s < it.s1;
    if (!p.valid) return;
    p.dx = dd[0];
    p.dy = dd[1];
    p.dz = dd[2];
    int cx, cy, cz;
    if (cols) {
      const uint32_t pc = __float_as_uint(dd[3]);
      cx = (int)(pc & 1023u) + 1;
      cy = (int)((pc >> 10) & 1023u) + 1;
      cz = (int)((pc >> 20) & 1023u) + 1;
    } else {
      cx = table_column(p.dx, spacing, nbdt, ncol);
      cy = table_column(p.dy, spacing, nbdt, ncol);
      cz = table_column(p.dz, spacing, nbdt, ncol);
    }
    ft_load_cols(ovgr, cy, p.oy, p.gy);
    ft_load_cols(ovgr, cx, p.ox, p.gx);
    ft_load_cols(ovgr, cz, p.oz, p.gz);
  };

  // the A rows of particle p: its y tables split into head and tail (Yo
  // from the overlap table, Yg from the gradient table)
  auto store_a = [&](const FtPart& p) {
    if (p.valid) {
      ft_store_a(ftsm, tid, p.oy);
      ft_store_a(ftsm + kFtA, tid, p.gy);
    }
  };

  auto issue = [&](int buf) {
    fence_after();
    const unsigned ao = sbase, ag = ao + kFtA;
    const unsigned bb = sbase + 2u * kFtA;
    // the K steps holding the small terms first
#pragma unroll
    for (int q = 3; q >= 0; --q) {
      const uint64_t bd = tc::smem_desc(bb + 256u * q, 128u, 1024u);
      mma_ss_tf32(tmem, tc::smem_desc(ao + 256u * q, 128u, 1024u), bd, idesc, q != 3 ? 1u : 0u);
      mma_ss_tf32(tmem + kFtColG, tc::smem_desc(ag + 256u * q, 128u, 1024u), bd, idesc, q != 3 ? 1u : 0u);
    }
    commit(smem_u32(&bars[buf]));
  };

  const int G = gridDim.x;
  auto item_at = [&](int t) { return (int)blockIdx.x + t * G; };
  auto load_item = [&](int item) { return ft_load_item(item, nitems, items); };
  auto resolve = [&](int item) { return ft_derive(load_item(item), n); };

  // items t (cur), t+1 (nxt, delta in dn), t+2 (after); item_cell of t+3
  FtItem cur = resolve(item_at(0));
  FtItem nxt = resolve(item_at(1));
  FtItem after = resolve(item_at(2));
  float dc[4] = {0.f, 0.f, 0.f, 0.f}, dn[4] = {0.f, 0.f, 0.f, 0.f};
  load_delta(cur, dc);
  load_delta(nxt, dn);
  int staged = -1;                 // cell code of the stencil in B
  unsigned phase = 0;              // bit b: parity of the next completion of bars[b]
  bool ok = true;                  // the same in every thread after each barrier
  unsigned pending = 0;            // bit b: a commit on bars[b] not yet seen complete

  unsigned sphase = 0;             // parity of the next completion of the stencil barrier
  bool staging = false;            // stencil copies issued and not yet seen complete
  FtPart pc;
  load_part(cur, dc, pc);
  if (cur.has) {
    ft_stage_b(cur, tid, &csol_map, raw, sbar);
    staging = true;
    store_a(pc);
    ok = __all_sync(0xffffffffu, mbar_wait(sbar, sphase));
    if (ok) {
      staging = false;
      sphase ^= 1u;
      if (tid < 100) {
        float c[10];
        ft_read_b(cur, tid, raw, c);
        ft_store_b(ftsm + 2u * kFtA, tid, c);
      }
    }
    staged = cur.code;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  fence_before();
  ok = __syncthreads_and(ok) != 0;
  if (tid == 0 && cur.has && ok) issue(0);
  if (cur.has && ok) pending |= 1u;

  int b = 0;
  for (int t = 0; cur.item >= 0; ++t) {
    const int nb = b ^ 1;
    // ---- loads: delta of t+2, cell data of t+3, item_cell of t+4, the
    // tables of t+1 and, when needed, its stencil
    float d2[4] = {0.f, 0.f, 0.f, 0.f};
    load_delta(after, d2);
    const FtRaw raw3 = load_item(item_at(t + 3));
    FtPart pn;
    load_part(nxt, dn, pn);
    const bool restage = nxt.has && ok && staged != nxt.code;
    if (restage) {
      ft_stage_b(nxt, tid, &csol_map, raw, sbar);  // the tile is free: read before the last barrier
      staging = true;
    }

    // ---- item t
    bool got = false;
    if (cur.has && ok && ((pending >> b) & 1u)) {
      // the same outcome in the whole warp: the tensor-memory loads of the
      // finish are warp-collective
      got = __all_sync(0xffffffffu, mbar_wait(smem_u32(&bars[b]), (phase >> b) & 1u));
      ok = got;
      if (got) {
        pending &= ~(1u << b);
        phase ^= 1u << b;
      }
    }
    float ax = 0.f, ay = 0.f, az = 0.f, ae = 0.f;
    if (got) {
      fence_after();
      float sx, sy, sz;
      ft_finish(lane_base, pc, sx, sy, sz);
      if (pc.valid) {
        float fx = -wf * sx, fy = -wf * sy, fz = -wf * sz;
        if (P.on) {
          float fx2, fy2, fz2, e;
          proj_term(P, cur.kx, cur.ky, cur.kz, pc.dx, pc.dy, pc.dz, x0, h, fx2, fy2, fz2, e);
          fx -= fx2;
          fy -= fy2;
          fz -= fz2;
          ax = fx2;
          ay = fy2;
          az = fz2;
          ae = e;
        }
        force[pc.s] = fx;
        force[Npad + pc.s] = fy;
        force[2 * Npad + pc.s] = fz;
      }
    }
    ax = warp_sumf(ax);
    ay = warp_sumf(ay);
    az = warp_sumf(az);
    ae = warp_sumf(ae);
    if (lane == 0) {
      red[b][warp][0] = ax;
      red[b][warp][1] = ay;
      red[b][warp][2] = az;
      red[b][warp][3] = ae;
    }

    // ---- item t+1's operands (their last reader, the MMAs of item t, has
    // completed: this warp saw it, or the item had none, or no MMA is issued
    // any more): the stencil, when it changed, and the particles' A rows
    if (restage) {
      const bool sok = __all_sync(0xffffffffu, mbar_wait(sbar, sphase));
      if (sok) {
        staging = false;
        sphase ^= 1u;
        if (ok && tid < 100) {
          float cb[10];
          ft_read_b(nxt, tid, raw, cb);
          ft_store_b(ftsm + 2u * kFtA, tid, cb);
        }
      }
      ok = ok && sok;
      staged = nxt.code;
    }
    if (ok) store_a(pn);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before();
    ok = __syncthreads_and(ok) != 0;  // after a wait that gave up, no more MMAs
    if (nxt.has && ok) {
      if (tid == 0) issue(nb);
      pending |= 1u << nb;
    }
    if (tid < 4)
      red_items[4 * (size_t)cur.item + tid] = ((red[b][0][tid] + red[b][1][tid]) + red[b][2][tid]) + red[b][3][tid];
    cur = nxt;
    nxt = after;
    after = ft_derive(raw3, n);
    pc = pn;
#pragma unroll
    for (int k = 0; k < 4; ++k) dn[k] = d2[k];
    b = nb;
  }

  if (!ok && tid == 0) atomicOr(&dsc->status, kStatusMmaTimeout);
  // nothing may still be in flight when the tensor memory is freed (after a
  // wait that gave up, at most one commit per barrier is outstanding)
  for (int bb = 0; bb < 2; ++bb)
    if (pending & (1u << bb)) mbar_wait(smem_u32(&bars[bb]), (phase >> bb) & 1u);
  if (staging) mbar_wait(sbar, sphase);  // no stencil copy may still be writing the tile
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kFtCols) : "memory");
  }
}

// The fine coefficients into rows of `pitch` floats (n even or odd; pitch a
// multiple of four, the padding zero): float2 pairs when n is even, so that
// both sides' rows start on 8-byte boundaries.
__global__ void k_pad_rows(const float* __restrict__ src, int n, float* __restrict__ dst, int pitch, int rows) {
  const int per = pitch / 2;
  const int64_t tot = (int64_t)rows * per;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / per;
    const int x = 2 * (int)(t - r * per);
    const float* s = src + r * n;
    float2 v = make_float2(0.f, 0.f);
    if ((n & 1) == 0) {
      if (x < n) v = *reinterpret_cast<const float2*>(s + x);
    } else {
      if (x < n) v.x = s[x];
      if (x + 1 < n) v.y = s[x + 1];
    }
    *reinterpret_cast<float2*>(dst + r * pitch + x) = v;
  }
}

// ------------------------------------------------------------------ tail
__device__ __forceinline__ void basis_vd(const double* g, int nk, int lin, double x, double& v, double& dv) {
  const int knot = (lin - 1) / 2 + 1, kind = (lin - 1) & 1;
  double a, h, s;
  if (knot > 1 && x <= g[knot - 1]) {
    if (x < g[knot - 2]) { v = 0; dv = 0; return; }
    h = g[knot - 1] - g[knot - 2]; a = (x - g[knot - 2]) / h; s = -1.0;
  } else if (knot < nk && x >= g[knot - 1]) {
    if (x > g[knot]) { v = 0; dv = 0; return; }
    h = g[knot] - g[knot - 1]; a = (g[knot] - x) / h; s = 1.0;
  } else {
    v = 0; dv = 0; return;
  }
  if (kind == 0) {
    v = 3 * (a * a) - 2 * (a * a * a);
    dv = -6 * (a - a * a) * s / h;
  } else {
    v = h * (a * a - a * a * a) * s;
    dv = -2 * a + 3 * (a * a);
  }
}

__device__ __forceinline__ int cell_index_d(const double* g, int nk, double x) {
  if (x < g[0] || x > g[nk - 1]) return 0;
  int lo = 0, hi = nk;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (g[mid] < x) lo = mid + 1; else hi = mid;
  }
  return max(1, lo);
}

__global__ void __launch_bounds__(kGThreads) k_tail(const int32_t* __restrict__ outlist, DeviceScalars* dsc,
                                                    int64_t Npad, const int32_t* __restrict__ k,
                                                    const float* __restrict__ d, const float* __restrict__ csolc,
                                                    const double* __restrict__ kc, int nkc, int nc, int nk,
                                                    float x0f, float hf, double x0, double h, double w,
                                                    float* __restrict__ force, double* __restrict__ red_tail) {
  const int cnt = dsc->outcount;
  const ProjF P = load_proj(dsc, w);
  const double Px = dsc->proj_pos[0], Py = dsc->proj_pos[1], Pz = dsc->proj_pos[2];
  const double q = dsc->proj_charge, R = dsc->proj_ball;
  float ax = 0.f, ay = 0.f, az = 0.f, ae = 0.f;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
    const int s = outlist[t];
    const int kxp = k[s], kyp = k[Npad + s], kzp = k[2 * Npad + s];
    const float dx0 = d[s], dy0 = d[Npad + s], dz0 = d[2 * Npad + s];
    double fx = 0, fy = 0, fz = 0;
    const double px = x0 + (double)(kxp - 1) * h + (double)dx0;
    const double py = x0 + (double)(kyp - 1) * h + (double)dy0;
    const double pz = x0 + (double)(kzp - 1) * h + (double)dz0;
    const int cx = cell_index_d(kc, nkc, px), cy = cell_index_d(kc, nkc, py), cz = cell_index_d(kc, nkc, pz);
    if (cx && cy && cz) {
      double vx[4], vy[4], vz[4], gx[4], gy[4], gz[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        basis_vd(kc, nkc, 2 * (cx - 1) + a + 1, px, vx[a], gx[a]);
        basis_vd(kc, nkc, 2 * (cy - 1) + a + 1, py, vy[a], gy[a]);
        basis_vd(kc, nkc, 2 * (cz - 1) + a + 1, pz, vz[a], gz[a]);
      }
      double ex = 0, ey = 0, ez = 0;
      for (int ak = 0; ak < 4; ++ak)
        for (int aj = 0; aj < 4; ++aj) {
          const float* row =
              csolc + (size_t)2 * (cx - 1) + (size_t)nc * ((2 * (cy - 1) + aj) + (size_t)nc * (2 * (cz - 1) + ak));
#pragma unroll
          for (int ai = 0; ai < 4; ++ai) {
            const double c = row[ai];
            ex -= c * gx[ai] * vy[aj] * vz[ak];
            ey -= c * vx[ai] * gy[aj] * vz[ak];
            ez -= c * vx[ai] * vy[aj] * gz[ak];
          }
        }
      fx = w * ex;
      fy = w * ey;
      fz = w * ez;
    }
    if (P.on) {
      const double dx = Px - px, dy = Py - py, dz = Pz - pz;
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double kern = r2 > R * R ? 1.0 / (r2 * sqrt(r2)) : 1.0 / (R * R * R);
      const double m = -w * q * kern;
      fx -= m * dx;
      fy -= m * dy;
      fz -= m * dz;
      if (P.ball) {
        // the CPU path: the same ball reaction on the projectile
        const double r = sqrt(r2);
        ax += (float)(m * dx);
        ay += (float)(m * dy);
        az += (float)(m * dz);
        ae += (float)(r < R ? -(3.0 - (r / R) * (r / R)) / (2.0 * R) : -1.0 / r);
      } else {
        // the device path: the Gaussian reaction on the projectile, at the
        // clamped cell's position
        const uint32_t cell = cell_key(kxp, kyp, kzp, nk);
        int kx, ky, kz;
        cell_knots(cell, nk, kx, ky, kz);
        float fx2, fy2, fz2, e;
        proj_term(P, kx, ky, kz, dx0, dy0, dz0, x0f, hf, fx2, fy2, fz2, e);
        ax += fx2;
        ay += fy2;
        az += fz2;
        ae += e;
      }
    }
    force[s] = (float)fx;
    force[Npad + s] = (float)fy;
    force[2 * Npad + s] = (float)fz;
  }
  block_red(ax, ay, az, ae, red_tail + 4 * blockIdx.x);
}

// ---------------------------------------------------------------- energy
// The interaction energy sum_p w phi(p) of interaction_energy
// (src/energy.jl:19-43) with phi the potential of the coefficients `csolf`
// (fine) and `csolc` (coarse): inside the host margin knots[3] < p <
// knots[end-2] (every axis) the smoothed potential of smoothed_potential
// (src/fields.jl:405-429, the 10^3 overlap-weighted sum at the nearest
// knots), else the coarse spline's value, else 0 (the reference's call
// passes no enclosed charge).
//
// One warp per work item of the last sort.  Between that sort and this
// call the cloud may have moved (the energy of the total potential is taken
// after the push), so the warp stages the 14^3 coefficients around its cell:
// the stencils of the cell and of its neighbours one knot away.  A particle
// further away, or inside the margin from a cell whose stencil does not fit
// the grid, reads its stencil from global memory.  Positions are rebuilt in
// float64 as the host does; the 10^3 sum is FP32, the sums over particles
// float64, one per work item, reduced in a fixed order.
constexpr int kEW = 14;   // tile rows (y) and planes (z): the stencils of the cell and its neighbours
constexpr int kEX = 16;   // tile row pitch (x): the cell's own stencil rows start 16-byte aligned
constexpr int kEThreads = 128;
constexpr int kEClaim = 8;     // work items a warp claims at once

// sum_{ii,jj,kk} c[ii + sy jj + sz kk] ox[ii] oy[jj] oz[kk] (c 8-byte aligned,
// sy and sz even): y first into five packed accumulators per plane, then x,
// then z, as the gather contracts.
// A column's overlap row from the interleaved table (its first ten floats of
// the 80-byte row): two 16-byte loads and one 8-byte load.
__device__ __forceinline__ void load_ov10(const float4* __restrict__ ovgr, int col, float (&v)[10]) {
  const float4* p = ovgr + (size_t)(col - 1) * 5;
  const float4 a = __ldg(p), b = __ldg(p + 1);
  const float2 c = __ldg(reinterpret_cast<const float2*>(p + 2));
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  v[8] = c.x; v[9] = c.y;
}

// The same sum from rows that start on 16-byte boundaries (row pitch sy and
// plane pitch sz multiples of four): two 16-byte and one 8-byte load a row.
__device__ __forceinline__ float smoothed_sum_a16(const float* __restrict__ c, int sy, int sz, const float (&ox)[10],
                                                  const float (&oy)[10], const float (&oz)[10]) {
  float2 ox2[5];
#pragma unroll
  for (int a = 0; a < 5; ++a) ox2[a] = make_float2(ox[2 * a], ox[2 * a + 1]);
  float phi = 0.f;
#pragma unroll 2
  for (int kk = 0; kk < 10; ++kk) {
    float2 y2[5];
#pragma unroll
    for (int a = 0; a < 5; ++a) y2[a] = make_float2(0.f, 0.f);
#pragma unroll
    for (int jj = 0; jj < 10; ++jj) {
      const float* row = c + jj * sy + kk * sz;
      const float4 c0 = *reinterpret_cast<const float4*>(row);
      const float4 c1 = *reinterpret_cast<const float4*>(row + 4);
      const float2 c2 = *reinterpret_cast<const float2*>(row + 8);
      const float2 cp[5] = {make_float2(c0.x, c0.y), make_float2(c0.z, c0.w), make_float2(c1.x, c1.y),
                            make_float2(c1.z, c1.w), c2};
      const float2 w = make_float2(oy[jj], oy[jj]);
#pragma unroll
      for (int a = 0; a < 5; ++a) y2[a] = __ffma2_rn(cp[a], w, y2[a]);
    }
    float2 t = make_float2(0.f, 0.f);
#pragma unroll
    for (int a = 0; a < 5; ++a) t = __ffma2_rn(ox2[a], y2[a], t);
    phi = fmaf(oz[kk], t.x + t.y, phi);
  }
  return phi;
}

__device__ __forceinline__ float smoothed_sum(const float* __restrict__ c, int sy, int sz, const float (&ox)[10],
                                              const float (&oy)[10], const float (&oz)[10]) {
  float2 ox2[5];
#pragma unroll
  for (int a = 0; a < 5; ++a) ox2[a] = make_float2(ox[2 * a], ox[2 * a + 1]);
  float phi = 0.f;
#pragma unroll 2
  for (int kk = 0; kk < 10; ++kk) {
    float2 y2[5];
#pragma unroll
    for (int a = 0; a < 5; ++a) y2[a] = make_float2(0.f, 0.f);
#pragma unroll
    for (int jj = 0; jj < 10; ++jj) {
      const float2* row = reinterpret_cast<const float2*>(c + jj * sy + kk * sz);
      const float2 w = make_float2(oy[jj], oy[jj]);
#pragma unroll
      for (int a = 0; a < 5; ++a) y2[a] = __ffma2_rn(row[a], w, y2[a]);
    }
    float2 t = make_float2(0.f, 0.f);
#pragma unroll
    for (int a = 0; a < 5; ++a) t = __ffma2_rn(ox2[a], y2[a], t);
    phi = fmaf(oz[kk], t.x + t.y, phi);
  }
  return phi;
}

__global__ void __launch_bounds__(kEThreads) k_energy(
    const int32_t* __restrict__ occupied, const int32_t* __restrict__ bounds,
    const int32_t* __restrict__ chunk_start, const int32_t* __restrict__ item_cell, DeviceScalars* dsc, int64_t Npad,
    const int32_t* __restrict__ k, const float* __restrict__ d, const float* __restrict__ csolf, int n, int nk,
    const float4* __restrict__ ovgr, int nbdt, int ncol, float spacing, double x0, double h, double lo, double hi,
    const float* __restrict__ csolc, const double* __restrict__ kc, int nkc, int nc, double w, int chunk,
    double* __restrict__ e_items) {
  extern __shared__ __align__(16) float etile[];  // [kEW][kEW][kEX]: the CTA's tile
  __shared__ int s_item;
  __shared__ double s_e[2][kEThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float* tile = etile;
  const int nitems = dsc->nitems;
  int cached = -1;
  // The CTA claims runs of kEClaim consecutive work items (a cell's items,
  // about eight at the headline size, share one staging of its tile) and
  // takes them one at a time, a particle a thread.
  for (;;) {
    if (tid == 0) s_item = (int)atomicAdd(&dsc->work_energy, (unsigned long long)kEClaim);
    __syncthreads();
    const int i0 = s_item;
    __syncthreads();  // every thread has the run before the next claim
    if (i0 >= nitems) break;
    const int i1 = min(i0 + kEClaim, nitems);
    for (int item = i0; item < i1; ++item) {
      const int g = item_cell[item];
      int kx, ky, kz;
      cell_knots((uint32_t)occupied[g], nk, kx, ky, kz);
      // 0-based corner of the block: the cell's stencil corner 2k - 6, less
      // four along x (the cell's own rows start 16-byte aligned) and two along
      // y and z; a particle of a neighbouring cell has its stencil inside it
      const int cx0 = 2 * kx - 10, cy0 = 2 * ky - 8, cz0 = 2 * kz - 8;
      if (g != cached) {
        __syncthreads();  // the previous item's threads are done with the tile
        for (int e = tid; e < kEW * kEW * kEX; e += kEThreads) {
          const int i = cx0 + e % kEX, j = cy0 + (e / kEX) % kEW, kk = cz0 + e / (kEX * kEW);
          tile[e] = (i >= 0 && j >= 0 && kk >= 0 && i < n && j < n && kk < n)
                        ? csolf[(size_t)i + (size_t)n * (j + (size_t)n * kk)]
                        : 0.f;
        }
        cached = g;
        __syncthreads();
      }
      const int s0 = bounds[g] + (item - chunk_start[g]) * chunk;
      const int s1 = min(s0 + chunk, bounds[g + 1]);
      double e = 0.0;
      for (int s = s0 + tid; s < s1; s += kEThreads) {
        const int kp[3] = {k[s], k[Npad + s], k[2 * Npad + s]};
        const float dp[3] = {d[s], d[Npad + s], d[2 * Npad + s]};
        double p[3];
        bool inside = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          p[a] = x0 + (double)(kp[a] - 1) * h + (double)dp[a];
          inside = inside && lo < p[a] && p[a] < hi;
        }
        double phi = 0.0;
        if (inside) {
          float ox[10], oy[10], oz[10];
          load_ov10(ovgr, table_column(dp[0], spacing, nbdt, ncol), ox);
          load_ov10(ovgr, table_column(dp[1], spacing, nbdt, ncol), oy);
          load_ov10(ovgr, table_column(dp[2], spacing, nbdt, ncol), oz);
          // stencil corner of the particle's own nearest knots, in the block
          const int bx = 2 * kp[0] - 6 - cx0, by = 2 * kp[1] - 6 - cy0, bz = 2 * kp[2] - 6 - cz0;
          // a particle still in the item's cell: rows 16-byte aligned, the
          // same rows as its warp's other such particles (broadcast loads); one
          // in a neighbouring cell: 8-byte loads at its offset (a second copy of
          // the tile shifted by two floats, so that those rows align too, was
          // measured slower: their lanes' scattered rows conflict in the banks)
          if (bx == 4 && by == 2 && bz == 2)
            phi = smoothed_sum_a16(tile + 4 + kEX * (2 + kEW * 2), kEX, kEX * kEW, ox, oy, oz);
          else if (bx >= 0 && by >= 0 && bz >= 0 && bx <= kEX - 10 && by <= kEW - 10 && bz <= kEW - 10)
            phi = smoothed_sum(tile + bx + kEX * (by + kEW * bz), kEX, kEX * kEW, ox, oy, oz);
          else
            phi = smoothed_sum(csolf + (size_t)(2 * kp[0] - 6) + (size_t)n * ((2 * kp[1] - 6) + (size_t)n * (2 * kp[2] - 6)),
                               n, n * n, ox, oy, oz);
        } else {
          const int ix = cell_index_d(kc, nkc, p[0]), iy = cell_index_d(kc, nkc, p[1]), iz = cell_index_d(kc, nkc, p[2]);
          if (ix && iy && iz) {
            double vx[4], vy[4], vz[4], dd;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
              basis_vd(kc, nkc, 2 * (ix - 1) + a + 1, p[0], vx[a], dd);
              basis_vd(kc, nkc, 2 * (iy - 1) + a + 1, p[1], vy[a], dd);
              basis_vd(kc, nkc, 2 * (iz - 1) + a + 1, p[2], vz[a], dd);
            }
            for (int ak = 0; ak < 4; ++ak)
              for (int aj = 0; aj < 4; ++aj) {
                const float* row =
                    csolc + (size_t)2 * (ix - 1) + (size_t)nc * ((2 * (iy - 1) + aj) + (size_t)nc * (2 * (iz - 1) + ak));
                const double wyz = vy[aj] * vz[ak];
#pragma unroll
                for (int ai = 0; ai < 4; ++ai) phi += (double)row[ai] * vx[ai] * wyz;
              }
          }
        }
        e += w * phi;
      }
      // the item's sum: each warp's butterfly, then the warps in order (the
      // partials alternate between two slots, so one barrier a item suffices)
      e = warp_sum(e);
      if (lane == 0) s_e[item & 1][warp] = e;
      __syncthreads();
      if (tid == 0) {
        double t = 0.0;
#pragma unroll
        for (int q = 0; q < kEThreads / 32; ++q) t += s_e[item & 1][q];
        e_items[item] = t;
      }
    }
  }
}

// Two levels of an order-fixed sum of one component: block b sums its
// contiguous share of the items, then one block the block sums.
__device__ __forceinline__ double block_sum1(const double* __restrict__ p, int begin, int end) {
  __shared__ double sh[256];
  const int t = threadIdx.x;
  double s = 0;
  for (int i = begin + t; i < end; i += blockDim.x) s += p[i];
  sh[t] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (t < o) sh[t] += sh[t + o];
    __syncthreads();
  }
  return sh[0];
}

__global__ void __launch_bounds__(256) k_energy_blocks(const double* __restrict__ items, const DeviceScalars* dsc,
                                                       double* __restrict__ block_out) {
  const int nitems = dsc->nitems;
  const int per = (nitems + gridDim.x - 1) / gridDim.x;
  const int b0 = min(nitems, (int)blockIdx.x * per), b1 = min(nitems, b0 + per);
  const double r = block_sum1(items, b0, b1);
  if (threadIdx.x == 0) block_out[blockIdx.x] = r;
}

__global__ void __launch_bounds__(256) k_energy_total(const double* __restrict__ blocks, int nblocks, double* out) {
  const double r = block_sum1(blocks, 0, nblocks);
  if (threadIdx.x == 0) *out = r;
}

}  // namespace

// The row-padded copy of the fine coefficients and the tensor map over it:
// dims (pitch, n, n) floats, x fastest; strides pitch * 4 and pitch * n * 4
// bytes (multiples of 16); box 20 x 10 x 10; no swizzle, zero fill.
size_t energy_smem() { return (size_t)kEW * kEW * kEX * sizeof(float); }

void field_setup(Ctx& c) {
  VLB_CUDA(cudaFuncSetAttribute(k_field_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFtSmem));
  VLB_CUDA(cudaFuncSetAttribute(k_energy, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)energy_smem()));
  // two CTAs of 55 KB need the 132 KB shared-memory split (58 % of 228 KB);
  // the remaining 124 KB of the SM's L1 holds the 80 KB interleaved tables
  VLB_CUDA(cudaFuncSetAttribute(k_field_tc, cudaFuncAttributePreferredSharedMemoryCarveout, 58));
  const int n = c.fine.n;
  c.csol_pitch = (n + 3) & ~3;
  const size_t rows = (size_t)c.csol_pitch * n * n;
  VLB_CUDA(cudaMalloc(&c.csol_rows, rows * sizeof(float)));
  VLB_CUDA(cudaMemset(c.csol_rows, 0, rows * sizeof(float)));
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q{};
  VLB_CUDA(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q));
  if (!fn || q != cudaDriverEntryPointSuccess) throw CudaError(cudaErrorNotSupported, __FILE__, __LINE__);
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  const cuuint64_t dims[3] = {(cuuint64_t)c.csol_pitch, (cuuint64_t)n, (cuuint64_t)n};
  const cuuint64_t strides[2] = {(cuuint64_t)c.csol_pitch * 4, (cuuint64_t)c.csol_pitch * n * 4};
  const cuuint32_t box[3] = {(cuuint32_t)kFtBoxX, 10, 10};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = reinterpret_cast<Encode>(fn)(&c.csol_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, c.csol_rows, dims,
                                                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError(cudaErrorInvalidValue, __FILE__, __LINE__);
}

void launch_forces(Ctx& c) {
  Level& F = c.fine;
  Level& C = c.coarse;
  Particles& P = c.part[c.cur];
  if (c.profile) VLB_CUDA(cudaEventRecord(c.ev[kEvGatherBegin], c.stream));
  if (c.field_tc && c.chunk <= kFtRows) {
    const int rows = F.n * F.n, per = c.csol_pitch / 2;
    k_pad_rows<<<grid_for(c, (int64_t)rows * per, 256, 8), 256, 0, c.stream>>>(F.csol, F.n, c.csol_rows,
                                                                               c.csol_pitch, rows);
    VLB_LAUNCHED(c);
    k_field_tc<<<2 * c.num_sms, kFtThreads, kFtSmem, c.stream>>>(
        c.item_rec, c.dsc, c.Npad, P.d, c.csol_map, F.n, F.nk,
        reinterpret_cast<const float4*>(c.ovgr), c.nbdt, c.ncol, c.spacing_f, c.x0f, c.hf, c.weight, c.force,
        c.chunk, c.red_items, c.cols_packed ? c.cols : nullptr);
  } else {
    VLB_CUDA(cudaMemsetAsync(&c.dsc->work_gather, 0, sizeof(unsigned long long), c.stream));
    k_field<<<c.num_sms * c.field_cps, kGThreads, 0, c.stream>>>(c.occupied, c.bounds, c.chunk_start, c.item_cell,
                                                                 c.dsc, c.Npad, P.d, F.csol, F.n, F.nk, c.overlap,
                                                                 c.gradient, c.nbdt, c.ncol, c.spacing_f, c.x0f,
                                                                 c.hf, c.weight, c.force, c.chunk, c.red_items);
  }
  VLB_LAUNCHED(c);
  if (c.profile) VLB_CUDA(cudaEventRecord(c.ev[kEvGatherEnd], c.stream));
  k_tail<<<c.num_sms, kGThreads, 0, c.stream>>>(c.outlist, c.dsc, c.Npad, P.k, P.d, C.csol, C.knots_d, C.nk,
                                                    C.n, F.nk, c.x0f, c.hf, c.x0, c.h, c.weight, c.force,
                                                    c.red_tail);
  VLB_LAUNCHED(c);
  k_red_blocks<<<c.num_sms, 256, 0, c.stream>>>(c.red_items, c.dsc, c.red_blocks);
  VLB_LAUNCHED(c);
  k_red_total<<<1, 256, 0, c.stream>>>(c.red_blocks, c.num_sms, c.red_tail, c.num_sms, c.dsc);
  VLB_LAUNCHED(c);
  c.have_forces = true;
}

// The interaction energy of the coefficients (csolf, csolc) over the cloud
// as it is, into *out; the work items of the last sort.
void launch_energy(Ctx& c, const float* csolf, const float* csolc, double* out) {
  Level& F = c.fine;
  Level& C = c.coarse;
  Particles& P = c.part[c.cur];
  VLB_CUDA(cudaMemsetAsync(&c.dsc->work_energy, 0, sizeof(unsigned long long), c.stream));
  k_energy<<<c.num_sms * 6, kEThreads, energy_smem(), c.stream>>>(
      c.occupied, c.bounds, c.chunk_start, c.item_cell, c.dsc, c.Npad, P.k, P.d, csolf, F.n, F.nk,
      reinterpret_cast<const float4*>(c.ovgr), c.nbdt,
      c.ncol, c.spacing_f, c.x0, c.h, F.h_knots[2], F.h_knots[F.nk - 3], csolc, C.knots_d, C.nk, C.n, c.weight,
      c.chunk, c.e_items);
  VLB_LAUNCHED(c);
  k_energy_blocks<<<c.num_sms, 256, 0, c.stream>>>(c.e_items, c.dsc, c.e_blocks);
  VLB_LAUNCHED(c);
  k_energy_total<<<1, 256, 0, c.stream>>>(c.e_blocks, c.num_sms, out);
  VLB_LAUNCHED(c);
}

}  // namespace vlb
