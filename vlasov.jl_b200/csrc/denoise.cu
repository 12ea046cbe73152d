// The learned denoiser of the fine density: training and inference kernels.
//
// The network (fixed shape): four 3^3 convolutions, 1 -> 16 -> 16 -> 16 -> 3
// channels, ReLU after the first three, no biases, zero padding at the
// grid's faces.  The three output channels are a charge flux F = f(s rho)
// (s a fixed input scale), and the output is its divergence added to the
// input:
//
//     out[v] = rho[v] + (1/s) sum_axes (F^a[v] - F^a[v - e_a]),
//
// F~a the flux with no flow through the grid's faces (zero on the last
// plane of its axis and before the first), F^ that flux limited so that no
// voxel gives more charge than it holds (k_flux_limit).  The correction
// moves charge between neighbouring voxels and adds none: the sum of out
// equals the sum of rho, and out >= min(rho, 0) (the exchange-correlation
// potential of the step needs rho > -1.6e-4; the network can make no new
// negative density).  Without biases f(0) = 0 and f is positively homogeneous, so empty
// space stays empty and the correction scales with the density.  Weights are
// BF16 (kept as float32 values that BF16 represents exactly), every product
// and sum is float32.
//
// Activations are channel-last float32 ([z][y][x][c], i fastest as the
// grids).  The volume is cut into 8^3 tiles.  A tile is flagged when its
// largest |rho| exceeds kTileThreshold times the volume's; the active tiles
// are the flagged ones and their neighbours, and the network is defined on
// them: every layer's activations (its input included) are zero outside the
// active tiles.  With the threshold at zero this is exact (the network's
// reach, four voxels, is less than a tile); above it, the faint density of a
// few escaped electrons (a pseudo-particle deposits ~1e-8 against a peak of
// ~4e-3) passes through unchanged instead of filling the grid with tiles.
//
//   k_conv16_tc           the 16 -> 16 layers (and their input-gradient
//                         passes) on the tensor cores: implicit GEMM, BF16
//                         weights and BF16 head + tail activations, FP32
//                         accumulation in tensor memory
//   k_conv<CIN, COUT>     the other layers on the CUDA cores (also the
//                         input-gradient pass, with the weights flipped and
//                         transposed), 256 threads per tile, two voxels per
//                         thread sharing the weight reads
//   k_conv_wgrad<..>      weight gradient, per-CTA partial sums over tiles,
//                         reduced in a fixed order by k_reduce_partials
//   k_flux_limit          the positivity limiter of the flux
//   k_divergence          out = rho + div F^ / s (F^ the limited flux)
//   k_loss, k_limit_tsum, mean squared error against the target and its
//   k_div_adjoint         gradient at the flux, through the limiter
//   k_adam                Adam update of the float32 master weights
//
// The same kernels serve the training loop (vlb_dn_*) and the in-step
// inference (vlb_set_denoiser + vlb_step_params.denoise).

#include <cstring>
#include <vector>

#include "tc_util.cuh"
#include "vlb_internal.cuh"

namespace vlb {

namespace {

constexpr int kT = 8;                  // tile edge (voxels)
constexpr int kH = kT + 2;             // halo edge
constexpr int kConvThreads = 256;      // two voxels per thread
constexpr int kLayers = 4;
constexpr int kLayerIn[kLayers] = {1, 16, 16, 16};
constexpr int kLayerOut[kLayers] = {16, 16, 16, 3};
constexpr float kTileThreshold = 1e-3f;   // of the volume's largest |rho|

__host__ __device__ constexpr int pad_stride(int c) { return c == 16 ? 20 : c; }  // float stride per halo voxel

struct Vol {
  int nx, ny, nz;
  int tx, ty, tz;  // tiles per axis
};

__device__ __forceinline__ void tile_origin(const Vol& v, int tile, int& x0, int& y0, int& z0) {
  x0 = (tile % v.tx) * kT;
  y0 = ((tile / v.tx) % v.ty) * kT;
  z0 = (tile / (v.tx * v.ty)) * kT;
}

// ---------------------------------------------------------------- tiles
// tmax[t] = the largest |x| in tile t.
__global__ void k_tile_max(const float* __restrict__ x, Vol v, float* __restrict__ tmax) {
  __shared__ float sh[256];
  const int tile = blockIdx.x;
  int x0, y0, z0;
  tile_origin(v, tile, x0, y0, z0);
  float m = 0.f;
  for (int e = threadIdx.x; e < kT * kT * kT; e += blockDim.x) {
    const int i = x0 + e % kT, j = y0 + (e / kT) % kT, k = z0 + e / (kT * kT);
    if (i < v.nx && j < v.ny && k < v.nz) m = fmaxf(m, fabsf(x[(size_t)i + (size_t)v.nx * (j + (size_t)v.ny * k)]));
  }
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = fmaxf(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) tmax[tile] = sh[0];
}

// gmax = the largest tmax (one block).
__global__ void k_volume_max(const float* __restrict__ tmax, int ntiles, float* __restrict__ gmax) {
  __shared__ float sh[1024];
  float m = 0.f;
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x) m = fmaxf(m, tmax[t]);
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = fmaxf(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *gmax = sh[0];
}

// Active tiles: a flagged tile (tmax > kTileThreshold gmax, and > 0) or a
// neighbour of one; amap[t] = 1 for them, compacted into `list`.
__global__ void k_tile_active(const float* __restrict__ tmax, const float* __restrict__ gmax, Vol v,
                              int32_t* __restrict__ amap, int32_t* __restrict__ list, int32_t* __restrict__ count) {
  const int ntiles = v.tx * v.ty * v.tz;
  const float tau = kTileThreshold * *gmax;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
    const int a = t % v.tx, b = (t / v.tx) % v.ty, c = t / (v.tx * v.ty);
    int on = 0;
    for (int dc = -1; dc <= 1 && !on; ++dc)
      for (int db = -1; db <= 1 && !on; ++db)
        for (int da = -1; da <= 1 && !on; ++da) {
          const int aa = a + da, bb = b + db, cc = c + dc;
          if (aa < 0 || bb < 0 || cc < 0 || aa >= v.tx || bb >= v.ty || cc >= v.tz) continue;
          const float m = tmax[aa + v.tx * (bb + v.ty * cc)];
          on = m > tau && m > 0.f;
        }
    amap[t] = on;
    if (on) list[atomicAdd(count, 1)] = t;
  }
}

// The active neighbours of each active tile as a 27-bit mask: bit d set when
// the tile next to it in direction d (d = dx + 3 dy + 9 dz, each in 0..2 for
// -1..+1) is inside and active.  The conv kernels read one word per tile.
__global__ void k_tile_nbmask(const int32_t* __restrict__ amap, const int32_t* __restrict__ list,
                              const int32_t* __restrict__ count, Vol v, uint32_t* __restrict__ nbmask) {
  const int n = *count;
  for (int li = blockIdx.x * blockDim.x + threadIdx.x; li < n; li += gridDim.x * blockDim.x) {
    const int t = list[li];
    const int a = t % v.tx, b = (t / v.tx) % v.ty, c = t / (v.tx * v.ty);
    uint32_t m = 0;
    for (int d = 0; d < 27; ++d) {
      const int aa = a + d % 3 - 1, bb = b + (d / 3) % 3 - 1, cc = c + d / 9 - 1;
      if (aa >= 0 && bb >= 0 && cc >= 0 && aa < v.tx && bb < v.ty && cc < v.tz && amap[aa + v.tx * (bb + v.ty * cc)])
        m |= 1u << d;
    }
    nbmask[t] = m;
  }
}

// Halo coordinate h (0..kH-1) -> which of the three tiles along the axis.
__device__ __forceinline__ int halo_side(int h) { return h == 0 ? 0 : (h == kH - 1 ? 2 : 1); }

// Voxel (i, j, k) of halo position (xx, yy, zz) inside the volume and in an
// active tile, by the tile's neighbour mask.
__device__ __forceinline__ bool live_m(const Vol& v, uint32_t m, int i, int j, int k, int xx, int yy, int zz) {
  return i >= 0 && j >= 0 && k >= 0 && i < v.nx && j < v.ny && k < v.nz &&
         ((m >> (halo_side(xx) + 3 * halo_side(yy) + 9 * halo_side(zz))) & 1u);
}

// The 10^3 halo of a tile, CIN channels per voxel, into shared memory rows of
// pad_stride(CIN) floats (zero outside the volume and the active tiles),
// times scale_in; 16-byte loads and stores when CIN is a multiple of 4.
template <int CIN>
__device__ __forceinline__ void stage_halo(const float* __restrict__ x, const Vol& v, uint32_t nbm, int x0, int y0,
                                           int z0, float* xs, float scale_in) {
  constexpr int PS = pad_stride(CIN);
  if constexpr (CIN % 4 == 0) {
#pragma unroll 4
    for (int e = threadIdx.x; e < kH * kH * kH * (CIN / 4); e += kConvThreads) {
      const int q = e % (CIN / 4), hv = e / (CIN / 4);
      const int xx = hv % kH, yy = (hv / kH) % kH, zz = hv / (kH * kH);
      const int i = x0 - 1 + xx, j = y0 - 1 + yy, k = z0 - 1 + zz;
      float4 val = make_float4(0.f, 0.f, 0.f, 0.f);
      if (live_m(v, nbm, i, j, k, xx, yy, zz)) {
        val = *reinterpret_cast<const float4*>(x + ((size_t)i + (size_t)v.nx * (j + (size_t)v.ny * k)) * CIN + 4 * q);
        val.x *= scale_in; val.y *= scale_in; val.z *= scale_in; val.w *= scale_in;
      }
      *reinterpret_cast<float4*>(xs + hv * PS + 4 * q) = val;
    }
  } else {
#pragma unroll 4
    for (int e = threadIdx.x; e < kH * kH * kH * CIN; e += kConvThreads) {
      const int ci = e % CIN, hv = e / CIN;
      const int xx = hv % kH, yy = (hv / kH) % kH, zz = hv / (kH * kH);
      const int i = x0 - 1 + xx, j = y0 - 1 + yy, k = z0 - 1 + zz;
      float val = 0.f;
      if (live_m(v, nbm, i, j, k, xx, yy, zz))
        val = x[((size_t)i + (size_t)v.nx * (j + (size_t)v.ny * k)) * CIN + ci] * scale_in;
      xs[hv * PS + ci] = val;
    }
  }
}

// -------------------------------------------------------------- the conv
// y[v][co] = sum_tap sum_ci w[tap][ci][co] * scale_in * x[v + tap - 1][ci]
// (zero outside the volume and outside the active tiles), then
// y = max(y, 0) when `relu`, and y = 0 where mask[v][co] <= 0 when `mask` is
// given (the input-gradient pass through a ReLU).  Only the tiles in `list`
// are written; the others are never read.
template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) k_conv(const float* __restrict__ x, const float* __restrict__ w,
                                                       float* __restrict__ y, Vol v, const int32_t* __restrict__ list,
                                                       const int32_t* __restrict__ count,
                                                       const uint32_t* __restrict__ nbmask, int relu,
                                                       const float* __restrict__ mask, float scale_in) {
  constexpr int PS = pad_stride(CIN);
  extern __shared__ __align__(16) float sm[];
  float* ws = sm;                                   // [27][CIN][COUT]
  float* xs = sm + 27 * CIN * COUT;                 // [kH^3][PS]
  for (int e = threadIdx.x; e < 27 * CIN * COUT; e += kConvThreads) ws[e] = w[e];
  const int n = *count;
  for (int li = blockIdx.x; li < n; li += gridDim.x) {
    int x0, y0, z0;
    tile_origin(v, list[li], x0, y0, z0);
    const uint32_t nbm = nbmask[list[li]];
    __syncthreads();
    stage_halo<CIN>(x, v, nbm, x0, y0, z0, xs, scale_in);
    __syncthreads();
    // thread: voxel (a, b, c) and (a, b, c + 4)
    const int a = threadIdx.x % kT, b = (threadIdx.x / kT) % kT, c = threadIdx.x / (kT * kT);
    float acc0[COUT], acc1[COUT];
#pragma unroll
    for (int co = 0; co < COUT; ++co) { acc0[co] = 0.f; acc1[co] = 0.f; }
    for (int tap = 0; tap < 27; ++tap) {
      const int da = tap % 3, db = (tap / 3) % 3, dc = tap / 9;
      const float* p0 = xs + ((a + da) + kH * ((b + db) + kH * (c + dc))) * PS;
      const float* p1 = p0 + 4 * kH * kH * PS;
      float xv0[CIN], xv1[CIN];
      if constexpr (CIN % 4 == 0) {
#pragma unroll
        for (int q = 0; q < CIN / 4; ++q) {
          const float4 t0 = *reinterpret_cast<const float4*>(p0 + 4 * q);
          const float4 t1 = *reinterpret_cast<const float4*>(p1 + 4 * q);
          xv0[4 * q] = t0.x; xv0[4 * q + 1] = t0.y; xv0[4 * q + 2] = t0.z; xv0[4 * q + 3] = t0.w;
          xv1[4 * q] = t1.x; xv1[4 * q + 1] = t1.y; xv1[4 * q + 2] = t1.z; xv1[4 * q + 3] = t1.w;
        }
      } else {
#pragma unroll
        for (int ci = 0; ci < CIN; ++ci) { xv0[ci] = p0[ci]; xv1[ci] = p1[ci]; }
      }
      const float* wt = ws + tap * CIN * COUT;
#pragma unroll
      for (int ci = 0; ci < CIN; ++ci) {
        if constexpr (COUT % 4 == 0) {
#pragma unroll
          for (int q = 0; q < COUT / 4; ++q) {
            const float4 wv = *reinterpret_cast<const float4*>(wt + ci * COUT + 4 * q);
            acc0[4 * q] = fmaf(xv0[ci], wv.x, acc0[4 * q]);
            acc0[4 * q + 1] = fmaf(xv0[ci], wv.y, acc0[4 * q + 1]);
            acc0[4 * q + 2] = fmaf(xv0[ci], wv.z, acc0[4 * q + 2]);
            acc0[4 * q + 3] = fmaf(xv0[ci], wv.w, acc0[4 * q + 3]);
            acc1[4 * q] = fmaf(xv1[ci], wv.x, acc1[4 * q]);
            acc1[4 * q + 1] = fmaf(xv1[ci], wv.y, acc1[4 * q + 1]);
            acc1[4 * q + 2] = fmaf(xv1[ci], wv.z, acc1[4 * q + 2]);
            acc1[4 * q + 3] = fmaf(xv1[ci], wv.w, acc1[4 * q + 3]);
          }
        } else {
#pragma unroll
          for (int co = 0; co < COUT; ++co) {
            acc0[co] = fmaf(xv0[ci], wt[ci * COUT + co], acc0[co]);
            acc1[co] = fmaf(xv1[ci], wt[ci * COUT + co], acc1[co]);
          }
        }
      }
    }
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int i = x0 + a, j = y0 + b, k = z0 + c + 4 * s;
      if (i >= v.nx || j >= v.ny || k >= v.nz) continue;
      const size_t vox = (size_t)i + (size_t)v.nx * (j + (size_t)v.ny * k);
      float* acc = s ? acc1 : acc0;
#pragma unroll
      for (int co = 0; co < COUT; ++co) {
        float r = acc[co];
        if (relu) r = fmaxf(r, 0.f);
        if (mask && !(mask[vox * COUT + co] > 0.f)) r = 0.f;
        y[vox * COUT + co] = r;
      }
    }
  }
}

// ------------------------------------------- the 16 -> 16 layers, tcgen05
// y[v][co] = sum_tap sum_ci w[tap][ci][co] x[v + tap - 1][ci] as an implicit
// GEMM on the tensor cores: M = 128 voxels (two z planes of the tile), N = 16
// output channels, K = 16 input channels per tap (one kind::f16 MMA), 27
// taps.  The weights are BF16 (exact); each activation is split into a BF16
// head and tail (x - head - tail ~ 2^-17 |x|), so two MMAs per tap give
// exact products summed in FP32 in tensor memory, the tails first.
//
// A shared-memory descriptor walks its 128 rows as 16 core matrices of 8
// rows at one stride.  A row is 16 bytes (8 channels) of one voxel, 8
// consecutive x make a core matrix, and the next core matrix is the next y
// -- and after eight of them the next z plane.  The halo is therefore kept
// three times, shifted in y by db = 0, 1, 2 (copy db holds halo rows
// y = b + db, b = 0..7, as [z 10][b 8][x 10]): in a copy a plane is 80 rows
// and eight y steps of 10 rows make exactly one plane, so tap (da, db, dc)
// of M block m is copy db from plane 2m + dc, column da, at stride 10 rows.
// Channel blocks of 8 are the K core matrices (LBO = one block).
constexpr int kTcConvWarps = 11;                        // staging warps (the first 8 also the epilogue)
constexpr int kTcEpiWarps = 8;
constexpr int kTcConvThreads = 32 * kTcConvWarps + 32;  // + the MMA warp: 12 warps
constexpr unsigned kHaloRows = kH * kT * kH;            // rows of one shifted copy: 800
constexpr unsigned kChBlockBytes = kHaloRows * 16;      // 8 channels: 12,800 B
constexpr unsigned kCopyBytes = 2 * kChBlockBytes;      // 16 channels: 25,600 B
constexpr unsigned kConvABytes = 6 * kCopyBytes;        // 3 shifts x (head, tail): 153,600 B
constexpr unsigned kConvBBytes = 27 * 512;              // the BF16 weight image: 13,824 B
constexpr size_t kConvTcSmem = kConvABytes + kConvBBytes + 64;
constexpr int kStageItems = (kH * kH * kH * 4 + 32 * kTcConvWarps - 1) / (32 * kTcConvWarps);  // 12

// The B image of one 16 -> 16 layer from its (BF16-valued) weights
// w[tap][ci][co]: per tap, [co group 2][ci block 2][co 8][ci 8] halves.
__global__ void k_conv16_image(const float* __restrict__ w, uint16_t* __restrict__ img) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 27 * 256; e += gridDim.x * blockDim.x) {
    const int tap = e >> 8, ci = (e >> 4) & 15, co = e & 15;
    img[tap * 256 + (co >> 3) * 128 + (ci >> 3) * 64 + (co & 7) * 8 + (ci & 7)] =
        (uint16_t)(__float_as_uint(w[e]) >> 16);
  }
}

// The staging warps' share of one tile's halo: 4 channels per item, every
// load in flight before the first use.
__device__ __forceinline__ void halo_load(const float* __restrict__ x, const Vol& v, uint32_t nbm, int x0, int y0,
                                          int z0, int tid, float4 (&tv)[kStageItems]) {
#pragma unroll
  for (int it = 0; it < kStageItems; ++it) {
    const int e = tid + 32 * kTcConvWarps * it;
    tv[it] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (e >= kH * kH * kH * 4) continue;
    const int q4 = e & 3, hv = e >> 2;
    const int xx = hv % kH, yy = (hv / kH) % kH, zz = hv / (kH * kH);
    const int i = x0 - 1 + xx, j = y0 - 1 + yy, k = z0 - 1 + zz;
    if (live_m(v, nbm, i, j, k, xx, yy, zz))
      tv[it] = *reinterpret_cast<const float4*>(x + ((size_t)i + (size_t)v.nx * (j + (size_t)v.ny * k)) * 16 + 4 * q4);
  }
}

// Head and tail of the items into each shifted copy that holds the voxel's row.
__device__ __forceinline__ void halo_store(unsigned char* A, const float4 (&tv)[kStageItems], int tid) {
  using namespace tc;
#pragma unroll
  for (int it = 0; it < kStageItems; ++it) {
    const int e = tid + 32 * kTcConvWarps * it;
    if (e >= kH * kH * kH * 4) continue;
    const int q4 = e & 3, hv = e >> 2;
    const int xx = hv % kH, yy = (hv / kH) % kH, zz = hv / (kH * kH);
    const float4 t = tv[it];
    const float h0 = bf16_rne(t.x), h1 = bf16_rne(t.y), h2 = bf16_rne(t.z), h3 = bf16_rne(t.w);
    const uint2 H = make_uint2(bf16_pack(h0, h1), bf16_pack(h2, h3));
    const uint2 Lo = make_uint2(bf16_pack(bf16_rne(t.x - h0), bf16_rne(t.y - h1)),
                                bf16_pack(bf16_rne(t.z - h2), bf16_rne(t.w - h3)));
    const unsigned inrow = (unsigned)(q4 >> 1) * kChBlockBytes + (unsigned)(q4 & 1) * 8u;
#pragma unroll
    for (int db = 0; db < 3; ++db) {
      const int b = yy - db;
      if (b < 0 || b >= kT) continue;
      const unsigned off = inrow + (unsigned)((zz * kT + b) * kH + xx) * 16u;
      *reinterpret_cast<uint2*>(A + (2 * db) * kCopyBytes + off) = H;
      *reinterpret_cast<uint2*>(A + (2 * db + 1) * kCopyBytes + off) = Lo;
    }
  }
}

__global__ void __launch_bounds__(kTcConvThreads, 1) k_conv16_tc(
    const float* __restrict__ x, const uint16_t* __restrict__ wimg, float* __restrict__ y, Vol v,
    const int32_t* __restrict__ list, const int32_t* __restrict__ count, const uint32_t* __restrict__ nbmask,
    int relu, const float* __restrict__ mask, int32_t* status) {
  using namespace tc;
  extern __shared__ __align__(128) float smf[];
  unsigned char* tsm = reinterpret_cast<unsigned char*>(smf);
  unsigned char* A = tsm;                                           // [db][part][ch block][z][b][x] x 16 B
  unsigned char* B = tsm + kConvABytes;                             // the weight image
  uint64_t* bar = reinterpret_cast<uint64_t*>(tsm + kConvABytes + kConvBBytes);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == kTcConvWarps) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(64)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(smem_u32(bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (unsigned e = tid; e < kConvBBytes / 16; e += blockDim.x)
    reinterpret_cast<uint4*>(B)[e] = reinterpret_cast<const uint4*>(wimg)[e];
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  fence_before();
  __syncthreads();
  fence_after();
  const unsigned tmem = *tmem_slot;
  const int n = *count;
  bool ok = true;
  unsigned phase = 0;
  // a software pipeline over the tiles: the staging warps hold the next
  // tile's halo in registers, its loads in flight while this tile's MMAs run
  float4 tv[kStageItems];
  int li = blockIdx.x;
  if (li < n && warp < kTcConvWarps) {
    int x0, y0, z0;
    tile_origin(v, list[li], x0, y0, z0);
    halo_load(x, v, nbmask[list[li]], x0, y0, z0, tid, tv);
  }
  for (; li < n; li += gridDim.x) {
    int x0, y0, z0;
    tile_origin(v, list[li], x0, y0, z0);
    const int next = li + gridDim.x;
    if (warp < kTcConvWarps) {
      halo_store(A, tv, tid);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == kTcConvWarps) {
      // ---- the MMAs: four M blocks of 16 accumulator columns; the
      // descriptors differ only in their start address
      if (lane == 0) {
        const unsigned idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);
        const uint64_t ad0 = smem_desc(smem_u32(A), kChBlockBytes, 16u * kH);
        const uint64_t bd0 = smem_desc(smem_u32(B), 128u, 256u);
        for (int m = 0; m < 4; ++m) {
          for (int part = 1; part >= 0; --part) {  // the tails first
#pragma unroll
            for (int tap = 0; tap < 27; ++tap) {
              const int da = tap % 3, db = (tap / 3) % 3, dc = tap / 9;
              const unsigned off = (unsigned)(2 * db + part) * kCopyBytes + (unsigned)((2 * m + dc) * kT * kH + da) * 16u;
              mma_ss_bf16(tmem + 16u * m, ad0 + (off >> 4), bd0 + (uint64_t)(512u * tap >> 4), idesc,
                          (part == 1 && tap == 0) ? 0u : 1u);
            }
          }
        }
        commit(smem_u32(bar));
      }
      __syncwarp();
    } else {
      // the next tile's halo loads go out now
      if (next < n) {
        int nx0, ny0, nz0;
        tile_origin(v, list[next], nx0, ny0, nz0);
        halo_load(x, v, nbmask[list[next]], nx0, ny0, nz0, tid, tv);
      }
      // ---- epilogue: warp w < 8 reads lanes 32 (w % 4).. of M blocks
      // 2 (w / 4) and 2 (w / 4) + 1; row r = a + 8 b + 64 z'
      ok = mbar_wait(smem_u32(bar), phase) && ok;
      fence_after();
      const int quarter = warp & 3, half = warp >> 2;
      const int r = 32 * quarter + lane;
      const int a = r & 7, b = (r >> 3) & 7, zq = r >> 6;
      for (int mm = 0; mm < (warp < kTcEpiWarps ? 2 : 0); ++mm) {
        const int m = 2 * half + mm;
        unsigned u[16];
        tmem_ld16(tmem + ((unsigned)(32 * quarter) << 16) + 16u * m, u);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int i = x0 + a, j = y0 + b, k = z0 + 2 * m + zq;
        if (!ok || i >= v.nx || j >= v.ny || k >= v.nz) continue;
        const size_t vox = (size_t)i + (size_t)v.nx * (j + (size_t)v.ny * k);
        float o[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          float t = __uint_as_float(u[c]);
          if (relu) t = fmaxf(t, 0.f);
          o[c] = t;
        }
        if (mask) {
          const float4* mk = reinterpret_cast<const float4*>(mask + vox * 16);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const float4 mv = mk[q];
            if (!(mv.x > 0.f)) o[4 * q] = 0.f;
            if (!(mv.y > 0.f)) o[4 * q + 1] = 0.f;
            if (!(mv.z > 0.f)) o[4 * q + 2] = 0.f;
            if (!(mv.w > 0.f)) o[4 * q + 3] = 0.f;
          }
        }
        float4* dst = reinterpret_cast<float4*>(y + vox * 16);
#pragma unroll
        for (int q = 0; q < 4; ++q) dst[q] = make_float4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
      }
    }
    phase ^= 1u;
    fence_before();
    const int bad = __syncthreads_or(!ok);
    fence_after();
    if (bad) break;
  }
  if (!ok) atomicOr(status, kStatusMmaTimeout);
  // no MMA may still be in flight when the tensor memory is freed
  if (__syncthreads_or(!ok) && warp == kTcConvWarps && lane == 0) mbar_wait(smem_u32(bar), phase ^ 1u);
  fence_before();
  __syncthreads();
  if (warp == kTcConvWarps) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64) : "memory");
  }
}

// gw[tap][ci][co] = sum_v x[v + tap - 1][ci] * g[v][co] over the active
// tiles; each CTA sums its tiles into partial[blockIdx.x][27 * CIN * COUT].
// Thread t owns (tap, ci) pairs t and t + 256 (432 pairs at CIN = 16).
template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) k_conv_wgrad(const float* __restrict__ x, const float* __restrict__ g,
                                                             Vol v, const int32_t* __restrict__ list,
                                                             const int32_t* __restrict__ count,
                                                             const uint32_t* __restrict__ nbmask,
                                                             float* __restrict__ partial, float scale_in) {
  constexpr int PS = pad_stride(CIN);
  constexpr int NP = 27 * CIN;           // (tap, ci) pairs
  constexpr int PER = (NP + kConvThreads - 1) / kConvThreads;
  extern __shared__ __align__(16) float sm[];
  float* xs = sm;                         // [kH^3][PS]
  float* gs = sm + kH * kH * kH * PS;     // [kT^3][COUT]
  float acc[PER][COUT];
#pragma unroll
  for (int p = 0; p < PER; ++p)
#pragma unroll
    for (int co = 0; co < COUT; ++co) acc[p][co] = 0.f;
  const int n = *count;
  for (int li = blockIdx.x; li < n; li += gridDim.x) {
    int x0, y0, z0;
    tile_origin(v, list[li], x0, y0, z0);
    const uint32_t nbm = nbmask[list[li]];
    __syncthreads();
    stage_halo<CIN>(x, v, nbm, x0, y0, z0, xs, scale_in);
    if constexpr (COUT % 4 == 0) {
      for (int e = threadIdx.x; e < kT * kT * kT * (COUT / 4); e += kConvThreads) {
        const int q = e % (COUT / 4), tv = e / (COUT / 4);
        const int i = x0 + tv % kT, j = y0 + (tv / kT) % kT, k = z0 + tv / (kT * kT);
        float4 val = make_float4(0.f, 0.f, 0.f, 0.f);
        if (i < v.nx && j < v.ny && k < v.nz)
          val = *reinterpret_cast<const float4*>(g + ((size_t)i + (size_t)v.nx * (j + (size_t)v.ny * k)) * COUT + 4 * q);
        *reinterpret_cast<float4*>(gs + tv * COUT + 4 * q) = val;
      }
    } else {
      for (int e = threadIdx.x; e < kT * kT * kT * COUT; e += kConvThreads) {
        const int co = e % COUT, tv = e / COUT;
        const int i = x0 + tv % kT, j = y0 + (tv / kT) % kT, k = z0 + tv / (kT * kT);
        float val = 0.f;
        if (i < v.nx && j < v.ny && k < v.nz) val = g[((size_t)i + (size_t)v.nx * (j + (size_t)v.ny * k)) * COUT + co];
        gs[tv * COUT + co] = val;
      }
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int pair = threadIdx.x + p * kConvThreads;
      if (pair >= NP) continue;
      const int tap = pair / CIN, ci = pair % CIN;
      const int da = tap % 3, db = (tap / 3) % 3, dc = tap / 9;
      for (int tv = 0; tv < kT * kT * kT; ++tv) {
        const int a = tv % kT, b = (tv / kT) % kT, c = tv / (kT * kT);
        const float xv = xs[((a + da) + kH * ((b + db) + kH * (c + dc))) * PS + ci];
        const float* gr = gs + tv * COUT;
#pragma unroll
        for (int co = 0; co < COUT; ++co) acc[p][co] = fmaf(xv, gr[co], acc[p][co]);
      }
    }
  }
  float* out = partial + (size_t)blockIdx.x * NP * COUT;
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int pair = threadIdx.x + p * kConvThreads;
    if (pair >= NP) continue;
#pragma unroll
    for (int co = 0; co < COUT; ++co) out[pair * COUT + co] = acc[p][co];
  }
}

// out[e] = sum_b partial[b][e], b in order.
__global__ void k_reduce_partials(const float* __restrict__ partial, int nb, int m, float* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nb; ++b) s += partial[(size_t)b * m + e];
    out[e] = s;
  }
}

// Voxel e's coordinates, the grid's extents and strides, by axis.
struct Cell {
  int ijk[3], n[3];
  size_t st[3];
  __device__ Cell(const Vol& v, size_t e) {
    n[0] = v.nx; n[1] = v.ny; n[2] = v.nz;
    st[0] = 1; st[1] = (size_t)v.nx; st[2] = (size_t)v.nx * v.ny;
    ijk[0] = (int)(e % v.nx); ijk[1] = (int)((e / v.nx) % v.ny); ijk[2] = (int)(e / st[2]);
  }
};

// The flux limiter.  The face flux p = F~a[u] (between u and u + e_a) moves
// charge from u + e_a into u when p > 0 and from u into u + e_a when p < 0:
// its donor is the voxel it leaves.  Voxel e gives at most its own charge
// c = s x[e]: with O its outflow (the sum of |p| over the faces it donates
// through), every flux it donates is scaled by
//     lam = 1 (O <= c),  c / O (O > c > 0),  0 (c <= 0),
// so that out >= min(x, 0) everywhere; the limited fluxes still cancel in
// pairs (no charge is added).
__global__ void k_flux_limit(const float* __restrict__ F, const float* __restrict__ x, float s, Vol v,
                             float* __restrict__ lam, float* __restrict__ outflow) {
  const size_t nvox = (size_t)v.nx * v.ny * v.nz;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nvox; e += (size_t)gridDim.x * blockDim.x) {
    const Cell q(v, e);
    float O = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (q.ijk[a] < q.n[a] - 1) O += fmaxf(-F[e * 3 + a], 0.f);        // face (e, e + e_a)
      if (q.ijk[a] > 0) O += fmaxf(F[(e - q.st[a]) * 3 + a], 0.f);      // face (e - e_a, e)
    }
    const float c = s * x[e];
    lam[e] = O <= c ? 1.f : (c > 0.f ? c / O : 0.f);
    outflow[e] = O;
  }
}

// div F^ at voxel e, F^ = the limited flux.
__device__ __forceinline__ float limited_divergence(const float* __restrict__ F, const float* __restrict__ lam,
                                                    const Vol& v, size_t e) {
  const Cell q(v, e);
  float div = 0.f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (q.ijk[a] < q.n[a] - 1) {
      const float p = F[e * 3 + a];
      div += p * (p > 0.f ? lam[e + q.st[a]] : lam[e]);
    }
    if (q.ijk[a] > 0) {
      const size_t u = e - q.st[a];
      const float p = F[u * 3 + a];
      div -= p * (p > 0.f ? lam[e] : lam[u]);
    }
  }
  return div;
}

// out = x + div F^ / s.
__global__ void k_divergence(const float* __restrict__ x, const float* __restrict__ F, const float* __restrict__ lam,
                             Vol v, float inv_s, float* __restrict__ out) {
  const size_t n = (size_t)v.nx * v.ny * v.nz;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    out[e] = x[e] + limited_divergence(F, lam, v, e) * inv_s;
}

// The loss: d = s x + div F^ - s t (the scaled output error); g = 2 d / nvox
// (its gradient); per-block partial sums of d^2 (float64).
__global__ void k_loss(const float* __restrict__ x, const float* __restrict__ F, const float* __restrict__ lam,
                       const float* __restrict__ t, float s, Vol v, float* __restrict__ g,
                       double* __restrict__ partial) {
  __shared__ double sh[256];
  double acc = 0;
  const size_t nvox = (size_t)v.nx * v.ny * v.nz;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nvox; e += (size_t)gridDim.x * blockDim.x) {
    const float d = s * x[e] + limited_divergence(F, lam, v, e) - s * t[e];
    g[e] = 2.f * d / (float)nvox;
    acc += (double)d * d;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// Backward through the limiter, first pass: T[e] = sum over the faces e
// donates through of G p, G = g[u] - g[u + e_a] the gradient at the
// limited flux of face (u, u + e_a).
__global__ void k_limit_tsum(const float* __restrict__ g, const float* __restrict__ F, Vol v,
                             float* __restrict__ tsum) {
  const size_t nvox = (size_t)v.nx * v.ny * v.nz;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nvox; e += (size_t)gridDim.x * blockDim.x) {
    const Cell q(v, e);
    float T = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (q.ijk[a] < q.n[a] - 1) {
        const float p = F[e * 3 + a];
        if (p < 0.f) T += (g[e] - g[e + q.st[a]]) * p;
      }
      if (q.ijk[a] > 0) {
        const size_t u = e - q.st[a];
        const float p = F[u * 3 + a];
        if (p > 0.f) T += (g[u] - g[e]) * p;
      }
    }
    tsum[e] = T;
  }
}

// Gradient at the network's flux F (the adjoint of the limited divergence):
// for face p = F~a[u] with donor d,
//     dL/dp = lam[d] G - [d limited] (lam[d] / O[d]) sign(p) T[d],
// d limited when O[d] > c[d] > 0; 0 on the last plane of axis a.
__global__ void k_div_adjoint(const float* __restrict__ g, const float* __restrict__ F, const float* __restrict__ x,
                              float s, const float* __restrict__ lam, const float* __restrict__ outflow,
                              const float* __restrict__ tsum, Vol v, float* __restrict__ G) {
  const size_t nvox = (size_t)v.nx * v.ny * v.nz;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nvox; e += (size_t)gridDim.x * blockDim.x) {
    const Cell q(v, e);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float r = 0.f;
      if (q.ijk[a] < q.n[a] - 1) {
        const size_t up = e + q.st[a];
        const float p = F[e * 3 + a];
        const size_t d = p > 0.f ? up : e;
        const float l = lam[d], O = outflow[d], c = s * x[d];
        r = l * (g[e] - g[up]);
        if (O > c && c > 0.f && p != 0.f) r -= (l / O) * (p > 0.f ? 1.f : -1.f) * tsum[d];
      }
      G[e * 3 + a] = r;
    }
  }
}

__global__ void k_sum_double(const double* __restrict__ partial, int n, double* out, double scale) {
  __shared__ double sh[256];
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0] * scale;
}

// Round to the nearest BF16 value, ties to even (kept as float32).
__device__ __forceinline__ float bf16_round(float f) {
  unsigned u = __float_as_uint(f);
  u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
  return __uint_as_float(u);
}

__global__ void k_bf16_round(const float* __restrict__ src, float* __restrict__ dst, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = bf16_round(src[i]);
}

// w'[tap'][co][ci] = w[tap][ci][co], tap' = 26 - tap: the weights of the
// input-gradient pass (a correlation with the flipped, transposed kernel).
__global__ void k_flip_weights(const float* __restrict__ w, float* __restrict__ wt, int cin, int cout) {
  const int m = 27 * cin * cout;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
    const int co = e % cout, ci = (e / cout) % cin, tap = e / (cin * cout);
    wt[((26 - tap) * cout + co) * cin + ci] = w[e];
  }
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

template <int CIN, int COUT>
size_t conv_smem() { return (size_t)(27 * CIN * COUT + kH * kH * kH * pad_stride(CIN)) * sizeof(float); }
template <int CIN, int COUT>
size_t wgrad_smem() { return (size_t)(kH * kH * kH * pad_stride(CIN) + kT * kT * kT * COUT) * sizeof(float); }

size_t layer_offset(int l) {
  size_t o = 0;
  for (int i = 0; i < l; ++i) o += 27 * (size_t)kLayerIn[i] * kLayerOut[i];
  return o;
}

}  // namespace

constexpr int kDnWeights = 27 * (1 * 16 + 16 * 16 + 16 * 16 + 16 * 3);  // 15,552

// Workspaces of the network on one volume.
struct Denoiser {
  Vol v{};
  int device = 0;
  int nblocks = 0;              // CTAs of the conv grids (persistent over tiles)
  int sms = 0;                  // CTAs of the tensor-core conv grid (one per SM)
  uint16_t* wimg = nullptr;     // BF16 weight image of the 16 -> 16 layer being run
  int32_t* status_own = nullptr;  // device flags of a stand-alone denoiser
  int32_t* status = nullptr;      // where its kernels raise flags (status_own, or a step's)
  float* tmax = nullptr;        // [tiles] largest |input| of each tile
  float* gmax = nullptr;        // [1] of the volume
  int32_t* amap = nullptr;      // [tiles] 1: active
  uint32_t* nbmask = nullptr;   // [tiles] active neighbours of each active tile (27 bits)
  int32_t* list = nullptr;      // [tiles]
  int32_t* count = nullptr;     // [1]
  float* act[kLayers] = {};     // output of layer l: [vox][kLayerOut[l]]
  float* gbuf[2] = {};          // gradients, [vox][16]
  float* gout = nullptr;        // gradient at the output, [vox]
  float* lam = nullptr;         // flux limiter of each donor voxel, [vox]
  float* outflow = nullptr;     // its unlimited outflow, [vox]
  float* tsum = nullptr;        // limiter backward sums, [vox]
  float* wr = nullptr;          // BF16-rounded weights used by the passes
  float* wt = nullptr;          // flipped/transposed weights of one layer
  float* partial = nullptr;     // [nblocks][27*16*16]
  double* lpart = nullptr;      // loss partials
  double* loss = nullptr;       // [1]
};

void dn_route_status(Denoiser* d, int32_t* status) { d->status = status; }

void dn_free(Denoiser* d) {
  if (!d) return;
  cudaSetDevice(d->device);
  cudaFree(d->tmax); cudaFree(d->gmax); cudaFree(d->amap); cudaFree(d->nbmask); cudaFree(d->list); cudaFree(d->count);
  for (auto& a : d->act) cudaFree(a);
  for (auto& g : d->gbuf) cudaFree(g);
  cudaFree(d->gout); cudaFree(d->lam); cudaFree(d->outflow); cudaFree(d->tsum);
  cudaFree(d->wimg); cudaFree(d->status_own);
  cudaFree(d->wr); cudaFree(d->wt); cudaFree(d->partial); cudaFree(d->lpart); cudaFree(d->loss);
  delete d;
}

Denoiser* dn_create(int nx, int ny, int nz, int device, int num_sms) {
  auto* d = new Denoiser();
  d->device = device;
  d->v = Vol{nx, ny, nz, (nx + kT - 1) / kT, (ny + kT - 1) / kT, (nz + kT - 1) / kT};
  const size_t ntiles = (size_t)d->v.tx * d->v.ty * d->v.tz, nvox = (size_t)nx * ny * nz;
  d->nblocks = num_sms * 2;
  d->sms = num_sms;
  auto alloc = [](void** p, size_t bytes) { VLB_CUDA(cudaMalloc(p, std::max<size_t>(bytes, 16))); };
  try {
    alloc((void**)&d->tmax, ntiles * 4);
    alloc((void**)&d->gmax, 4);
    alloc((void**)&d->amap, ntiles * 4);
    alloc((void**)&d->nbmask, ntiles * 4);
    alloc((void**)&d->list, ntiles * 4);
    alloc((void**)&d->count, 4);
    for (int l = 0; l < kLayers; ++l) alloc((void**)&d->act[l], nvox * kLayerOut[l] * 4);
    for (auto& g : d->gbuf) alloc((void**)&g, nvox * 16 * 4);
    alloc((void**)&d->gout, nvox * 4);
    alloc((void**)&d->wimg, 27 * 256 * 2);
    alloc((void**)&d->status_own, 4);
    VLB_CUDA(cudaMemset(d->status_own, 0, 4));
    d->status = d->status_own;
    alloc((void**)&d->lam, nvox * 4);
    alloc((void**)&d->outflow, nvox * 4);
    alloc((void**)&d->tsum, nvox * 4);
    alloc((void**)&d->wr, kDnWeights * 4);
    alloc((void**)&d->wt, 27 * 16 * 16 * 4);
    alloc((void**)&d->partial, (size_t)d->nblocks * 27 * 16 * 16 * 4);
    alloc((void**)&d->lpart, 1024 * 8);
    alloc((void**)&d->loss, 8);
  } catch (...) {
    dn_free(d);
    throw;
  }
  static bool attrs = false;
  if (!attrs) {
    VLB_CUDA(cudaFuncSetAttribute(k_conv16_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kConvTcSmem));
    VLB_CUDA(cudaFuncSetAttribute(k_conv<1, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)conv_smem<1, 16>()));
    VLB_CUDA(cudaFuncSetAttribute(k_conv<16, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)conv_smem<16, 3>()));
    VLB_CUDA(cudaFuncSetAttribute(k_conv<3, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)conv_smem<3, 16>()));
    VLB_CUDA(cudaFuncSetAttribute(k_conv_wgrad<1, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)wgrad_smem<1, 16>()));
    VLB_CUDA(cudaFuncSetAttribute(k_conv_wgrad<16, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)wgrad_smem<16, 16>()));
    VLB_CUDA(cudaFuncSetAttribute(k_conv_wgrad<16, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)wgrad_smem<16, 3>()));
    attrs = true;
  }
  return d;
}

namespace {

void conv(Denoiser& d, int cin, int cout, const float* x, const float* w, float* y, bool relu, const float* mask,
          float scale_in, cudaStream_t s) {
  const int g = d.nblocks;
  if (cin == 1 && cout == 16)
    k_conv<1, 16><<<g, kConvThreads, conv_smem<1, 16>(), s>>>(x, w, y, d.v, d.list, d.count, d.nbmask, relu, mask, scale_in);
  else if (cin == 16 && cout == 16) {
    // on the tensor cores (scale_in is 1 for these layers)
    k_conv16_image<<<27, 256, 0, s>>>(w, d.wimg);
    VLB_CUDA(cudaGetLastError());
    k_conv16_tc<<<d.sms, kTcConvThreads, kConvTcSmem, s>>>(x, d.wimg, y, d.v, d.list, d.count, d.nbmask, relu, mask,
                                                         d.status);
  }
  else if (cin == 16 && cout == 3)
    k_conv<16, 3><<<g, kConvThreads, conv_smem<16, 3>(), s>>>(x, w, y, d.v, d.list, d.count, d.nbmask, relu, mask, scale_in);
  else if (cin == 3 && cout == 16)
    k_conv<3, 16><<<g, kConvThreads, conv_smem<3, 16>(), s>>>(x, w, y, d.v, d.list, d.count, d.nbmask, relu, mask, scale_in);
  else
    throw ArgError("unsupported conv shape");
  VLB_CUDA(cudaGetLastError());
}

void wgrad(Denoiser& d, int cin, int cout, const float* x, const float* g, float* gw, float scale_in,
           cudaStream_t s) {
  const int nb = d.nblocks, m = 27 * cin * cout;
  if (cin == 1 && cout == 16)
    k_conv_wgrad<1, 16><<<nb, kConvThreads, wgrad_smem<1, 16>(), s>>>(x, g, d.v, d.list, d.count, d.nbmask, d.partial,
                                                                       scale_in);
  else if (cin == 16 && cout == 16)
    k_conv_wgrad<16, 16><<<nb, kConvThreads, wgrad_smem<16, 16>(), s>>>(x, g, d.v, d.list, d.count, d.nbmask, d.partial,
                                                                         scale_in);
  else if (cin == 16 && cout == 3)
    k_conv_wgrad<16, 3><<<nb, kConvThreads, wgrad_smem<16, 3>(), s>>>(x, g, d.v, d.list, d.count, d.nbmask, d.partial,
                                                                       scale_in);
  else
    throw ArgError("unsupported conv shape");
  VLB_CUDA(cudaGetLastError());
  k_reduce_partials<<<(m + 255) / 256, 256, 0, s>>>(d.partial, nb, m, gw);
  VLB_CUDA(cudaGetLastError());
}

}  // namespace

constexpr int kForwardLaunches = 6 + kLayers;  // kernels dn_forward launches

// Active tiles of input x, BF16 rounding of the weights, the forward pass
// (act[3] = F = f(s x), three channels, zero outside the active tiles;
// act[0..2] written on the active tiles only) and the flux limiter.
void dn_forward(Denoiser& d, const float* x, float s, const float* w_master, cudaStream_t st) {
  const size_t ntiles = (size_t)d.v.tx * d.v.ty * d.v.tz, nvox = (size_t)d.v.nx * d.v.ny * d.v.nz;
  k_tile_max<<<(unsigned)ntiles, 256, 0, st>>>(x, d.v, d.tmax);
  VLB_CUDA(cudaGetLastError());
  k_volume_max<<<1, 1024, 0, st>>>(d.tmax, (int)ntiles, d.gmax);
  VLB_CUDA(cudaGetLastError());
  VLB_CUDA(cudaMemsetAsync(d.count, 0, 4, st));
  k_tile_active<<<(unsigned)((ntiles + 255) / 256), 256, 0, st>>>(d.tmax, d.gmax, d.v, d.amap, d.list, d.count);
  VLB_CUDA(cudaGetLastError());
  k_tile_nbmask<<<(unsigned)((ntiles + 255) / 256), 256, 0, st>>>(d.amap, d.list, d.count, d.v, d.nbmask);
  VLB_CUDA(cudaGetLastError());
  k_bf16_round<<<(kDnWeights + 255) / 256, 256, 0, st>>>(w_master, d.wr, kDnWeights);
  VLB_CUDA(cudaGetLastError());
  for (int l = 0; l < kLayers; ++l) {
    if (l == kLayers - 1) VLB_CUDA(cudaMemsetAsync(d.act[l], 0, nvox * kLayerOut[l] * 4, st));  // the flux, read everywhere
    conv(d, kLayerIn[l], kLayerOut[l], l == 0 ? x : d.act[l - 1], d.wr + layer_offset(l), d.act[l], l < 3, nullptr,
         l == 0 ? s : 1.f, st);
  }
  k_flux_limit<<<(unsigned)std::min<size_t>((nvox + 255) / 256, 65535), 256, 0, st>>>(d.act[3], x, s, d.v, d.lam,
                                                                                       d.outflow);
  VLB_CUDA(cudaGetLastError());
}

// Loss against target t (same scale s) and the gradient of the master
// weights into gw (after dn_forward on the same x).
void dn_backward(Denoiser& d, const float* x, const float* t, float s, float* gw, cudaStream_t st) {
  const size_t nvox = (size_t)d.v.nx * d.v.ny * d.v.nz;
  const int lb = 1024;
  k_loss<<<lb, 256, 0, st>>>(x, d.act[3], d.lam, t, s, d.v, d.gout, d.lpart);
  VLB_CUDA(cudaGetLastError());
  k_sum_double<<<1, 256, 0, st>>>(d.lpart, lb, d.loss, 1.0 / (double)nvox);
  VLB_CUDA(cudaGetLastError());
  k_limit_tsum<<<lb, 256, 0, st>>>(d.gout, d.act[3], d.v, d.tsum);
  VLB_CUDA(cudaGetLastError());
  k_div_adjoint<<<lb, 256, 0, st>>>(d.gout, d.act[3], x, s, d.lam, d.outflow, d.tsum, d.v, d.gbuf[0]);
  VLB_CUDA(cudaGetLastError());
  int cur = 0;  // gbuf[cur]: gradient at the output of layer l
  for (int l = kLayers - 1; l >= 0; --l) {
    const int cin = kLayerIn[l], cout = kLayerOut[l];
    const float* in = l == 0 ? x : d.act[l - 1];
    wgrad(d, cin, cout, in, d.gbuf[cur], gw + layer_offset(l), l == 0 ? s : 1.f, st);
    if (l == 0) break;
    // gradient at the input of layer l = conv^T(g) masked by the ReLU of layer l-1
    k_flip_weights<<<(27 * cin * cout + 255) / 256, 256, 0, st>>>(d.wr + layer_offset(l), d.wt, cin, cout);
    VLB_CUDA(cudaGetLastError());
    conv(d, cout, cin, d.gbuf[cur], d.wt, d.gbuf[cur ^ 1], false, d.act[l - 1], 1.f, st);
    cur ^= 1;
  }
}

void dn_adam(Denoiser& d, float* w, const float* g, float* m, float* v, float lr, int step, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<(kDnWeights + 255) / 256, 256, 0, st>>>(w, g, m, v, kDnWeights, lr, b1, b2, 1e-8f, c1, c2);
  VLB_CUDA(cudaGetLastError());
}

const float* dn_output(const Denoiser& d) { return d.act[3]; }
double* dn_loss_ptr(const Denoiser& d) { return d.loss; }
int dn_active_tiles(const Denoiser& d) {
  int n = 0;
  cudaMemcpy(&n, d.count, 4, cudaMemcpyDeviceToHost);
  return n;
}

}  // namespace vlb

// ------------------------------------------------------------- in the step
namespace vlb {
namespace {

// The deposit's charge is (N - nout) w after its renormalisation; keep the
// prediction (renormalised to that charge) when its own charge is within
// `tol` of it, else keep the deposit.
__global__ void k_denoise_select(float* __restrict__ rho, const float* __restrict__ pred, size_t n,
                                 DeviceScalars* dsc, double npart_global, double w, double tol) {
  const double q_dep = (npart_global - dsc->xch[0]) * w;
  const double q_pred = dsc->xch[1];
  const bool use = fabs(q_pred - q_dep) <= tol && q_pred > 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) dsc->denoised = use ? 1 : 0;
  if (!use) return;
  const float sc = (float)(q_dep / q_pred);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    rho[i] = pred[i] * sc;
}

}  // namespace

void launch_denoise(Ctx& c, int64_t npart_global) {
  Level& F = c.fine;
  const size_t tot = (size_t)F.n * F.n * F.n;
  Denoiser& d = *c.dn;
  dn_forward(d, F.rho, (float)c.dn_scale, c.dn_weights, c.stream);
  c.launches += kForwardLaunches;
  k_divergence<<<grid_for(c, (int64_t)tot, 256, 8), 256, 0, c.stream>>>(F.rho, dn_output(d), d.lam, d.v,
                                                                         (float)(1.0 / c.dn_scale), c.dn_pred);
  VLB_LAUNCHED(c);
  launch_grid_charge(c, F, c.dn_pred, &c.dsc->xch[1]);
  k_denoise_select<<<grid_for(c, (int64_t)tot, 256, 8), 256, 0, c.stream>>>(F.rho, c.dn_pred, tot, c.dsc,
                                                                             (double)npart_global, c.weight, c.dn_tol);
  VLB_LAUNCHED(c);
}

void free_denoiser(Ctx& c) {
  if (c.dn) dn_free(c.dn);
  c.dn = nullptr;
  if (c.dn_weights) cudaFree(c.dn_weights);
  if (c.dn_pred) cudaFree(c.dn_pred);
  c.dn_weights = nullptr;
  c.dn_pred = nullptr;
}

}  // namespace vlb

// --------------------------------------------------------------- C ABI
using namespace vlb;

struct vlb_denoiser {
  Denoiser* d = nullptr;
};

namespace {
int dn_fail(int code, const std::string& m) {
  set_last_error(m);
  return code;
}
template <class F>
int dn_guard(F&& f) {
  try {
    return f();
  } catch (const CudaError& e) {
    return dn_fail(VLB_ERR_CUDA, cuda_msg(e.err, "denoiser"));
  } catch (const ArgError& e) {
    return dn_fail(VLB_ERR_ARG, e.msg);
  } catch (const std::bad_alloc&) {
    return dn_fail(VLB_ERR_NOMEM, "host allocation failed");
  }
}
}  // namespace

extern "C" {

int vlb_dn_weight_count(void) { return kDnWeights; }

int vlb_dn_create(int32_t nx, int32_t ny, int32_t nz, int32_t device, vlb_denoiser** out) {
  if (!out || nx < 1 || ny < 1 || nz < 1) return dn_fail(VLB_ERR_ARG, "vlb_dn_create: bad volume");
  *out = nullptr;
  return dn_guard([&]() -> int {
    VLB_CUDA(cudaSetDevice(device));
    int sms = 148;
    VLB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    auto* h = new vlb_denoiser();
    try {
      h->d = dn_create(nx, ny, nz, device, sms);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return VLB_OK;
  });
}

int vlb_dn_destroy(vlb_denoiser* h) {
  if (!h) return VLB_OK;
  dn_free(h->d);
  delete h;
  return VLB_OK;
}

int vlb_dn_forward(vlb_denoiser* h, const float* x, float scale, const float* weights, float* out, void* stream) {
  if (!h || !x || !weights || !out || !(scale > 0)) return dn_fail(VLB_ERR_ARG, "vlb_dn_forward: bad arguments");
  return dn_guard([&]() -> int {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Denoiser& d = *h->d;
    VLB_CUDA(cudaSetDevice(d.device));
    dn_forward(d, x, scale, weights, s);
    const size_t n = (size_t)d.v.nx * d.v.ny * d.v.nz;
    k_divergence<<<(unsigned)std::min<size_t>((n + 255) / 256, 65535), 256, 0, s>>>(x, dn_output(d), d.lam, d.v,
                                                                                      1.f / scale, out);
    VLB_CUDA(cudaGetLastError());
    return VLB_OK;
  });
}

int vlb_dn_gradient(vlb_denoiser* h, const float* x, const float* target, float scale, const float* weights,
                    float* grad, double* loss, void* stream) {
  if (!h || !x || !target || !weights || !grad || !(scale > 0))
    return dn_fail(VLB_ERR_ARG, "vlb_dn_gradient: bad arguments");
  return dn_guard([&]() -> int {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Denoiser& d = *h->d;
    VLB_CUDA(cudaSetDevice(d.device));
    dn_forward(d, x, scale, weights, s);
    dn_backward(d, x, target, scale, grad, s);
    if (loss) {
      VLB_CUDA(cudaMemcpyAsync(loss, dn_loss_ptr(d), sizeof(double), cudaMemcpyDeviceToHost, s));
      VLB_CUDA(cudaStreamSynchronize(s));
    }
    return VLB_OK;
  });
}

int vlb_dn_adam(vlb_denoiser* h, float* weights, const float* grad, float* m, float* v, float lr, int32_t step,
                void* stream) {
  if (!h || !weights || !grad || !m || !v || step < 1) return dn_fail(VLB_ERR_ARG, "vlb_dn_adam: bad arguments");
  return dn_guard([&]() -> int {
    VLB_CUDA(cudaSetDevice(h->d->device));
    dn_adam(*h->d, weights, grad, m, v, lr, step, static_cast<cudaStream_t>(stream));
    return VLB_OK;
  });
}

int vlb_dn_status(vlb_denoiser* h, int32_t* flags) {
  if (!h || !flags) return dn_fail(VLB_ERR_ARG, "vlb_dn_status: bad arguments");
  return dn_guard([&]() -> int {
    Denoiser& d = *h->d;
    VLB_CUDA(cudaSetDevice(d.device));
    VLB_CUDA(cudaDeviceSynchronize());
    VLB_CUDA(cudaMemcpy(flags, d.status_own, 4, cudaMemcpyDeviceToHost));
    VLB_CUDA(cudaMemset(d.status_own, 0, 4));
    return VLB_OK;
  });
}

int vlb_dn_active_tiles(vlb_denoiser* h, int32_t* n) {
  if (!h || !n) return dn_fail(VLB_ERR_ARG, "vlb_dn_active_tiles: bad arguments");
  return dn_guard([&]() -> int {
    VLB_CUDA(cudaSetDevice(h->d->device));
    VLB_CUDA(cudaDeviceSynchronize());
    *n = dn_active_tiles(*h->d);
    return VLB_OK;
  });
}

}  // extern "C"
