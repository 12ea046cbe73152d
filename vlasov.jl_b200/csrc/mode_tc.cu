// The rotating mode product on the fifth-generation tensor cores, in split
// precision: the plain FP32 product of poisson.cu computed as
//
//     dest[p + m*i'] = sum_i A[i', i] * src[i + n*p]
//                    ~ sum_i (Alo Bhi + Ahi Blo + Ahi Bhi)[p, i']
//
// with every operand x split into a head and a tail, products accumulated in
// FP32 in tensor memory (src/tensorsolver.jl:217-223 computes the same
// product with SGEMM on CUDA devices).  Two splits:
//   - 3xTF32 (kind::tf32): hi = rna(x) to 10 mantissa bits, lo = rna(x - hi);
//     the dropped lo*lo term and the rounding of the tails are of order
//     2^-22 |x|: close to FP32 accuracy;
//   - BF16x3 (kind::f16 with BF16 operands): hi = rn(x) to 7 mantissa bits,
//     lo = rn(x - hi); x - hi - lo and lo*lo are of order 2^-16 |x|, at twice
//     the MMA rate of TF32.
// The accumulator rounds at every MMA, so the small terms go first and the
// head products last.
//
// As a GEMM, D[p, i'] = sum_i S[p, i] A[i', i] with both operands K-major:
//   - the MMA's A operand is a tile of 128 consecutive p (rows of src, each
//     n contiguous floats).  It is bulk-copied raw into shared memory, split
//     into hi/lo by eight warps (warps w and w+4 share the rows 32(w%4).. of
//     their tensor-memory lane quarter and take alternate K groups of 8 TF32
//     or 16 BF16) and written to tensor memory with tcgen05.st, lane r =
//     row r, one TF32 or two packed BF16 (the lower K in the low half) per
//     column;
//   - the MMA's B operand is the n x n matrix (eigenvectors, their inverse, or
//     S^-1), split into hi/lo once at context creation (in both formats) and
//     stored K-chunk by K-chunk in the canonical K-major no-swizzle layout of
//     8-row x 16-byte core matrices, so bulk copies put it in shared memory
//     as the MMA reads it, one mbarrier per chunk;
//   - D is 128 lanes x N columns of FP32 in tensor memory, read back with
//     tcgen05.ld by the eight warps (thread r: row r, half of the columns)
//     and stored to dest[p + m*i'], 32 consecutive p per warp and column.
// A ninth warp issues the copies and the MMAs: the MMAs of K chunk c start
// as soon as the eight warps have split it (named barrier 1 + c), while they
// split chunk c+1.
//
// One launch runs a whole chain of up to three products with the same
// matrix (the three rotations of one operator): the matrix is loaded once,
// and a grid barrier separates the products (cooperative launch: every CTA
// is resident; one tile per CTA).  The epilogues of the FP32 kernel (times
// 1/(lx+ly+lz), into the interior of phi) are applied on the way out.
//
// Every wait is bounded: an mbarrier or grid-barrier wait that gives up sets
// a status flag and the kernel runs on to its end, waiting (bounded) for its
// own copies before it frees the tensor memory.  Named barriers hand each
// split chunk to the MMA warp; every thread passes each exactly once per
// product.

#include <algorithm>
#include <cstring>
#include <vector>

#include "tc_util.cuh"
#include "vlb_internal.cuh"

namespace vlb {

namespace {

constexpr int kTcRows = 128;       // p rows per CTA (the MMA's M)
constexpr int kTcConvWarps = 8;    // split and epilogue warps
constexpr int kTcConv = 32 * kTcConvWarps;
constexpr int kTcThreads = kTcConv + 32;  // + the copy / MMA warp
constexpr int kTcChunk = 32;       // K elements per pipeline stage
constexpr int kTcMaxChunks = 5;    // kpad8 <= 160
constexpr int kTcMaxStages = 3;    // products per launch
// mbarriers: [0, 12) raw rows of lane quarter q of product s (4 s + q),
// [12, 15) MMAs of product s, [15, 20) matrix chunk c
constexpr int kBarRaw = 0, kBarMma = 4 * kTcMaxStages, kBarImg = kBarMma + kTcMaxStages;
constexpr int kTcBars = kBarImg + kTcMaxChunks;
constexpr int kDoneBarrier = 8;    // named barrier: the MMAs of a product are done

struct TcStage {
  const float* src;
  float* dest;
  int epi;  // 0 plain, 1 times invl, 2 into the interior of phi
};

struct TcArgs {
  TcStage st[kTcMaxStages];
  int nst;
  const void* img;       // B operand image: hi then lo, each npad16 x kpad (TF32 or BF16)
  const float* invl;     // epi 1
  DeviceScalars* dsc;
  unsigned* sync;        // grid-barrier counter, zero at launch
  long long m;
  int n, npad16, kpad, pitch;   // kpad: K padded to the MMA's K (8 TF32, 16 BF16)
  int colH, colL, ncols;
  unsigned raw_bytes, img_bytes;
};

using namespace tc;

__device__ __forceinline__ void tc_fence_before() { fence_before(); }
__device__ __forceinline__ void tc_fence_after() { fence_after(); }

// The chains' B images: LBO = 128 B between the two K halves of one MMA step.
__device__ __forceinline__ uint64_t smem_desc(unsigned addr, unsigned sbo) { return tc::smem_desc(addr, 128u, sbo); }

__device__ __forceinline__ void named_arrive(int id, int count) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// All CTAs of the (cooperative) launch: this CTA's stores of the previous
// product, plain and bulk, are visible to every CTA's copies of the next.
__device__ __forceinline__ bool grid_sync(unsigned* ctr, unsigned target) {
  bool ok = true;
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __threadfence();
    atomicAdd(ctr, 1u);
    unsigned v = 0;
    for (long long it = 0; it < kSpinLimit; ++it) {
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(ctr) : "memory");
      if (v >= target) break;
      __nanosleep(64);
    }
    ok = v >= target;
    asm volatile("fence.proxy.async.global;" ::: "memory");
  }
  __syncthreads();
  tc_fence_after();
  return ok;
}

template <bool BF>
__global__ void __launch_bounds__(kTcThreads, 1) k_mode_chain_tc(TcArgs a) {
  constexpr unsigned ES = BF ? 2u : 4u;   // bytes per B element
  constexpr int EPC = 16 / (int)ES;       // B elements per 16-byte core-matrix row
  constexpr int KM = 2 * EPC;             // K of one MMA (two core matrices)
  constexpr int G = KM;                   // K elements per split group (8 tensor-memory columns)
  constexpr int CPK = BF ? 2 : 1;         // A elements per tensor-memory column
  extern __shared__ __align__(128) unsigned char smem[];
  float* raw = reinterpret_cast<float*>(smem);                                   // [128][pitch]
  unsigned char* Bimg = smem + a.raw_bytes;                                      // hi, lo
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + a.raw_bytes + 2 * a.img_bytes);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(bars + kTcBars);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nch = (a.kpad + kTcChunk - 1) / kTcChunk;
  const long long p0 = (long long)blockIdx.x * kTcRows;
  const int rows = (int)min((long long)kTcRows, a.m - p0);
  const int n = a.n;

  if (warp == kTcConvWarps) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(a.ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int b = 0; b < kTcBars; ++b) mbar_init(smem_u32(&bars[b]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tmem_slot;

  // the matrix image, once for the whole chain
  if (warp == kTcConvWarps) {
    if (lane == 0)
      for (int c = 0; c < nch; ++c)
        mbar_expect_tx(smem_u32(&bars[kBarImg + c]),
                       2u * (unsigned)a.npad16 * (unsigned)min(kTcChunk, a.kpad - kTcChunk * c) * ES);
    __syncwarp();
    if (lane < 2 * nch) {
      // lane 2c: head of chunk c, lane 2c+1: its tail
      const int c = lane >> 1, part = lane & 1;
      const unsigned off = (unsigned)a.npad16 * (unsigned)(kTcChunk * c) * ES + (part ? a.img_bytes : 0u);
      const unsigned bytes = (unsigned)a.npad16 * (unsigned)min(kTcChunk, a.kpad - kTcChunk * c) * ES;
      bulk_g2s(smem_u32(Bimg) + off, reinterpret_cast<const char*>(a.img) + off, bytes, smem_u32(&bars[kBarImg + c]));
    }
  }

  bool ok = true;
  for (int s = 0; s < a.nst; ++s) {
    if (s > 0) ok = grid_sync(a.sync, (unsigned)s * gridDim.x) && ok;
    const TcStage st = a.st[s];
    const unsigned bar_mma = smem_u32(&bars[kBarMma + s]);
    if (warp == kTcConvWarps) {
      // ---- the raw tile of this product, one mbarrier per lane quarter
      // of 32 rows so that each quarter's split starts when its rows land
      if (lane < 4) {
        const int qrows = max(0, min(32, rows - 32 * lane));
        mbar_expect_tx(smem_u32(&bars[kBarRaw + 4 * s + lane]), (unsigned)qrows * (unsigned)n * 4u);
      }
      __syncwarp();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      const char* srow = reinterpret_cast<const char*>(st.src + p0 * n);
      if (a.pitch == n) {
        // quarter q: rows 32q .. 32q+31 contiguous, qrows * n * 4 bytes (a
        // multiple of 16: n = 2 mod 4 and qrows even); lanes 4q..4q+3 copy it
        const int q = lane >> 3, part = lane & 7;
        const int qrows = max(0, min(32, rows - 32 * q));
        const unsigned qbytes = (unsigned)qrows * (unsigned)n * 4u;
        const unsigned piece = ((qbytes + 7u) / 8u + 15u) & ~15u;
        const unsigned off = part * piece;
        if (off < qbytes)
          bulk_g2s(smem_u32(raw + (size_t)32 * q * n) + off, srow + (size_t)32 * q * n * 4 + off,
                   min(piece, qbytes - off), smem_u32(&bars[kBarRaw + 4 * s + q]));
      } else {
        for (int r = lane; r < rows; r += 32)
          bulk_g2s(smem_u32(raw + (size_t)r * a.pitch), srow + (size_t)r * n * 4, (unsigned)n * 4u,
                   smem_u32(&bars[kBarRaw + 4 * s + (r >> 5)]));
      }
      // ---- MMAs: the small terms chunk by chunk, then the head products
      const unsigned idesc = (1u << 4)                                          // D: F32
                             | (BF ? (1u << 7) | (1u << 10) : (2u << 7) | (2u << 10))  // A, B: BF16 or TF32
                             | ((unsigned)(a.npad16 >> 3) << 17)                // N
                             | ((unsigned)(kTcRows >> 4) << 24);                // M
      const unsigned bh = smem_u32(Bimg), bl = bh + a.img_bytes;
      for (int c = 0; c < nch; ++c) {
        named_sync(1 + c, kTcThreads);
        if (lane == 0) {
          tc_fence_after();
          if (s == 0) ok = mbar_wait(smem_u32(&bars[kBarImg + c]), 0) && ok;
          const int kw = min(kTcChunk, a.kpad - kTcChunk * c);
          const unsigned cbase = (unsigned)a.npad16 * (unsigned)(kTcChunk * c) * ES;
          const unsigned sbo = (unsigned)(kw / EPC) * 128u;
          for (int q = 0; q < kw / KM; ++q) {
            const unsigned kb = cbase + 256u * q, ka = (unsigned)(kTcChunk * c + KM * q) / CPK;
            mma_ts<BF>(tmem, tmem + a.colL + ka, smem_desc(bh + kb, sbo), idesc, (c > 0 || q > 0) ? 1u : 0u);
            mma_ts<BF>(tmem, tmem + a.colH + ka, smem_desc(bl + kb, sbo), idesc, 1u);
          }
        }
        __syncwarp();
      }
      if (lane == 0) {
        for (int c = 0; c < nch; ++c) {
          const int kw = min(kTcChunk, a.kpad - kTcChunk * c);
          const unsigned cbase = (unsigned)a.npad16 * (unsigned)(kTcChunk * c) * ES;
          const unsigned sbo = (unsigned)(kw / EPC) * 128u;
          for (int q = 0; q < kw / KM; ++q)
            mma_ts<BF>(tmem, tmem + a.colH + (unsigned)(kTcChunk * c + KM * q) / CPK,
                       smem_desc(bh + cbase + 256u * q, sbo), idesc, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_mma)
                     : "memory");
        // one thread watches the MMAs; the split warps sleep on a named barrier
        ok = mbar_wait(bar_mma, 0) && ok;
      }
      __syncwarp();
      named_arrive(kDoneBarrier, kTcThreads);
    } else {
      // ---- split: row r of the tile, K groups of 8 alternating between the
      // two warps of a lane quarter
      const int quarter = warp & 3, half = warp >> 2;
      const int r = 32 * quarter + lane;
      const unsigned lane_base = tmem + ((unsigned)(32 * quarter) << 16);
      const bool okA = mbar_wait(smem_u32(&bars[kBarRaw + 4 * s + quarter]), 0);
      ok = okA && ok;
      const bool valid = r < rows;
      const float* row = raw + (size_t)r * a.pitch;
      for (int c = 0; c < nch; ++c) {
        const int kend = min(kTcChunk * (c + 1), a.kpad);
        for (int k0 = kTcChunk * c + G * half; k0 < kend; k0 += 2 * G) {
          float v[G];
          if (a.pitch % 4 == 0) {
#pragma unroll
            for (int q = 0; q < G / 4; ++q) {
              float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
              if (valid && k0 + 4 * q < n) t = *reinterpret_cast<const float4*>(row + k0 + 4 * q);
              v[4 * q] = t.x; v[4 * q + 1] = t.y; v[4 * q + 2] = t.z; v[4 * q + 3] = t.w;
            }
          } else {
#pragma unroll
            for (int q = 0; q < G / 2; ++q) {
              float2 t = make_float2(0.f, 0.f);
              if (valid && k0 + 2 * q < n) t = *reinterpret_cast<const float2*>(row + k0 + 2 * q);
              v[2 * q] = t.x; v[2 * q + 1] = t.y;
            }
          }
          float hi[8], lo[8];
          if constexpr (BF) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const float h0 = bf16_rne(v[2 * j]), h1 = bf16_rne(v[2 * j + 1]);
              const float l0 = bf16_rne(__fsub_rn(v[2 * j], h0)), l1 = bf16_rne(__fsub_rn(v[2 * j + 1], h1));
              hi[j] = __uint_as_float(bf16_pack(h0, h1));
              lo[j] = __uint_as_float(bf16_pack(l0, l1));
            }
          } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              hi[j] = tf32_rna(v[j]);
              lo[j] = tf32_rna(__fsub_rn(v[j], hi[j]));
            }
          }
          tmem_st8(lane_base + (unsigned)(a.colH + k0 / CPK), hi);
          tmem_st8(lane_base + (unsigned)(a.colL + k0 / CPK), lo);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        tc_fence_before();
        named_arrive(1 + c, kTcThreads);
      }
      // ---- epilogue: D row r, 32-column groups alternating between the
      // halves; every store instruction writes 32 consecutive p of one i'
      named_sync(kDoneBarrier, kTcThreads);
      tc_fence_after();
      const long long p = p0 + r;
      for (int c32 = 32 * half; c32 < a.npad16; c32 += 64) {
        unsigned v[32];
        tmem_ld16(lane_base + (unsigned)c32, v);
        if (c32 + 16 < a.npad16) tmem_ld16(lane_base + (unsigned)(c32 + 16), v + 16);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (!valid) continue;
        if (st.epi == 1) {
          // every factor in flight before the first store (dest and invl
          // could alias as far as the compiler knows)
          float f[32];
#pragma unroll
          for (int j = 0; j < 32; ++j) f[j] = c32 + j < n ? __ldg(a.invl + p + a.m * (c32 + j)) : 0.f;
#pragma unroll
          for (int j = 0; j < 32; ++j) v[j] = __float_as_uint(__uint_as_float(v[j]) * f[j]);
        }
        if (st.epi == 2) {
          const int N = n + 2;
          const int i = (int)(p % n), jj = (int)(p / n);
          float* base = st.dest + (size_t)(i + 1) + (size_t)N * (jj + 1);
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            if (c32 + j >= n) break;
            base[(size_t)N * N * (c32 + j + 1)] = __uint_as_float(v[j]);
          }
        } else {
          float* base = st.dest + p;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            if (c32 + j >= n) break;
            base[a.m * (c32 + j)] = __uint_as_float(v[j]);
          }
        }
      }
    }
  }
  if (!ok) atomicOr(&a.dsc->status, kStatusMmaTimeout);
  // nothing may still be in flight when the tensor memory is freed
  if (!ok) {
    if (warp == kTcConvWarps && lane == 0) {
      for (int c = 0; c < nch; ++c) mbar_wait(smem_u32(&bars[kBarImg + c]), 0);
      for (int s = 0; s < a.nst; ++s) mbar_wait(smem_u32(&bars[kBarMma + s]), 0);
    }
    if (warp < kTcConvWarps)
      for (int s = 0; s < a.nst; ++s) mbar_wait(smem_u32(&bars[kBarRaw + 4 * s + (warp & 3)]), 0);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kTcConvWarps) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.ncols) : "memory");
  }
}

int raw_pitch(int n) {
  if (n % 4 != 0) return n;  // n = 2 mod 4: contiguous rows, 8-byte loads
  int p = n;
  while ((p / 4) % 2 == 0) p += 4;  // 16-byte rows, an odd number of 16-byte groups
  return p;
}

int round_up(int x, int m) { return (x + m - 1) / m * m; }

TcArgs tc_args(const TcImage& A, long long m, bool bf) {
  TcArgs a{};
  a.n = A.n;
  a.npad16 = A.npad16;
  a.kpad = bf ? A.kpad16 : A.kpad8;
  a.m = m;
  a.pitch = raw_pitch(A.n);
  a.raw_bytes = (unsigned)round_up(kTcRows * a.pitch * 4, 128);
  a.img_bytes = (unsigned)((size_t)A.npad16 * a.kpad * (bf ? 2 : 4));
  const int kcols = bf ? a.kpad / 2 : a.kpad;  // tensor-memory columns of one A split
  a.colH = round_up(A.npad16, 32);
  a.colL = a.colH + round_up(kcols, 32);
  int need = a.colL + kcols, cols = 32;
  while (cols < need) cols *= 2;
  a.ncols = cols;
  a.img = bf ? static_cast<const void*>(A.bimg) : static_cast<const void*>(A.img);
  return a;
}

size_t tc_smem(const TcArgs& a) { return (size_t)a.raw_bytes + 2 * (size_t)a.img_bytes + 8 * kTcBars + 16; }

}  // namespace

bool tc_supported(int n) {
  // N (npad16) <= 256 and the three column ranges within 512
  if (n < 8 || n > 144 || n % 2 || (n + 7) / 8 * 8 > kTcChunk * kTcMaxChunks) return false;
  TcImage t;
  t.n = n;
  t.npad16 = round_up(n, 16);
  t.kpad8 = round_up(n, 8);
  t.kpad16 = round_up(n, 16);
  for (bool bf : {false, true}) {
    const TcArgs a = tc_args(t, 1, bf);
    if (a.ncols > 512 || tc_smem(a) > 227 * 1024 || a.kpad > kTcChunk * kTcMaxChunks) return false;
  }
  return true;
}

namespace {
float round_bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;  // nearest, ties to even
  std::memcpy(&f, &u, 4);
  return f;
}
uint16_t bits_bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return (uint16_t)(u >> 16);
}
}  // namespace

TcImage make_tc_image(const double* A, int n) {
  TcImage t;
  if (!tc_supported(n)) return t;
  t.n = n;
  t.npad16 = round_up(n, 16);
  t.kpad8 = round_up(n, 8);
  t.kpad16 = round_up(n, 16);
  const size_t per = (size_t)t.npad16 * t.kpad8, bper = (size_t)t.npad16 * t.kpad16;
  std::vector<uint16_t> hb(2 * bper, 0);
  std::vector<float> h(2 * per, 0.f);
  for (int r = 0; r < n; ++r)
    for (int k = 0; k < n; ++k) {
      const double x = A[(size_t)r * n + k];
      uint32_t u;
      const float f = (float)x;
      std::memcpy(&u, &f, 4);
      u = (u + 0x1000u) & 0xFFFFE000u;  // round the magnitude to 10 mantissa bits, ties away
      float hi;
      std::memcpy(&hi, &u, 4);
      float lo = (float)(x - (double)hi);
      std::memcpy(&u, &lo, 4);
      u = (u + 0x1000u) & 0xFFFFE000u;
      std::memcpy(&lo, &u, 4);
      // chunk c of kTcChunk K elements is one contiguous block (npad16 rows);
      // inside it, 8-row groups of (width / 4) core matrices of 8 x 16 bytes
      const int c = k / kTcChunk, kc = k - kTcChunk * c;
      const int width = std::min(kTcChunk, t.kpad8 - kTcChunk * c);
      const size_t o = (size_t)t.npad16 * kTcChunk * c + (size_t)(r / 8) * (width / 4) * 32 +
                       (size_t)(kc / 4) * 32 + (size_t)(r % 8) * 4 + (kc % 4);
      h[o] = hi;
      h[per + o] = lo;
      // the BF16 image: core matrices of 8 rows x 8 halves
      const int bwidth = std::min(kTcChunk, t.kpad16 - kTcChunk * c);
      const size_t bo = (size_t)t.npad16 * kTcChunk * c + (size_t)(r / 8) * (bwidth / 8) * 64 +
                        (size_t)(kc / 8) * 64 + (size_t)(r % 8) * 8 + (kc % 8);
      const float bh = round_bf16((float)x);
      const float bl = round_bf16((float)(x - (double)bh));
      hb[bo] = bits_bf16(bh);
      hb[bper + bo] = bits_bf16(bl);
    }
  void* d = nullptr;
  VLB_CUDA(cudaMalloc(&d, 2 * per * sizeof(float)));
  t.img = static_cast<float*>(d);
  VLB_CUDA(cudaMemcpy(t.img, h.data(), 2 * per * sizeof(float), cudaMemcpyHostToDevice));
  VLB_CUDA(cudaMalloc(&d, 2 * bper * sizeof(uint16_t)));
  t.bimg = static_cast<uint16_t*>(d);
  VLB_CUDA(cudaMemcpy(t.bimg, hb.data(), 2 * bper * sizeof(uint16_t), cudaMemcpyHostToDevice));
  return t;
}

void tc_setup(Ctx& c) {
  VLB_CUDA(cudaFuncSetAttribute(k_mode_chain_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  VLB_CUDA(cudaFuncSetAttribute(k_mode_chain_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  if (!c.tc_sync) {
    void* d = nullptr;
    VLB_CUDA(cudaMalloc(&d, 64 * sizeof(unsigned)));
    c.tc_sync = static_cast<unsigned*>(d);
    VLB_CUDA(cudaMemset(c.tc_sync, 0, 64 * sizeof(unsigned)));
  }
}

void launch_mode_chain_tc(Ctx& c, const TcImage& A, int nst, const float* const* src, float* const* dest,
                          const int* epi, long long m, const float* invl) {
  if (!A.img || !A.bimg) throw ArgError("no tensor-core image for this matrix (the products need an even n <= 144)");
  if (nst < 1 || nst > kTcMaxStages) throw ArgError("a tensor-core chain has 1 to 3 products");
  const bool bf = c.mode_precision == VLB_POISSON_BF16X3;
  TcArgs a = tc_args(A, m, bf);
  a.nst = nst;
  for (int s = 0; s < nst; ++s) a.st[s] = TcStage{src[s], dest[s], epi[s]};
  a.invl = invl;
  a.dsc = c.dsc;
  a.sync = c.tc_sync;
  const unsigned grid = (unsigned)((m + kTcRows - 1) / kTcRows);
  if ((int)grid > c.num_sms) throw ArgError("tensor-core chain: more tiles than SMs");
  VLB_CUDA(cudaMemsetAsync(c.tc_sync, 0, sizeof(unsigned), c.stream));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kTcThreads);
  cfg.dynamicSmemBytes = tc_smem(a);
  cfg.stream = c.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (bf)
    VLB_CUDA(cudaLaunchKernelEx(&cfg, k_mode_chain_tc<true>, a));
  else
    VLB_CUDA(cudaLaunchKernelEx(&cfg, k_mode_chain_tc<false>, a));
  VLB_LAUNCHED(c);
}

}  // namespace vlb
