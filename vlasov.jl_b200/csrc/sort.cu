// Stable counting sort of the packed cloud by fine cell, on the device.
//
// Replaces the reference's _device_sort! (src/accelerator.jl:421-446:
// atomic histogram, host scan, unstable atomic placement, copy back) and its
// out-of-stencil list (src/kernels.jl:1041-1058).  The order produced here is
// the stable order of the host cellsort! (src/sorting.jl:163-204): by cell,
// then by index before the sort.
//
//   1. cell keys + warp-aggregated histogram over nk^3 cells;
//   2. a decoupled look-back scan that compacts the occupied cells;
//   3. one CTA scans the occupied cells (a few thousand): their bounds, the
//      gather's work items (chunks of at most `chunk` particles) and the
//      out-of-stencil slots, all functions of the cell alone; one warp per
//      occupied cell then writes the item list and the out-of-stencil list
//      (increasing slot order);
//   4. LSD radix sort of (key, index) in passes of at most 10 bits, each
//      pass stable (warp multi-split ranks + a scanned digit table);
//   5. one gather of the 48-byte records into the other buffer (swap).
//
// Every spin of the look-back is bounded: after kSpinLimit polls (or the
// context's scan_wait_polls) the tile records kStatusScanTimeout in the
// step's status word and stops waiting; it then sums its predecessors'
// inputs itself, so the scan's result stays exact and every index it hands
// on stays in range.

#include "vlb_internal.cuh"

namespace vlb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;  // 4096
constexpr int kRadixThreads = 256;
constexpr int kRadixWarps = kRadixThreads / 32;
constexpr int kRadixPerWarp = 512;
constexpr int kRadixTile = kRadixWarps * kRadixPerWarp;  // 4096
constexpr int kMaxDigitBits = 10;
constexpr long long kSpinLimit = 1ll << 22;

constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagIncl = 2ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1;

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---------------------------------------------------------------- keys
// Cell key of every particle and the histogram of cells.  The cloud is
// nearly sorted from the previous step, so neighbouring lanes usually share
// a cell: one atomic per group of equal keys in a warp.
__global__ void __launch_bounds__(256) k_keys_hist(int64_t N, int64_t Npad, const int32_t* __restrict__ k,
                                                   int nk, uint32_t* __restrict__ keys,
                                                   int32_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * blockDim.x / 32;
  for (int64_t base = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x - lane); base < N; base += warps * 32) {
    int64_t i = base + lane;
    bool valid = i < N;
    unsigned m = __ballot_sync(0xffffffffu, valid);
    if (valid) {
      uint32_t key = cell_key(k[i], k[Npad + i], k[2 * Npad + i], nk);
      keys[i] = key;
      unsigned peers = __match_any_sync(m, key);
      int leader = __ffs(peers) - 1;
      if (lane == leader) atomicAdd(&counts[key], __popc(peers));
    }
  }
}

// -------------------------------------------------------------- the scan
// Exclusive scan of n unsigned values produced by `in`, delivered to `out`
// as (index, exclusive prefix, value).  Single pass: tiles take tickets in
// launch order and read their prefix from their predecessors' published
// aggregates (decoupled look-back).  `total` receives the sum.
struct ScanInArray { const uint32_t* a; __device__ uint32_t operator()(int64_t i) const { return a[i]; } };
struct ScanOutArray { uint32_t* a; __device__ void operator()(int64_t i, uint32_t p, uint32_t) const { a[i] = p; } };

struct ScanInOccupied { const int32_t* c; __device__ uint32_t operator()(int64_t i) const { return c[i] > 0 ? 1u : 0u; } };
struct ScanOutOccupied {
  int32_t* occupied;
  int32_t* index;  // dense cell -> occupied index (meaningful for occupied cells only)
  __device__ void operator()(int64_t i, uint32_t p, uint32_t v) const {
    if (v) {
      occupied[p] = (int32_t)i;
      index[i] = (int32_t)p;
    }
  }
};

// One CTA over the occupied cells g < nocc (in increasing cell order):
// exclusive prefixes of the particle count (bounds), of the number of work
// items (ceil(count / chunk)) and of the particles of cells whose 10^3
// stencil leaves the fine grid (out_start, -1 for the others); totals into
// bounds[nocc], nitems and outcount.
constexpr int kListThreads = 1024;

__device__ __forceinline__ void block_scan3(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t* tot) {
  // exclusive scan of three counters over the CTA; tot receives the sums
  __shared__ uint32_t sh[3][kListThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t v[3] = {a, b, c}, incl[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    uint32_t x = v[q];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    incl[q] = x;
    if (lane == 31) sh[q][w] = x;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      uint32_t x = sh[q][lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      sh[q][lane] = x;  // inclusive over warps
    }
  }
  __syncthreads();
  const uint32_t wb[3] = {w ? sh[0][w - 1] : 0u, w ? sh[1][w - 1] : 0u, w ? sh[2][w - 1] : 0u};
  a = wb[0] + incl[0] - v[0];
  b = wb[1] + incl[1] - v[1];
  c = wb[2] + incl[2] - v[2];
  tot[0] = sh[0][31];
  tot[1] = sh[1][31];
  tot[2] = sh[2][31];
}

__global__ void __launch_bounds__(kListThreads) k_cell_lists(const int32_t* __restrict__ counts,
                                                             const int32_t* __restrict__ occupied, DeviceScalars* dsc,
                                                             int nk, int n, int32_t* __restrict__ bounds,
                                                             int32_t* __restrict__ chunk_start,
                                                             int32_t* __restrict__ out_start, int chunk,
                                                             int parity) {
  // chunks of kListThreads * 4 occupied cells, four consecutive cells per
  // thread: their cell codes, then their counts, as independent loads; a
  // block scan of the thread sums and the running totals of earlier chunks
  constexpr int kPer = 4;
  const int nocc = dsc->noccupied;
  uint32_t carry[3] = {0u, 0u, 0u};
  for (int base = 0; base < nocc; base += kListThreads * kPer) {
    const int g0 = base + (int)threadIdx.x * kPer;
    int cell[kPer];
    uint32_t cnt[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) cell[j] = g0 + j < nocc ? occupied[g0 + j] : -1;
#pragma unroll
    for (int j = 0; j < kPer; ++j) cnt[j] = cell[j] >= 0 ? (uint32_t)counts[cell[j]] : 0u;
    bool fits[kPer];
    uint32_t sc = 0, sch = 0, so = 0;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      int kx = 1, ky = 1, kz = 1;
      if (cell[j] >= 0) cell_knots((uint32_t)cell[j], nk, kx, ky, kz);
      fits[j] = cell[j] < 0 || field_fits(kx, ky, kz, n);
      sc += cnt[j];
      sch += (cnt[j] + chunk - 1) / chunk;
      if (!fits[j]) so += cnt[j];
    }
    uint32_t tot[3];
    block_scan3(sc, sch, so, tot);
    sc += carry[0];
    sch += carry[1];
    so += carry[2];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int g = g0 + j;
      if (g >= nocc) break;
      bounds[g] = (int32_t)sc;
      chunk_start[g] = (int32_t)sch;
      out_start[g] = fits[j] ? -1 : (int32_t)so;
      sc += cnt[j];
      sch += (cnt[j] + chunk - 1) / chunk;
      if (!fits[j]) so += cnt[j];
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) carry[q] += tot[q];
    __syncthreads();  // block_scan3's shared sums are reused by the next chunk
  }
  if (threadIdx.x == 0) {
    bounds[nocc] = (int32_t)carry[0];
    dsc->nitems = (int32_t)carry[1];
    dsc->outcount = (int32_t)carry[2];
    dsc->nocc_par[parity] = nocc;
    dsc->nitems_par[parity] = (int32_t)carry[1];
  }
}

// One warp per occupied cell: its work items and, for cells whose stencil
// leaves the fine grid, its slots in the out-of-stencil list.
__global__ void __launch_bounds__(256) k_expand_lists(const int32_t* __restrict__ occupied,
                                                      const int32_t* __restrict__ bounds,
                                                      const int32_t* __restrict__ chunk_start,
                                                      const int32_t* __restrict__ out_start, const DeviceScalars* dsc,
                                                      int32_t* __restrict__ item_cell, int4* __restrict__ item_rec,
                                                      int32_t* __restrict__ outlist, int chunk, int nk) {
  const int nocc = dsc->noccupied;
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < nocc; g += warps) {
    const int b0 = bounds[g], cnt = bounds[g + 1] - b0;
    const int nch = (cnt + chunk - 1) / chunk, c0 = chunk_start[g];
    const int code = occupied[g];
    int kx, ky, kz;
    cell_knots((uint32_t)code, nk, kx, ky, kz);
    const int knots = kx | (ky << 10) | (kz << 20);
    for (int ch = lane; ch < nch; ch += 32) {
      item_cell[c0 + ch] = g;
      const int s0 = b0 + ch * chunk;
      item_rec[c0 + ch] = make_int4(code, s0, min(s0 + chunk, b0 + cnt), knots);
    }
    const int o0 = out_start[g];
    if (o0 >= 0)
      for (int j = lane; j < cnt; j += 32) outlist[o0 + j] = b0 + j;
  }
}

template <class In, class Out>
__global__ void __launch_bounds__(kScanThreads) k_scan(In in, Out out, int64_t n, unsigned long long* status,
                                                       unsigned long long* ticket, int32_t* total,
                                                       int32_t* err, long long spin_limit, const int32_t* gate) {
  if (gate && *gate == 0) return;  // a gated scan of the radix path that the step did not take
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ unsigned long long s_prefix;
  __shared__ unsigned long long s_part[kScanThreads / 32];
  __shared__ unsigned long long s_agg;
  __shared__ int64_t s_tile;
  __shared__ int s_fallback;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) {
    s_tile = (int64_t)atomicAdd(ticket, 1ull);
    s_fallback = 0;
  }
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t base = tile * kScanTile + (int64_t)tid * kScanItems;
  uint32_t v[kScanItems];
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    int64_t i = base + j;
    v[j] = i < n ? in(i) : 0u;
    sum += v[j];
  }
  // block exclusive scan of the thread sums
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    uint32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < kScanThreads / 32) s_warp[lane] = wi - w;  // exclusive warp offsets
    if (lane == kScanThreads / 32 - 1) {
      unsigned long long agg = wi;  // tile aggregate
      unsigned long long prefix = 0;
      s_agg = agg;
      if (tile == 0) {
        st_relaxed(&status[0], kFlagIncl | agg);
      } else {
        st_relaxed(&status[tile], kFlagAgg | agg);
        // spin_limit < 0: give up before the first poll (a test of the fallback)
        bool gave_up = spin_limit < 0;
        int64_t j = tile - 1;
        long long spins = 0;
        while (!gave_up && j >= 0) {
          unsigned long long s = ld_relaxed(&status[j]);
          unsigned long long flag = s & ~kValMask;
          if (flag == 0) {
            if (++spins > spin_limit) { gave_up = true; break; }
            __nanosleep(32);
            continue;
          }
          prefix += s & kValMask;
          if (flag == kFlagIncl) break;
          --j;
        }
        if (gave_up) {
          atomicOr(err, kStatusScanTimeout);
          s_fallback = 1;  // the CTA sums the predecessors' inputs itself, below
        } else {
          st_relaxed(&status[tile], kFlagIncl | (prefix + agg));
        }
      }
      s_prefix = prefix;
      if (total && !s_fallback && (tile + 1) * (int64_t)kScanTile >= n) *total = (int32_t)(prefix + agg);
    }
  }
  __syncthreads();
  if (s_fallback) {
    // The wait gave up: the tile's exclusive prefix straight from the inputs
    // of every earlier tile (bounded work, no waiting), published as the
    // look-back would have published it.  The scan's result is unchanged;
    // the status bit reports that a wait ran out.
    const int64_t lim = tile * (int64_t)kScanTile;
    unsigned long long acc = 0;
    for (int64_t i = tid; i < lim; i += kScanThreads) acc += in(i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) s_part[wid] = acc;
    __syncthreads();
    if (tid == 0) {
      unsigned long long prefix = 0;
      for (int w = 0; w < kScanThreads / 32; ++w) prefix += s_part[w];
      st_relaxed(&status[tile], kFlagIncl | (prefix + s_agg));
      if (total && (tile + 1) * (int64_t)kScanTile >= n) *total = (int32_t)(prefix + s_agg);
      s_prefix = prefix;
    }
    __syncthreads();
  }
  uint32_t run = (uint32_t)s_prefix + s_warp[wid] + (incl - sum);
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    int64_t i = base + j;
    if (i < n) out(i, run, v[j]);
    run += v[j];
  }
}

template <class In, class Out>
void scan(Ctx& c, In in, Out out, int64_t n, int slot, int32_t* total, const int32_t* gate = nullptr,
          cudaStream_t stream = nullptr) {
  if (n <= 0) return;
  int64_t tiles = (n + kScanTile - 1) / kScanTile;
  int64_t per_slot = c.scan_status_size / 8;
  if (tiles > per_slot) throw ArgError("scan larger than its status slot");
  unsigned long long* st = c.scan_status + slot * per_slot;
  const long long limit = c.scan_wait_polls == 0 ? kSpinLimit : (long long)c.scan_wait_polls;
  k_scan<In, Out><<<(unsigned)tiles, kScanThreads, 0, stream ? stream : c.stream>>>(
      in, out, n, st, &c.dsc->scan_tiles[slot], total, &c.dsc->status, limit, gate);
  VLB_LAUNCHED(c);
}

// ------------------------------------------------------------- radix sort
__global__ void __launch_bounds__(kRadixThreads) k_radix_upsweep(const uint32_t* __restrict__ keys, int64_t N,
                                                                 int shift, uint32_t mask,
                                                                 uint32_t* __restrict__ table, int64_t ntiles,
                                                                 const int32_t* gate) {
  if (gate && *gate == 0) return;
  __shared__ uint32_t hist[1 << kMaxDigitBits];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int b = tid; b <= (int)mask; b += kRadixThreads) hist[b] = 0;
  __syncthreads();
  const int64_t tile = blockIdx.x;
  constexpr int R = kRadixPerWarp / 32;
  uint32_t kv[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t e = tile * kRadixTile + (int64_t)w * kRadixPerWarp + r * 32 + lane;
    kv[r] = e < N ? keys[e] : 0u;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    int64_t e = tile * kRadixTile + (int64_t)w * kRadixPerWarp + r * 32 + lane;
    bool valid = e < N;
    unsigned m = __ballot_sync(0xffffffffu, valid);
    if (valid) {
      uint32_t d = (kv[r] >> shift) & mask;
      unsigned peers = __match_any_sync(m, d);
      if (lane == __ffs(peers) - 1) atomicAdd(&hist[d], (uint32_t)__popc(peers));
    }
  }
  __syncthreads();
  for (int b = tid; b <= (int)mask; b += kRadixThreads) table[(int64_t)b * ntiles + tile] = hist[b];
}

// The tile's scatter.  Its digit bases (one column of the scanned table,
// strided by the tile count) are staged in shared memory first, their loads
// in flight with the keys', so that no element waits on a global load for
// its address.
__global__ void __launch_bounds__(kRadixThreads) k_radix_downsweep(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, uint32_t* __restrict__ keys_out,
    uint32_t* __restrict__ vals_out, int64_t N, int shift, uint32_t mask, const uint32_t* __restrict__ table,
    int64_t ntiles, const int32_t* gate) {
  if (gate && *gate == 0) return;
  __shared__ uint32_t whist[kRadixWarps][1 << kMaxDigitBits];
  __shared__ uint32_t sbase[1 << kMaxDigitBits];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int nb = (int)mask + 1;
  for (int b = tid; b < nb; b += kRadixThreads) sbase[b] = table[(int64_t)b * ntiles + blockIdx.x];
  for (int b = lane; b < nb; b += 32) whist[w][b] = 0;
  __syncwarp();
  const int64_t tile = blockIdx.x;
  constexpr int R = kRadixPerWarp / 32;
  uint32_t key[R], val[R], local[R];
  unsigned valid_bits = 0;
  // every load of the thread in flight before the ranking uses them
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t e = tile * kRadixTile + (int64_t)w * kRadixPerWarp + r * 32 + lane;
    const bool valid = e < N;
    key[r] = valid ? keys_in[e] : 0u;
    val[r] = valid ? (vals_in ? vals_in[e] : (uint32_t)e) : 0u;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    int64_t e = tile * kRadixTile + (int64_t)w * kRadixPerWarp + r * 32 + lane;
    bool valid = e < N;
    unsigned m = __ballot_sync(0xffffffffu, valid);
    local[r] = 0;
    if (valid) {
      valid_bits |= 1u << r;
      uint32_t d = (key[r] >> shift) & mask;
      unsigned peers = __match_any_sync(m, d);
      int leader = __ffs(peers) - 1;
      uint32_t b = 0;
      if (lane == leader) {
        b = whist[w][d];
        whist[w][d] = b + (uint32_t)__popc(peers);
      }
      b = __shfl_sync(m, b, leader);
      local[r] = b + (uint32_t)__popc(peers & lanemask_lt());
    }
    __syncwarp();
  }
  __syncthreads();
  // exclusive scan over warps, per digit
  for (int b = tid; b < nb; b += kRadixThreads) {
    uint32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < kRadixWarps; ++ww) {
      uint32_t t = whist[ww][b];
      whist[ww][b] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (!(valid_bits & (1u << r))) continue;
    uint32_t d = (key[r] >> shift) & mask;
    uint32_t pos = sbase[d] + whist[w][d] + local[r];
    if (keys_out) keys_out[pos] = key[r];
    vals_out[pos] = val[r];
  }
}

// ------------------------------------------------ the nearly sorted path
// After a step the cloud is still in the order of its last sort: slots are
// grouped by old cell (in increasing cell order), and the push has written
// every particle's new cell key.  A particle that moves at most one cell per
// axis has a key difference D = new - old equal to one of 27 offsets
// dx + nk dy + nk^2 dz (dx, dy, dz in {-1, 0, 1}; direction d = (dx + 1) +
// 3 (dy + 1) + 9 (dz + 1)).  The stable order by new key then follows from
// counts alone: the particles of new cell c come from the old cells
// c - off(d), in increasing old-cell order (decreasing d), each group in slot
// order.  So
//   A  counts, per old work item and direction, its particles;
//   A2 turns them into each item's prefix within its cell, and the cell's
//      totals per direction;
//   B  gives each (old cell, direction) group its first slot in the new
//      order: one warp per new cell sums the groups that precede it;
//   C  ranks each particle within its group by slot: perm[base + prefix +
//      rank] = s.
// A particle whose D is none of the 27 offsets sets sort_far, and the step
// takes the radix passes instead (gated on that flag).  Each new cell's
// groups must add up to its count from the push's histogram, else B sets
// the flag as well: the path never guesses.

// Direction of a key difference D, or -1 for none of the 27 offsets.  With
// t = D + 1 + nk + nk^2 = dx' + nk dy' + nk^2 dz' (each primed digit in 0..2
// for a neighbour), the digits come from comparisons: dz' is 2, 1 or 0 as t
// reaches 2 nk^2, nk^2 or not, dy' likewise on the remainder, and the last
// remainder dx' must be at most 2 (any other D leaves a larger one).
__device__ __forceinline__ int direction_of(int64_t D, int nk) {
  if (D == 0) return 13;  // most particles stay in their cell
  const int64_t nk2 = (int64_t)nk * nk;
  int64_t t = D + 1 + nk + nk2;
  if (t < 0) return -1;
  const int dz = t >= 2 * nk2 ? 2 : (t >= nk2 ? 1 : 0);
  t -= dz * nk2;
  const int dy = t >= 2 * (int64_t)nk ? 2 : (t >= nk ? 1 : 0);
  t -= (int64_t)dy * nk;
  if (t > 2) return -1;
  return (int)t + 3 * dy + 9 * dz;
}

__device__ __forceinline__ int64_t direction_offset(int d, int nk) {
  const int dx = d % 3 - 1, dy = (d / 3) % 3 - 1, dz = d / 9 - 1;
  return dx + (int64_t)nk * (dy + (int64_t)nk * dz);
}

constexpr int kDirs = 27;
constexpr int kNearThreads = 256;
constexpr int kNearKeys = 4;  // 32-slot rounds whose keys a warp loads at once (a work item of 128)

// The work items of the last sort (runs of at most chunk_old particles of
// one old cell, in slot order) spread the work evenly: A and C take one warp
// per item, A2 one warp per old cell over its few items.

// A: per item, the particles of each direction -> item_dir[item][27].  The
// item's old cell code and slots come from the last sort's item records (one
// load, the next item's in flight meanwhile).
__global__ void __launch_bounds__(kNearThreads) k_near_count(const int4* __restrict__ rec_old, DeviceScalars* dsc,
                                                            int par_old, const uint32_t* __restrict__ keys, int nk,
                                                            int32_t* __restrict__ item_dir) {
  __shared__ int32_t cnt[kNearThreads / 32][kDirs];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nitems = dsc->nitems_par[par_old];
  const int warps = gridDim.x * (kNearThreads / 32);
  bool far = false;
  int item = blockIdx.x * (kNearThreads / 32) + w;
  int4 rec = item < nitems ? rec_old[item] : make_int4(0, 0, 0, 0);
  for (; item < nitems; item += warps) {
    const int next = item + warps;
    const int4 rnext = next < nitems ? rec_old[next] : make_int4(0, 0, 0, 0);
    if (lane < kDirs) cnt[w][lane] = 0;
    __syncwarp();
    const int64_t o = rec.x;
    const int s0 = rec.y, s1 = rec.z;
    for (int base = s0; base < s1; base += 32 * kNearKeys) {
      uint32_t kv[kNearKeys];  // the keys of up to 32 kNearKeys slots, all loads in flight
#pragma unroll
      for (int u = 0; u < kNearKeys; ++u) {
        const int s = base + 32 * u + lane;
        kv[u] = s < s1 ? keys[s] : 0u;
      }
#pragma unroll
      for (int u = 0; u < kNearKeys; ++u) {
        const int s = base + 32 * u + lane;
        const bool valid = s < s1;
        const unsigned m = __ballot_sync(0xffffffffu, valid);
        if (m == 0) break;
        if (valid) {
          const int d = direction_of((int64_t)kv[u] - o, nk);
          far |= d < 0;
          const unsigned peers = __match_any_sync(m, d < 0 ? kDirs : d);
          if (d >= 0 && lane == __ffs(peers) - 1) cnt[w][d] += __popc(peers);
        }
        __syncwarp();
      }
    }
    if (lane < kDirs) item_dir[(size_t)item * kDirs + lane] = cnt[w][lane];
    __syncwarp();
    rec = rnext;
  }
  if (__any_sync(0xffffffffu, far) && lane == 0) atomicOr(&dsc->sort_far, 1);
}

// A2: per old cell (one warp, lane d a direction), the exclusive prefix of
// its items' counts in item order, in place, and the cell's totals.
__global__ void __launch_bounds__(kNearThreads) k_near_prefix(const int32_t* __restrict__ cstart_old,
                                                             const DeviceScalars* dsc, int par_old,
                                                             int32_t* __restrict__ item_dir,
                                                             int32_t* __restrict__ dir_cnt) {
  if (dsc->sort_far) return;
  const int lane = threadIdx.x & 31;
  const int nocc = dsc->nocc_par[par_old], nitems = dsc->nitems_par[par_old];
  const int warps = gridDim.x * (kNearThreads / 32);
  for (int g = blockIdx.x * (kNearThreads / 32) + (threadIdx.x >> 5); g < nocc; g += warps) {
    const int i0 = cstart_old[g], i1 = g + 1 < nocc ? cstart_old[g + 1] : nitems;
    if (lane >= kDirs) continue;
    int run = 0;
    for (int i = i0; i < i1; i += 16) {  // up to sixteen independent loads in flight
      int v[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) v[u] = i + u < i1 ? item_dir[(size_t)(i + u) * kDirs + lane] : 0;
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        if (i + u < i1) item_dir[(size_t)(i + u) * kDirs + lane] = run;
        run += v[u];
      }
    }
    dir_cnt[(size_t)g * kDirs + lane] = run;
  }
}

// B: one warp per new occupied cell c.  Lane l < 27 holds the group of
// direction d = 26 - l (its old cell c - off(d) increases with l); an
// exclusive scan over the lanes gives each group's first slot.
__global__ void __launch_bounds__(kNearThreads) k_near_bases(const int32_t* __restrict__ occ_new,
                                                            const int32_t* __restrict__ bnd_new,
                                                            const int32_t* __restrict__ occ_old,
                                                            const int32_t* __restrict__ cidx_old,
                                                            DeviceScalars* dsc, int par_old, int ncell, int nk,
                                                            const int32_t* __restrict__ dir_cnt,
                                                            int32_t* __restrict__ dir_base) {
  if (dsc->sort_far) return;
  const int lane = threadIdx.x & 31;
  const int nocc_new = dsc->noccupied, nocc_old = dsc->nocc_par[par_old];
  const int warps = gridDim.x * (kNearThreads / 32);
  bool bad = false;
  for (int g = blockIdx.x * (kNearThreads / 32) + (threadIdx.x >> 5); g < nocc_new; g += warps) {
    const int64_t c = occ_new[g];
    int len = 0, gs = -1;
    const int d = kDirs - 1 - lane;
    if (lane < kDirs) {
      const int64_t src = c - direction_offset(d, nk);
      if (src >= 0 && src < ncell) {
        const int go = cidx_old[src];
        if (go >= 0 && go < nocc_old && occ_old[go] == (int32_t)src) {
          gs = go;
          len = dir_cnt[(size_t)go * kDirs + d];
        }
      }
    }
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int start = bnd_new[g];
    if (len > 0) dir_base[(size_t)gs * kDirs + d] = start + incl - len;
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    bad |= total != bnd_new[g + 1] - start;
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&dsc->sort_far, 2);
}

// C: one warp per item, slots in order, a running rank per direction from
// the group's first slot, the item's prefix within its cell: perm[rank] = s.
// The item's old cell code and slots come from the last sort's item records,
// its old occupied index from the item's cell (two independent loads).
__global__ void __launch_bounds__(kNearThreads) k_near_place(const int32_t* __restrict__ item_old,
                                                            const int4* __restrict__ rec_old,
                                                            const DeviceScalars* dsc, int par_old,
                                                            const uint32_t* __restrict__ keys, int nk,
                                                            const int32_t* __restrict__ item_dir,
                                                            const int32_t* __restrict__ dir_base,
                                                            uint32_t* __restrict__ perm) {
  if (dsc->sort_far) return;
  __shared__ int32_t run[kNearThreads / 32][kDirs];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nitems = dsc->nitems_par[par_old];
  const int warps = gridDim.x * (kNearThreads / 32);
  for (int item = blockIdx.x * (kNearThreads / 32) + w; item < nitems; item += warps) {
    const int g = item_old[item];
    const int4 rec = rec_old[item];
    if (lane < kDirs)
      run[w][lane] = dir_base[(size_t)g * kDirs + lane] + item_dir[(size_t)item * kDirs + lane];
    __syncwarp();
    const int64_t o = rec.x;
    const int s0 = rec.y, s1 = rec.z;
    for (int base = s0; base < s1; base += 32 * kNearKeys) {
      uint32_t kv[kNearKeys];  // the keys of up to 32 kNearKeys slots, all loads in flight
#pragma unroll
      for (int u = 0; u < kNearKeys; ++u) {
        const int s = base + 32 * u + lane;
        kv[u] = s < s1 ? keys[s] : 0u;
      }
#pragma unroll
      for (int u = 0; u < kNearKeys; ++u) {  // slot order: the ranks follow it
        const int s = base + 32 * u + lane;
        const bool valid = s < s1;
        const unsigned m = __ballot_sync(0xffffffffu, valid);
        if (m == 0) break;
        if (valid) {
          const int d = direction_of((int64_t)kv[u] - o, nk);  // >= 0: A found no far particle
          const unsigned peers = __match_any_sync(m, d);
          const int leader = __ffs(peers) - 1;
          const int r0 = run[w][d];
          perm[r0 + __popc(peers & lanemask_lt())] = (uint32_t)s;
          __syncwarp(m);
          if (lane == leader) run[w][d] = r0 + __popc(peers);
        }
        __syncwarp();
      }
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------- the move
// What the move needs to write each slot's packed deposit columns (cols null:
// none).
struct DepCols {
  uint32_t* cols = nullptr;
  float x0 = 0, h = 0, lo = 0, hi = 0, spacing = 0;
  int nbdt = 0, ncol = 0;
};

// Moves the records into slot order: dst[s] = src[perm[s]], the position
// arrays (k, delta) when kPos, the previous positions (pk, pdelta) when
// kPrev.  Four consecutive slots per thread: one 16-byte load of their
// permutation entries, the gathered loads all in flight, then one 16-byte
// store per component array (Npad is a multiple of 64).  Reads follow the
// permutation of a nearly sorted cloud, so they stay within a few pages.
// A step whose push follows leaves (pk, pdelta) where they are: the push
// reads them through the permutation and writes them in slot order.  With
// dc.cols set the move also writes each slot's packed deposit columns and
// window flag (deposit_cols of the moved k and delta), so that the fine
// deposit reads four bytes a particle instead of 24.
template <bool kPos, bool kPrev>
__global__ void __launch_bounds__(256) k_gather_records(int64_t N, int64_t Npad, const uint32_t* __restrict__ perm,
                                                        const int32_t* __restrict__ k0, const float* __restrict__ d0,
                                                        const int32_t* __restrict__ pk0, const float* __restrict__ pd0,
                                                        int32_t* __restrict__ k1, float* __restrict__ d1,
                                                        int32_t* __restrict__ pk1, float* __restrict__ pd1,
                                                        const DepCols dc = DepCols{}) {
  const int64_t nq = N / 4;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = 4 * q;
    const uint4 pv = *reinterpret_cast<const uint4*>(perm + s);
    const int64_t i[4] = {pv.x, pv.y, pv.z, pv.w};
    int kv[3][4], pkv[3][4];
    float dv[3][4], pdv[3][4];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (kPos) {
          kv[c][u] = __ldg(k0 + c * Npad + i[u]);
          dv[c][u] = __ldg(d0 + c * Npad + i[u]);
        }
        if (kPrev) {
          pkv[c][u] = __ldg(pk0 + c * Npad + i[u]);
          pdv[c][u] = __ldg(pd0 + c * Npad + i[u]);
        }
      }
    if (kPos && dc.cols) {
      uint32_t cv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        cv[u] = deposit_cols(kv[0][u], kv[1][u], kv[2][u], dv[0][u], dv[1][u], dv[2][u], dc.x0, dc.h, dc.lo, dc.hi,
                             dc.spacing, dc.nbdt, dc.ncol);
      *reinterpret_cast<uint4*>(dc.cols + s) = make_uint4(cv[0], cv[1], cv[2], cv[3]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (kPos) {
        *reinterpret_cast<int4*>(k1 + c * Npad + s) = make_int4(kv[c][0], kv[c][1], kv[c][2], kv[c][3]);
        *reinterpret_cast<float4*>(d1 + c * Npad + s) = make_float4(dv[c][0], dv[c][1], dv[c][2], dv[c][3]);
      }
      if (kPrev) {
        *reinterpret_cast<int4*>(pk1 + c * Npad + s) = make_int4(pkv[c][0], pkv[c][1], pkv[c][2], pkv[c][3]);
        *reinterpret_cast<float4*>(pd1 + c * Npad + s) = make_float4(pdv[c][0], pdv[c][1], pdv[c][2], pdv[c][3]);
      }
    }
  }
  // the last N mod 4 slots
  for (int64_t s = 4 * nq + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = perm[s];
    if (kPos && dc.cols)
      dc.cols[s] = deposit_cols(k0[i], k0[Npad + i], k0[2 * Npad + i], d0[i], d0[Npad + i], d0[2 * Npad + i], dc.x0,
                                dc.h, dc.lo, dc.hi, dc.spacing, dc.nbdt, dc.ncol);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (kPos) {
        k1[c * Npad + s] = k0[c * Npad + i];
        d1[c * Npad + s] = d0[c * Npad + i];
      }
      if (kPrev) {
        pk1[c * Npad + s] = pk0[c * Npad + i];
        pd1[c * Npad + s] = pd0[c * Npad + i];
      }
    }
  }
}

}  // namespace

int grid_for(const Ctx& c, int64_t n, int threads, int per_sm) {
  int64_t want = (n + threads - 1) / threads;
  int64_t cap = (int64_t)c.num_sms * per_sm;
  return (int)std::max<int64_t>(1, std::min(want, cap));
}

// The previous positions of a sort that deferred their move, into slot
// order (before anything else reads them).
void settle_prev(Ctx& c) {
  if (!c.prev_deferred) return;
  const Particles& P = c.part[c.cur ^ 1];
  const Particles& Q = c.part[c.cur];
  k_gather_records<false, true><<<grid_for(c, (c.N + 3) / 4, 256, c.move_cps), 256, 0, c.stream>>>(
      c.N, c.Npad, c.perm, P.k, P.d, P.pk, P.pd, Q.k, Q.d, Q.pk, Q.pd);
  VLB_LAUNCHED(c);
  c.prev_deferred = false;
}

// The LSD radix passes over the cell keys (2 or 3 passes of up to 10 bits)
// into perm, on `s`, gated on `gate` when it is set; returns the launches.
long long radix_passes(Ctx& c, cudaStream_t s, const int32_t* gate) {
  const long long before = c.launches;
  const int64_t N = c.N;
  int bits = 1;
  while ((1ll << bits) < (long long)c.ncell) ++bits;
  int passes = (bits + kMaxDigitBits - 1) / kMaxDigitBits;
  if (passes > 3) throw ArgError("too many cells for the radix sort");
  const int64_t ntiles = (N + kRadixTile - 1) / kRadixTile;
  int shift = 0;
  const uint32_t* kin = c.keys;
  const uint32_t* vin = nullptr;
  for (int p = 0; p < passes; ++p) {
    int b = (bits - shift + (passes - p) - 1) / (passes - p);  // spread the bits evenly
    uint32_t mask = (1u << b) - 1u;
    bool last = p == passes - 1;
    uint32_t* kout = last ? c.skeys : (p % 2 == 0 ? c.keys_alt : c.keys);
    uint32_t* vout = ((passes - 1 - p) % 2 == 0) ? c.perm : c.vals_alt;
    k_radix_upsweep<<<(unsigned)ntiles, kRadixThreads, 0, s>>>(kin, N, shift, mask, c.radix_table, ntiles, gate);
    VLB_LAUNCHED(c);
    scan(c, ScanInArray{c.radix_table}, ScanOutArray{c.radix_table}, (int64_t)(mask + 1) * ntiles, 2 + p, nullptr,
         gate, s);
    k_radix_downsweep<<<(unsigned)ntiles, kRadixThreads, 0, s>>>(kin, vin, kout, vout, N, shift, mask,
                                                                c.radix_table, ntiles, gate);
    VLB_LAUNCHED(c);
    kin = kout;
    vin = vout;
    shift += b;
  }
  return c.launches - before;
}

void launch_sort(Ctx& c, bool defer_prev) {
  settle_prev(c);
  const int64_t N = c.N;
  const int nk = c.fine.nk, n = c.fine.n;
  Particles& P = c.part[c.cur];
  Particles& Q = c.part[c.cur ^ 1];
  // the products of the last sort describe part[cur]'s order (parity po);
  // this sort writes parity pn, which describes part[cur ^ 1]
  const int po = c.cur, pn = c.cur ^ 1;
  const bool near = c.keys_ready && c.order_valid;
  c.occupied = c.occ_buf[pn];
  c.bounds = c.bnd_buf[pn];
  c.item_cell = c.item_buf[pn];
  c.item_rec = c.rec_buf[pn];
  c.chunk_start = c.cstart_buf[pn];
  c.chunk_par[pn] = c.chunk;
  VLB_CUDA(cudaMemsetAsync(c.scan_status, 0, c.scan_status_size * sizeof(unsigned long long), c.stream));
  VLB_CUDA(cudaMemsetAsync(c.dsc->scan_tiles, 0, sizeof(c.dsc->scan_tiles), c.stream));
  if (!c.keys_ready) {
    VLB_CUDA(cudaMemsetAsync(c.counts, 0, sizeof(int32_t) * c.ncell, c.stream));
    k_keys_hist<<<grid_for(c, N, 256, 8), 256, 0, c.stream>>>(N, c.Npad, P.k, nk, c.keys, c.counts);
    VLB_LAUNCHED(c);
  }
  // the occupied cells, then their bounds, work items and out-of-stencil
  // slots (cell_off holds the out-of-stencil start of each occupied cell)
  scan(c, ScanInOccupied{c.counts}, ScanOutOccupied{c.occupied, c.cidx_buf[pn]}, c.ncell, 1, &c.dsc->noccupied);
  k_cell_lists<<<1, kListThreads, 0, c.stream>>>(c.counts, c.occupied, c.dsc, nk, n, c.bounds, c.chunk_start,
                                                 c.cell_off, c.chunk, pn);
  VLB_LAUNCHED(c);
  k_expand_lists<<<c.num_sms * 4, 256, 0, c.stream>>>(c.occupied, c.bounds, c.chunk_start, c.cell_off, c.dsc,
                                                      c.item_cell, c.item_rec, c.outlist, c.chunk, c.fine.nk);
  VLB_LAUNCHED(c);
  // the histogram is spent: zero it for the push that may refill it
  VLB_CUDA(cudaMemsetAsync(c.counts, 0, sizeof(int32_t) * c.ncell, c.stream));
  c.keys_ready = false;
  const int32_t* gate = nullptr;
  if (near) {
    const int grid = c.num_sms * 8;
    k_near_count<<<grid, kNearThreads, 0, c.stream>>>(c.rec_buf[po], c.dsc, po, c.keys, nk, c.item_dir);
    VLB_LAUNCHED(c);
    k_near_prefix<<<grid, kNearThreads, 0, c.stream>>>(c.cstart_buf[po], c.dsc, po, c.item_dir, c.dir_cnt);
    VLB_LAUNCHED(c);
    k_near_bases<<<grid, kNearThreads, 0, c.stream>>>(c.occupied, c.bounds, c.occ_buf[po], c.cidx_buf[po], c.dsc,
                                                      po, c.ncell, nk, c.dir_cnt, c.dir_base);
    VLB_LAUNCHED(c);
    k_near_place<<<grid, kNearThreads, 0, c.stream>>>(c.item_buf[po], c.rec_buf[po], c.dsc, po, c.keys, nk,
                                                      c.item_dir, c.dir_base, c.perm);
    VLB_LAUNCHED(c);
    gate = &c.dsc->sort_far;  // the radix passes below run only if that path gave up
  }
  // the radix passes: gated on the fallback flag after the single-pass
  // placement (they launch and return at once unless it is set).  A
  // conditional graph node around them was measured: the node cost a replayed
  // step more (1.959 against 1.900 ms at 8e6) than the gated launches do.
  radix_passes(c, c.stream, gate);
  const int mgrid = grid_for(c, (N + 3) / 4, 256, c.move_cps);
  DepCols dc;
  if (c.cols_packed) {
    dc.cols = c.cols;
    dc.x0 = c.x0f;
    dc.h = c.hf;
    dc.lo = c.lo_f;
    dc.hi = c.hi_f;
    dc.spacing = c.spacing_f;
    dc.nbdt = c.nbdt;
    dc.ncol = c.ncol;
  }
  if (defer_prev)
    k_gather_records<true, false><<<mgrid, 256, 0, c.stream>>>(N, c.Npad, c.perm, P.k, P.d, P.pk, P.pd, Q.k, Q.d,
                                                               Q.pk, Q.pd, dc);
  else
    k_gather_records<true, true><<<mgrid, 256, 0, c.stream>>>(N, c.Npad, c.perm, P.k, P.d, P.pk, P.pd, Q.k, Q.d,
                                                              Q.pk, Q.pd, dc);
  VLB_LAUNCHED(c);
  c.prev_deferred = defer_prev;
  c.cur ^= 1;
  c.sorted = true;
  c.items_valid = true;
  c.order_valid = true;
  c.last_sort_near = near;
}

}  // namespace vlb
