// A total-charge reduction for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc when they need a
// result:
//   - an embedding runtime (a Julia or Python host with its own caching
//     allocator) whose pool has already claimed the GPU's memory, so a fresh
//     cudaMalloc fails or fragments it;
//   - a plugin whose host forbids allocation outside its set-up phase;
//   - a loop that must not stall, since cudaMalloc can synchronise the device.
//
// vlb_total_charge_noalloc serves them.  It computes sum rho m0x m0y m0z over
// a density the caller already holds on the device; the reduction is the one
// the fine deposit uses before its renormalisation, same operations in the
// same order.  Its only scratch is one float64 partial per (j, k) column.
// That scratch lives in the file-scope array below, a fixed 512 KiB that
// every GPU which loads the library keeps until the process exits.  Grids
// are limited to kNoAllocMaxN points per axis.
//
// The array's name in host code is a host-side stand-in, not a device
// address: a kernel handed it would fault, or silently use the wrong memory
// where the GPU can reach host memory.  So the first call on each device,
// with that device current, asks the runtime for the array's device address
// (cudaGetSymbolAddress) and caches it; the kernels receive that address.
// Make that first call before any stream capture.  The cached address is
// only good while the device's context lives: a device reset, or a primary
// context torn down and recreated between calls, is not supported.
//
// All calls share the one array, which keeps the last call's contents.
// Nothing in it must start at zero: every call writes all the n*n partials
// it then reads.  Calls that overlap on the GPU -- on two streams, or from
// two threads without ordering -- race on the array; issue them on one
// stream or wait between them.

#include <mutex>
#include <string>

#include "vlb_internal.cuh"

namespace vlb {
namespace {

constexpr int kNoAllocMaxN = 256;  // points per axis
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxN * kNoAllocMaxN];

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Per (j,k) column: sum_i rho[i,j,k] m0[i], times m0[j] m0[k].  One warp
// per column: lane l sums i = l, l+32, ... in order, then the fixed
// butterfly over the lanes.
__global__ void __launch_bounds__(256) k_noalloc_columns(const float* __restrict__ rho, const double* __restrict__ m0,
                                                         int n, double* __restrict__ partial) {
  const int t = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (t >= n * n) return;
  const int j = t % n, k = t / n;
  double s = 0;
  for (int i = lane; i < n; i += 32) s += (double)rho[(size_t)t * n + i] * m0[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) partial[t] = s * m0[j] * m0[k];
}

// One block: the fixed-order sum of the column partials.
__global__ void __launch_bounds__(1024) k_noalloc_total(const double* __restrict__ partial, int m, double* out) {
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

int noalloc_fail(int code, const std::string& msg) {
  set_last_error(msg);  // read back through vlb_last_error()
  return code;
}

}  // namespace
}  // namespace vlb

using namespace vlb;

extern "C" int vlb_total_charge_noalloc(const float* rho, const double* m0, int32_t n, double* q, void* stream) {
  if (!rho || !m0 || !q)
    return noalloc_fail(VLB_ERR_ARG, "vlb_total_charge_noalloc: null device pointer");
  if (n < 1 || n > kNoAllocMaxN)
    return noalloc_fail(VLB_ERR_ARG, "vlb_total_charge_noalloc: n = " + std::to_string(n) +
                                         " points per axis; the static scratch holds at most " +
                                         std::to_string(kNoAllocMaxN));
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(VLB_ERR_CUDA, cuda_msg(e, "cudaGetDevice"));
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return noalloc_fail(VLB_ERR_ARG, "vlb_total_charge_noalloc: device ordinal out of range");
  double* partials = nullptr;
  {
    // set-up, once per device, with that device current
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_partials);
      if (e != cudaSuccess) return noalloc_fail(VLB_ERR_CUDA, cuda_msg(e, "cudaGetSymbolAddress"));
      g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    partials = g_noalloc_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int cols = n * n;
  k_noalloc_columns<<<(cols + 7) / 8, 256, 0, s>>>(rho, m0, n, partials);
  k_noalloc_total<<<1, 1024, 0, s>>>(partials, cols, q);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(VLB_ERR_CUDA, cuda_msg(e, "vlb_total_charge_noalloc launch"));
  return VLB_OK;
}
