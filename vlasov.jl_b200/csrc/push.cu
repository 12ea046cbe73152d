// Time integration: the packed position Verlet of the cloud
// (src/kernels.jl:985-1025, src/particles.jl:337-349), the projectile's step
// (src/accelerator.jl:746-756, src/projectile.jl:298-304), and the capture
// diagnostic q(<R) (src/projectile.jl:243-247).
//
// The Verlet update of (k, delta) is the reference's Float32 arithmetic
// operation for operation, so the integer cell updates and the offsets are
// bit-identical to it for identical inputs:
//
//     kn = 2k - pk;  dn = (2 delta - pdelta) + a f;  m = round(dn / h)
//     k' = kn + m;   delta' = dn - m h;   gap = (k' - pk) h + (delta' - pdelta)
//
// The three diagnostics (kinetic energy, the part beyond rcmax, angular
// momentum) are reduced per CTA in float64.

#include "vlb_internal.cuh"

namespace vlb {

int grid_for(const Ctx& c, int64_t n, int threads, int per_sm);

namespace {

__device__ __forceinline__ void verlet1(int kq, float dq, int ok, float od, float a, float f, float h, int& kn,
                                        float& dn, float& gap) {
  kn = 2 * kq - ok;
  dn = fadd(fsub(fmul(2.f, dq), od), fmul(a, f));
  const int m = __float2int_rn(fdiv(dn, h));
  kn += m;
  dn = fsub(dn, fmul((float)m, h));
  gap = fadd(fmul((float)(kn - ok), h), fsub(dn, od));
}

__global__ void __launch_bounds__(256) k_push(int64_t N, int64_t Npad, int32_t* __restrict__ k, float* __restrict__ d,
                                              int32_t* __restrict__ pk, float* __restrict__ pd,
                                              const float* __restrict__ force, float a, float h, float x0, float pfac,
                                              float r2max, float inv2M, double* diag) {
  double ek = 0, eo = 0, lx = 0, ly = 0, lz = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    int kq[3], ko[3], kn[3];
    float dq[3], od[3], dn[3], gap[3], q[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      kq[c] = k[c * Npad + i];
      dq[c] = d[c * Npad + i];
      ko[c] = pk[c * Npad + i];
      od[c] = pd[c * Npad + i];
      verlet1(kq[c], dq[c], ko[c], od[c], a, force[c * Npad + i], h, kn[c], dn[c], gap[c]);
      q[c] = fadd(fadd(x0, fmul((float)(kq[c] - 1), h)), dq[c]);
    }
    const float px = fmul(gap[0], pfac), py = fmul(gap[1], pfac), pz = fmul(gap[2], pfac);
    const float e = fmul(fadd(fadd(fmul(px, px), fmul(py, py)), fmul(pz, pz)), inv2M);
    ek += e;
    const float r2 = fadd(fadd(fmul(q[0], q[0]), fmul(q[1], q[1])), fmul(q[2], q[2]));
    if (r2 > r2max) eo += e;
    lx += (double)fsub(fmul(q[1], pz), fmul(q[2], py));
    ly += (double)fsub(fmul(q[2], px), fmul(q[0], pz));
    lz += (double)fsub(fmul(q[0], py), fmul(q[1], px));
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      k[c * Npad + i] = kn[c];
      d[c * Npad + i] = dn[c];
      pk[c * Npad + i] = kq[c];
      pd[c * Npad + i] = dq[c];
    }
  }
  __shared__ double sh[5][8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double v[5] = {ek, eo, lx, ly, lz};
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    v[c] = warp_sum(v[c]);
    if (lane == 0) sh[c][w] = v[c];
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double s = 0;
    for (int ww = 0; ww < (int)(blockDim.x / 32); ++ww) s += sh[threadIdx.x][ww];
    atomicAdd(&diag[threadIdx.x], s);
  }
}

// projectile_forces!(cloud, acc, proj, jel) then step!(proj, F, dt)
__global__ void k_projectile(DeviceScalars* dsc, double w, double dt, double nions, double jrad, int advance) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double* P = dsc->proj_pos;
  const double q = dsc->proj_charge;
  const double r2 = P[0] * P[0] + P[1] * P[1] + P[2] * P[2];
  const double modf = r2 > jrad * jrad ? nions * q / pow(r2, 1.5) : q / 64.0;  // rs^3 = 4^3
  double F[3];
  for (int c = 0; c < 3; ++c) {
    F[c] = modf * P[c] + dsc->red[c];
    dsc->proj_force[c] = F[c];
  }
  dsc->e_el = w * q * dsc->red[3];
  const double r = sqrt(r2);
  dsc->e_jel = q * (r < jrad ? -nions * (3 - (r / jrad) * (r / jrad)) / (2 * jrad) : -nions / r);
  if (advance && dsc->proj_active) {
    const double M = dsc->proj_mass;
    for (int c = 0; c < 3; ++c) {
      const double nw = 2 * dsc->proj_pos[c] - dsc->proj_prev[c] + (dt * dt / M) * F[c];
      dsc->proj_vel[c] = (nw - dsc->proj_prev[c]) / (2 * dt);
      dsc->proj_prev[c] = dsc->proj_pos[c];
      dsc->proj_pos[c] = nw;
    }
  }
}

// particles within `radius` of the projectile (float64 positions)
__global__ void __launch_bounds__(256) k_enclosed(int64_t N, int64_t Npad, const int32_t* __restrict__ k,
                                                  const float* __restrict__ d, double x0, double h, double r2,
                                                  DeviceScalars* dsc) {
  const double P0 = dsc->proj_pos[0], P1 = dsc->proj_pos[1], P2 = dsc->proj_pos[2];
  unsigned long long cnt = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    const double px = x0 + (double)(k[i] - 1) * h + (double)d[i] - P0;
    const double py = x0 + (double)(k[Npad + i] - 1) * h + (double)d[Npad + i] - P1;
    const double pz = x0 + (double)(k[2 * Npad + i] - 1) * h + (double)d[2 * Npad + i] - P2;
    if (px * px + py * py + pz * pz < r2) ++cnt;
  }
  cnt = __reduce_add_sync(0xffffffffu, (unsigned)cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&dsc->enclosed, cnt);
}

// Long chains of independent FMAs: the FP32 pipe's ceiling at the current
// clocks, the denominator of the gather's and deposit's roofline.
__global__ void __launch_bounds__(256) k_fma_peak(float* out, int iters, float a, float b) {
  float x[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) x[j] = threadIdx.x * 1e-7f + j;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 16; ++r)
#pragma unroll
      for (int j = 0; j < 8; ++j) x[j] = fmaf(x[j], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += x[j];
  if (s == 1234.5f) out[blockIdx.x] = s;  // keeps the chains alive
}

}  // namespace

double measure_fp32_peak(int device) {
  VLB_CUDA(cudaSetDevice(device));
  int sms = 0;
  VLB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  float* out = nullptr;
  VLB_CUDA(cudaMalloc(&out, sizeof(float) * sms * 8));
  cudaEvent_t e0, e1;
  VLB_CUDA(cudaEventCreate(&e0));
  VLB_CUDA(cudaEventCreate(&e1));
  const int iters = 4096, blocks = sms * 8, threads = 256;
  k_fma_peak<<<blocks, threads>>>(out, iters / 8, 0.999f, 1e-3f);  // warm-up
  VLB_CUDA(cudaEventRecord(e0));
  k_fma_peak<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
  VLB_CUDA(cudaEventRecord(e1));
  VLB_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  VLB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  const double flops = 2.0 * 16 * 8 * (double)iters * blocks * threads;
  return flops / (ms * 1e-3) / 1e12;
}

void launch_push(Ctx& c, double dt, double rcmax) {
  Particles& P = c.part[c.cur];
  const double M = c.weight;  // ELECTRON_MASS * weight
  VLB_CUDA(cudaMemsetAsync(c.dsc->diag, 0, sizeof(c.dsc->diag), c.stream));
  k_push<<<grid_for(c, c.N, 256, 8), 256, 0, c.stream>>>(
      c.N, c.Npad, P.k, P.d, P.pk, P.pd, c.force, (float)(dt * dt / M), c.hf, c.x0f, (float)(M / (2 * dt)),
      (float)(rcmax * rcmax), (float)(1 / (2 * M)), c.dsc->diag);
  VLB_LAUNCHED(c);
}

void launch_projectile_update(Ctx& c, double dt, double nions, double jradius, int advance) {
  k_projectile<<<1, 32, 0, c.stream>>>(c.dsc, c.weight, dt, nions, jradius, advance);
  VLB_LAUNCHED(c);
}

void launch_projectile_force_only(Ctx& c, double nions, double jradius) {
  k_projectile<<<1, 32, 0, c.stream>>>(c.dsc, c.weight, 0.0, nions, jradius, 0);
  VLB_LAUNCHED(c);
}

void launch_enclosed(Ctx& c, double radius) {
  Particles& P = c.part[c.cur];
  VLB_CUDA(cudaMemsetAsync(&c.dsc->enclosed, 0, sizeof(unsigned long long), c.stream));
  k_enclosed<<<grid_for(c, c.N, 256, 8), 256, 0, c.stream>>>(c.N, c.Npad, P.k, P.d, c.x0, c.h, radius * radius,
                                                             c.dsc);
  VLB_LAUNCHED(c);
}

}  // namespace vlb
