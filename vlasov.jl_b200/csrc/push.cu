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

// Four consecutive particles per thread, 16-byte loads and stores of every
// component array (Npad is a multiple of 64).  With kGathered the previous
// positions are read from (pk_src, pd_src) at perm[slot] -- where the step's
// sort left them -- and written in slot order like the rest; otherwise they
// are read in place.  When `r2cap` > 0 the same pass
// counts the particles within sqrt(r2cap) of the projectile after the step
// (enclosed_charge, float64 positions), which the reference reads after
// step! on the host.  When `keys` is set it also writes the cell key of
// every new position and adds it to the cell histogram (zero on entry) --
// the first stage of the next step's sort, done while the positions are in
// registers.
template <bool kGathered>
__global__ void __launch_bounds__(256) k_push(int64_t N, int64_t Npad, int32_t* __restrict__ k, float* __restrict__ d,
                                              int32_t* __restrict__ pk, float* __restrict__ pd,
                                              const int32_t* __restrict__ pk_src, const float* __restrict__ pd_src,
                                              const uint32_t* __restrict__ perm,
                                              const float* __restrict__ force, float a, float h, float x0, float pfac,
                                              float r2max, float inv2M, double* diag, double r2cap, double x0d,
                                              double hd, DeviceScalars* dsc, uint32_t* __restrict__ keys,
                                              int32_t* __restrict__ counts, int nk) {
  double ek = 0, eo = 0, lx = 0, ly = 0, lz = 0;
  unsigned cnt = 0;
  const double P0 = dsc->proj_pos[0], P1 = dsc->proj_pos[1], P2 = dsc->proj_pos[2];
  const int64_t nq = (N + 3) / 4;
  for (int64_t qi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; qi < nq; qi += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i0 = 4 * qi;
    int kq[3][4], ko[3][4], kn[3][4];
    float dq[3][4], od[3][4], dn[3][4], gap[3][4], ff[3][4];
    int64_t src[4] = {0, 0, 0, 0};
    if (kGathered) {
      if (i0 + 3 < N) {
        const uint4 pv = *reinterpret_cast<const uint4*>(perm + i0);
        src[0] = pv.x; src[1] = pv.y; src[2] = pv.z; src[3] = pv.w;
      } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) src[u] = i0 + u < N ? (int64_t)perm[i0 + u] : 0;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int4 a4 = *reinterpret_cast<const int4*>(k + c * Npad + i0);
      const float4 b4 = *reinterpret_cast<const float4*>(d + c * Npad + i0);
      const float4 f4 = *reinterpret_cast<const float4*>(force + c * Npad + i0);
      kq[c][0] = a4.x; kq[c][1] = a4.y; kq[c][2] = a4.z; kq[c][3] = a4.w;
      dq[c][0] = b4.x; dq[c][1] = b4.y; dq[c][2] = b4.z; dq[c][3] = b4.w;
      ff[c][0] = f4.x; ff[c][1] = f4.y; ff[c][2] = f4.z; ff[c][3] = f4.w;
      if (kGathered) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          // padding slots past N: any value (their result is not kept)
          ko[c][u] = i0 + u < N ? __ldg(pk_src + c * Npad + src[u]) : kq[c][u];
          od[c][u] = i0 + u < N ? __ldg(pd_src + c * Npad + src[u]) : dq[c][u];
        }
      } else {
        const int4 c4 = *reinterpret_cast<const int4*>(pk + c * Npad + i0);
        const float4 d4 = *reinterpret_cast<const float4*>(pd + c * Npad + i0);
        ko[c][0] = c4.x; ko[c][1] = c4.y; ko[c][2] = c4.z; ko[c][3] = c4.w;
        od[c][0] = d4.x; od[c][1] = d4.y; od[c][2] = d4.z; od[c][3] = d4.w;
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      float q[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        verlet1(kq[c][u], dq[c][u], ko[c][u], od[c][u], a, ff[c][u], h, kn[c][u], dn[c][u], gap[c][u]);
        q[c] = fadd(fadd(x0, fmul((float)(kq[c][u] - 1), h)), dq[c][u]);
      }
      if (i0 + u < N) {
        const float px = fmul(gap[0][u], pfac), py = fmul(gap[1][u], pfac), pz = fmul(gap[2][u], pfac);
        const float e = fmul(fadd(fadd(fmul(px, px), fmul(py, py)), fmul(pz, pz)), inv2M);
        ek += e;
        const float r2 = fadd(fadd(fmul(q[0], q[0]), fmul(q[1], q[1])), fmul(q[2], q[2]));
        if (r2 > r2max) eo += e;
        lx += (double)fsub(fmul(q[1], pz), fmul(q[2], py));
        ly += (double)fsub(fmul(q[2], px), fmul(q[0], pz));
        lz += (double)fsub(fmul(q[0], py), fmul(q[1], px));
        if (r2cap > 0) {
          const double ex = x0d + (double)(kn[0][u] - 1) * hd + (double)dn[0][u] - P0;
          const double ey = x0d + (double)(kn[1][u] - 1) * hd + (double)dn[1][u] - P1;
          const double ez = x0d + (double)(kn[2][u] - 1) * hd + (double)dn[2][u] - P2;
          if (ex * ex + ey * ey + ez * ez < r2cap) ++cnt;
        }
      } else {
        // padding slots past N keep their (unused) contents
#pragma unroll
        for (int c = 0; c < 3; ++c) { kn[c][u] = kq[c][u]; dn[c][u] = dq[c][u]; }
      }
    }
    if (keys) {
      // warp-aggregated histogram: the cloud is sorted, so lanes mostly share
      // cells; one atomic per group of equal keys for each of the 4 slots
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const bool valid = i0 + u < N;
        const unsigned m = __ballot_sync(__activemask(), valid);
        if (valid) {
          const uint32_t key = cell_key(kn[0][u], kn[1][u], kn[2][u], nk);
          keys[i0 + u] = key;
          const unsigned peers = __match_any_sync(m, key);
          if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&counts[key], __popc(peers));
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (i0 + 3 < N) {
        *reinterpret_cast<int4*>(k + c * Npad + i0) = make_int4(kn[c][0], kn[c][1], kn[c][2], kn[c][3]);
        *reinterpret_cast<float4*>(d + c * Npad + i0) = make_float4(dn[c][0], dn[c][1], dn[c][2], dn[c][3]);
        *reinterpret_cast<int4*>(pk + c * Npad + i0) = make_int4(kq[c][0], kq[c][1], kq[c][2], kq[c][3]);
        *reinterpret_cast<float4*>(pd + c * Npad + i0) = make_float4(dq[c][0], dq[c][1], dq[c][2], dq[c][3]);
      } else {
        for (int u = 0; u < 4 && i0 + u < N; ++u) {
          k[c * Npad + i0 + u] = kn[c][u];
          d[c * Npad + i0 + u] = dn[c][u];
          pk[c * Npad + i0 + u] = kq[c][u];
          pd[c * Npad + i0 + u] = dq[c][u];
        }
      }
    }
  }
  __shared__ double sh[5][8];
  __shared__ unsigned shc[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double v[5] = {ek, eo, lx, ly, lz};
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    v[c] = warp_sum(v[c]);
    if (lane == 0) sh[c][w] = v[c];
  }
  cnt = __reduce_add_sync(0xffffffffu, cnt);
  if (lane == 0) shc[w] = cnt;
  __syncthreads();
  if (threadIdx.x < 5) {
    double s = 0;
    for (int ww = 0; ww < (int)(blockDim.x / 32); ++ww) s += sh[threadIdx.x][ww];
    diag[5 * blockIdx.x + threadIdx.x] = s;  // this CTA's partial, summed in order by k_diag_total
  } else if (threadIdx.x == 5 && r2cap > 0) {
    unsigned long long s = 0;
    for (int ww = 0; ww < (int)(blockDim.x / 32); ++ww) s += shc[ww];
    if (s) atomicAdd(&dsc->enclosed, s);
  }
}

// diag[c] = the CTA partials of k_push in CTA order (a fixed order: the
// push's grid-stride split of the particles is static).
__global__ void __launch_bounds__(256) k_diag_total(const double* __restrict__ part, int nb, double* diag) {
  __shared__ double sh[5][256];
  const int t = threadIdx.x;
  double s[5] = {0, 0, 0, 0, 0};
  for (int b = t; b < nb; b += blockDim.x)
#pragma unroll
    for (int c = 0; c < 5; ++c) s[c] += part[5 * b + c];
#pragma unroll
  for (int c = 0; c < 5; ++c) sh[c][t] = s[c];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (t < o)
#pragma unroll
      for (int c = 0; c < 5; ++c) sh[c][t] += sh[c][t + o];
    __syncthreads();
  }
  if (t < 5) diag[t] = sh[t][0];
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

// ---- the film: what scripts/xenon.jl:396-410 reads back for a frame of its
// movie, kept on the device.  Each kernel returns at once unless the step
// asked for a frame (film_due, uploaded with the projectile), so the three
// stay in a captured step.  Frame f = film_next: the fine density's plane
// average Float32.((rho[:, :, iz1] + rho[:, :, iz2]) ./ 2), then four
// float64 scalars: the projectile's x and y after its step, the step's count
// within the capture radius of it (enclosed_charge, src/projectile.jl:243),
// and the count within the film radius of the origin (the script's net
// charge, 196 - w #{|r| < 35}).  Frames past the capacity are counted, not
// stored.
__global__ void __launch_bounds__(256) k_film_slice(const float* __restrict__ rho, int n, int iz1, int iz2,
                                                    float* __restrict__ frames, int cap,
                                                    const DeviceScalars* __restrict__ dsc) {
  if (!dsc->film_due) return;
  const int f = dsc->film_next;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= cap || t >= n * n) return;
  const size_t nn = (size_t)n * n;
  frames[(size_t)f * nn + t] = __fmul_rn(__fadd_rn(rho[(size_t)iz1 * nn + t], rho[(size_t)iz2 * nn + t]), 0.5f);
}

// Particles within sqrt(r2) of the origin, float64 positions as k_enclosed.
__global__ void __launch_bounds__(256) k_film_count(int64_t N, int64_t Npad, const int32_t* __restrict__ k,
                                                    const float* __restrict__ d, double x0, double h, double r2,
                                                    DeviceScalars* dsc) {
  if (!dsc->film_due) return;
  unsigned long long cnt = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    const double px = x0 + (double)(k[i] - 1) * h + (double)d[i];
    const double py = x0 + (double)(k[Npad + i] - 1) * h + (double)d[Npad + i];
    const double pz = x0 + (double)(k[2 * Npad + i] - 1) * h + (double)d[2 * Npad + i];
    if (px * px + py * py + pz * pz < r2) ++cnt;
  }
  cnt = __reduce_add_sync(0xffffffffu, (unsigned)cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&dsc->film_inside, cnt);
}

__global__ void k_film_finish(double* __restrict__ scalars, int cap, int have_capture, DeviceScalars* dsc) {
  if (!dsc->film_due) return;
  const int f = dsc->film_next;
  if (f < cap) {
    scalars[4 * (size_t)f + 0] = dsc->proj_pos[0];
    scalars[4 * (size_t)f + 1] = dsc->proj_pos[1];
    scalars[4 * (size_t)f + 2] = have_capture ? (double)dsc->enclosed : 0.0;
    scalars[4 * (size_t)f + 3] = (double)dsc->film_inside;
  }
  dsc->film_next = f + 1;
  dsc->film_inside = 0;
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

void launch_push(Ctx& c, double dt, double rcmax, double capture_radius, bool keys) {
  Particles& P = c.part[c.cur];
  const double M = c.weight;  // ELECTRON_MASS * weight
  if (capture_radius > 0) VLB_CUDA(cudaMemsetAsync(&c.dsc->enclosed, 0, sizeof(unsigned long long), c.stream));
  const int grid = grid_for(c, (c.N + 3) / 4, 256, c.push_cps);
  const Particles& O = c.part[c.cur ^ 1];  // where a deferring sort left the previous positions
  auto go = [&](auto kern) {
    kern<<<grid, 256, 0, c.stream>>>(
        c.N, c.Npad, P.k, P.d, P.pk, P.pd, O.pk, O.pd, c.perm, c.force, (float)(dt * dt / M), c.hf, c.x0f,
        (float)(M / (2 * dt)), (float)(rcmax * rcmax), (float)(1 / (2 * M)), c.diag_part,
        capture_radius > 0 ? capture_radius * capture_radius : 0.0, c.x0, c.h, c.dsc, keys ? c.keys : nullptr,
        c.counts, c.fine.nk);
  };
  if (c.prev_deferred)
    go(k_push<true>);
  else
    go(k_push<false>);
  VLB_LAUNCHED(c);
  c.prev_deferred = false;
  k_diag_total<<<1, 256, 0, c.stream>>>(c.diag_part, grid, c.dsc->diag);
  VLB_LAUNCHED(c);
  c.keys_ready = keys;
}

void launch_projectile_update(Ctx& c, double dt, double nions, double jradius, int advance) {
  k_projectile<<<1, 32, 0, c.stream>>>(c.dsc, c.weight, dt, nions, jradius, advance);
  VLB_LAUNCHED(c);
}

void launch_projectile_force_only(Ctx& c, double nions, double jradius) {
  k_projectile<<<1, 32, 0, c.stream>>>(c.dsc, c.weight, 0.0, nions, jradius, 0);
  VLB_LAUNCHED(c);
}

void launch_film(Ctx& c, double capture_radius) {
  Particles& P = c.part[c.cur];
  const int n = c.fine.n;
  k_film_slice<<<(n * n + 255) / 256, 256, 0, c.stream>>>(c.fine.rho, n, c.film_iz1, c.film_iz2, c.film_frames,
                                                         c.film_cap, c.dsc);
  VLB_LAUNCHED(c);
  k_film_count<<<grid_for(c, c.N, 256, 8), 256, 0, c.stream>>>(c.N, c.Npad, P.k, P.d, c.x0, c.h, c.film_r2, c.dsc);
  VLB_LAUNCHED(c);
  k_film_finish<<<1, 1, 0, c.stream>>>(c.film_scalars, c.film_cap, capture_radius > 0 ? 1 : 0, c.dsc);
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
