// Host-side set-up helpers of the C ABI: the thesis's ran2 generator, the
// Thomas-Fermi sampling of the initial cloud, and the (k, delta) packing of
// positions.  They run once per simulation and need no GPU.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/vlasov_b200.h"

namespace {

// ran2 as it appears in the thesis code (src/random.jl:31-90): Numerical
// Recipes' combined L'Ecuyer generator with a Bays-Durham shuffle, whose
// IQ1 reads 3668 instead of 53668.  Schrage's guard then no longer holds and
// k*IR1 overflows 32 bits; the overflow is reproduced with wrapping
// arithmetic, which is what the Fortran (and the reference's Int32) does.
constexpr int32_t IM1 = 2147483563, IM2 = 2147483399, IMM1 = IM1 - 1;
constexpr int32_t IA1 = 40014, IA2 = 40692, IQ2 = 52774, IR1 = 12211, IR2 = 3791;
constexpr int NTAB = 32;
constexpr int32_t NDIV = 1 + (IMM1 - 1) / NTAB;

inline int32_t wrap_add(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
inline int32_t wrap_sub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
inline int32_t wrap_mul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }

inline int32_t schrage(int32_t x, int32_t q, int32_t r, int32_t a, int32_t m) {
  const int32_t k = x / q;  // truncating, as Julia's div
  x = wrap_sub(wrap_mul(a, wrap_sub(x, wrap_mul(k, q))), wrap_mul(k, r));
  return x < 0 ? wrap_add(x, m) : x;
}

struct Ran2 {
  int32_t idum, idum2, iy, iq1;
  int32_t iv[NTAB];

  Ran2(int32_t seed, bool consistent) {
    iq1 = consistent ? 53668 : 3668;
    idum = std::max<int32_t>(-seed, 1);
    idum2 = idum;
    for (int j = 0; j < NTAB; ++j) iv[j] = 0;
    for (int j = NTAB + 8; j >= 1; --j) {
      idum = schrage(idum, iq1, IR1, IA1, IM1);
      if (j <= NTAB) iv[j - 1] = idum;
    }
    iy = iv[0];
  }

  float next() {
    idum = schrage(idum, iq1, IR1, IA1, IM1);
    idum2 = schrage(idum2, IQ2, IR2, IA2, IM2);
    const int32_t j = 1 + iy / NDIV;
    iy = wrap_sub(iv[j - 1], idum2);
    iv[j - 1] = idum;
    if (iy < 1) iy = wrap_add(iy, IMM1);
    const float am = 1.0f / (float)IM1;
    const float rnmx = 1.0f - (float)1.2e-7;
    const float v = am * (float)iy;
    return v < rnmx ? v : rnmx;
  }
};

// _interp_regular (src/initial.jl:161-168); u in [0,1]
inline double interp_regular(const double* v, double u, int n) {
  int j = std::min((int)std::floor(u * (n - 1)) + 1, n - 1);  // 1-based
  const double a = (double)(j - 1) / (n - 1);
  const double b = (double)j / (n - 1);
  return v[j - 1] + (v[j] - v[j - 1]) * (u - a) / (b - a);
}

// _on_sphere (src/initial.jl:323-328)
inline void on_sphere(double r, double uphi, double umu, double* out) {
  const double mu = 2 * umu - 1;
  const double s = std::sqrt(1 - mu * mu);
  const double phi = (2 * M_PI) * uphi;
  out[0] = r * std::cos(phi) * s;
  out[1] = r * std::sin(phi) * s;
  out[2] = r * mu;
}

}  // namespace

extern "C" {

int vlb_ran2(int32_t seed, int32_t consistent, int64_t n, float* out) {
  if (!out || n < 0) return VLB_ERR_ARG;
  Ran2 rng(seed, consistent != 0);
  for (int64_t i = 0; i < n; ++i) out[i] = rng.next();
  return VLB_OK;
}

}  // extern "C"

// The seeded Thomas-Fermi draw as a stream: the generator and the profile
// persist between draws, so a cloud drawn in consecutive chunks is the
// one-shot cloud (src/initial.jl:94-113, six uniforms per particle).
struct vlb_sampler {
  Ran2 rng;
  std::vector<double> q, rho;
  double rmax, weight;
  vlb_sampler(int32_t seed, bool consistent) : rng(seed, consistent), rmax(0), weight(0) {}
};

namespace {

void draw(vlb_sampler& S, int64_t n, double* positions, double* momenta) {
  const double fermi = std::cbrt(3 * (M_PI * M_PI));  // FERMI_COEFFICIENT
  const int nq = (int)S.q.size(), nrho = (int)S.rho.size();
  for (int64_t i = 0; i < n; ++i) {
    double x[6];
    for (int a = 0; a < 6; ++a) x[a] = (double)S.rng.next();
    if (!positions) continue;  // a skipped particle still consumes its six uniforms
    const double r = interp_regular(S.q.data(), x[0], nq);
    on_sphere(r, x[1], x[2], positions + 3 * i);
    const double rho = interp_regular(S.rho.data(), r / S.rmax, nrho);
    const double p = std::cbrt(x[3]) * fermi * std::cbrt(rho);
    on_sphere(p * S.weight, x[4], x[5], momenta + 3 * i);
  }
}

}  // namespace

extern "C" {

int vlb_sampler_create(const double* quantiles, int32_t nq, const double* density, int32_t nrho, double rmax,
                       double weight, int32_t seed, int32_t consistent, vlb_sampler** out) {
  if (!out) return VLB_ERR_ARG;
  *out = nullptr;
  if (!quantiles || !density || nq < 2 || nrho < 2 || !(rmax > 0)) return VLB_ERR_ARG;
  try {
    vlb_sampler* S = new vlb_sampler(seed, consistent != 0);
    S->q.assign(quantiles, quantiles + nq);
    S->rho.assign(density, density + nrho);
    S->rmax = rmax;
    S->weight = weight;
    *out = S;
  } catch (...) {
    return VLB_ERR_NOMEM;
  }
  return VLB_OK;
}

int vlb_sampler_draw(vlb_sampler* sampler, int64_t n, double* positions, double* momenta) {
  if (!sampler || n < 0 || (!positions) != (!momenta)) return VLB_ERR_ARG;
  draw(*sampler, n, positions, momenta);
  return VLB_OK;
}

int vlb_sampler_destroy(vlb_sampler* sampler) {
  if (!sampler) return VLB_ERR_ARG;
  delete sampler;
  return VLB_OK;
}

int vlb_sample_thomas_fermi(const double* quantiles, int32_t nq, const double* density, int32_t nrho, double rmax,
                            int64_t npart, double weight, int32_t seed, int32_t consistent, double* positions,
                            double* momenta) {
  if (!quantiles || !density || !positions || !momenta || nq < 2 || nrho < 2 || npart < 0 || !(rmax > 0))
    return VLB_ERR_ARG;
  vlb_sampler* S = nullptr;
  if (int rc = vlb_sampler_create(quantiles, nq, density, nrho, rmax, weight, seed, consistent, &S)) return rc;
  draw(*S, npart, positions, momenta);
  delete S;
  return VLB_OK;
}

int vlb_pack_positions(int64_t npart, const double* positions, double x0, double h, int32_t* knode, float* delta) {
  if (!positions || !knode || !delta || npart < 0 || !(h > 0)) return VLB_ERR_ARG;
  for (int64_t i = 0; i < npart; ++i)
    for (int a = 0; a < 3; ++a) {
      const double x = positions[3 * i + a];
      const int32_t k = (int32_t)std::nearbyint((x - x0) / h) + 1;  // round, ties to even
      knode[a * npart + i] = k;
      delta[a * npart + i] = (float)(x - (x0 + (double)(k - 1) * h));
    }
  return VLB_OK;
}

int vlb_unpack_positions(int64_t npart, const int32_t* knode, const float* delta, double x0, double h,
                         double* positions) {
  if (!positions || !knode || !delta || npart < 0) return VLB_ERR_ARG;
  for (int64_t i = 0; i < npart; ++i)
    for (int a = 0; a < 3; ++a)
      positions[3 * i + a] = x0 + (double)(knode[a * npart + i] - 1) * h + (double)delta[a * npart + i];
  return VLB_OK;
}

}  // extern "C"
