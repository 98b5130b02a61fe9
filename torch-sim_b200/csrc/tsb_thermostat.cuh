// Per-system thermostat arithmetic shared by the thermostat kernels and the
// persistent fused MD kernel (same FP64 operations and random streams in both).
//
// * nhc_substep: one Nose-Hoover-chain sub-step (torch_sim/integrators/md.py:388-455)
// * sy_weight: Suzuki-Yoshida composition weights (Yoshida 1990, Suzuki 1993)
// * nhc_half: chain_steps x sy_steps sub-steps (md.py:457-514); returns the
//   momentum factor
// * thermo_normal / gamma_deviate: counter-based draws for the V-rescale factor
// * vrescale_lambda: the CSVR factor (torch_sim/integrators/nvt.py:594-654)
#pragma once

#include <math.h>

#include "tsb_rng.cuh"

namespace tsb {

constexpr int kMaxChain = 16;

__device__ inline double sy_weight(int n, int k) {
  // Suzuki-Yoshida composition weights (Yoshida 1990, Suzuki 1993)
  switch (n) {
    case 3: {
      const double w[3] = {0.828981543588751, -0.657963087177502, 0.828981543588751};
      return w[k];
    }
    case 5: {
      const double w[5] = {0.2967324292201065, 0.2967324292201065, -0.186929716880426,
                           0.2967324292201065, 0.2967324292201065};
      return w[k];
    }
    case 7: {
      const double w[7] = {0.784513610477560, 0.235573213359357, -1.17767998417887,
                           1.31518632068391, -1.17767998417887, 0.235573213359357,
                           0.784513610477560};
      return w[k];
    }
    default:
      return 1.0;
  }
}

// One chain sub-step of length `delta` (chain masses q with reciprocals iq,
// positions x, momenta v, M = chain length); returns the particle-momentum
// factor and updates ke.  The forward pass reuses the backward pass's factors
// exp(-delta/8 v_{j+1}/q_{j+1}): v_{j+1} does not change in between, so the
// values are identical.  Divisions by q are multiplications by 1/q (one
// thread runs these sub-steps serially).
__device__ inline double nhc_substep(double delta, int M, const double *iq, double *x,
                                     double *v, double &ke, double nf, double kt) {
  const double d2 = delta / 2.0, d4 = d2 / 2.0, d8 = d4 / 2.0;
  const int m = M - 1;
  double sj[kMaxChain];
  if (m > 0) v[m] += d4 * (v[m - 1] * v[m - 1] * iq[m - 1] - kt);
  for (int j = m - 1; j > 0; --j) {
    const double g = v[j - 1] * v[j - 1] * iq[j - 1] - kt;
    const double s = exp(-d8 * v[j + 1] * iq[j + 1]);
    sj[j] = s;
    v[j] = s * (s * v[j] + d4 * g);
  }
  {
    const double g = 2.0 * ke - nf * kt;
    const double s = m > 0 ? exp(-d8 * v[1] * iq[1]) : 1.0;
    sj[0] = s;
    v[0] = s * (s * v[0] + d4 * g);
  }
  const double scale = exp(-d2 * v[0] * iq[0]);
  ke = ke * (scale * scale);
  for (int j = 0; j < M; ++j) x[j] = x[j] + d2 * v[j] * iq[j];
  double g = 2.0 * ke - nf * kt;
  for (int j = 0; j < m; ++j) {
    const double s = sj[j];
    v[j] = s * (s * v[j] + d4 * g);
    g = v[j] * v[j] * iq[j] - kt;
  }
  v[m] += d4 * g;
  return scale;
}

// chain_steps x sy_steps sub-steps over a chain time step h (or one sub-step
// of length h when both are 1); x, v in/out, ke in/out; returns the product of
// the momentum factors
__device__ inline double nhc_half(double h, int M, int nc, int nsy, const double *q, double *x,
                                  double *v, double &ke, double nf, double kt) {
  double iq[kMaxChain];
  for (int j = 0; j < M; ++j) iq[j] = 1.0 / q[j];
  if (nc == 1 && nsy == 1) return nhc_substep(h, M, iq, x, v, ke, nf, kt);
  double tot = 1.0;
  const double delta = h / nc;
  for (int sub = 0; sub < nc * nsy; ++sub)
    tot *= nhc_substep(delta * sy_weight(nsy, sub % nsy), M, iq, x, v, ke, nf, kt);
  return tot;
}

// uniform in (0, 1] with 53 random bits from two 32-bit words
__device__ inline double u53(uint32_t a, uint32_t b) {
  return ((double)((uint64_t)(a >> 5) * 67108864ull + (b >> 6)) + 1.0) *
         1.1102230246251565e-16;
}

// Philox words for (seed, system, counter, slot): the slot separates the draws
// of one step; the tag word keeps these streams apart from the Langevin ones
__device__ inline U4 thermo_words(uint64_t seed, int64_t s, uint64_t counter, uint32_t slot) {
  U4 c{(uint32_t)s, 0xC5A00000u ^ slot, (uint32_t)counter, (uint32_t)(counter >> 32)};
  return philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
}

__device__ inline double thermo_normal(uint64_t seed, int64_t s, uint64_t counter,
                                       uint32_t slot) {
  const U4 r = thermo_words(seed, s, counter, slot);
  return sqrt(-2.0 * log(u53(r.x, r.y))) * cospi(2.0 * u53(r.z, r.w));
}

// Gamma(a, 1) deviate, a > 0 (Marsaglia & Tsang, ACM TOMS 26:363, 2000; a < 1
// through Gamma(a + 1) U^(1/a)); at most 64 proposals (acceptance > 95 % for
// a >= 1), after which the mode-like value d is returned
__device__ inline double gamma_deviate(double a, uint64_t seed, int64_t s, uint64_t counter) {
  double boost = 1.0;
  if (a < 1.0) {
    const U4 r = thermo_words(seed, s, counter, 1u);
    boost = pow(u53(r.x, r.y), 1.0 / a);
    a += 1.0;
  }
  const double d = a - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
  for (uint32_t k = 0; k < 64; ++k) {
    const double xn = thermo_normal(seed, s, counter, 16u + 2u * k);
    const double v0 = 1.0 + c * xn;
    if (v0 <= 0.0) continue;
    const double v = v0 * v0 * v0;
    const U4 r = thermo_words(seed, s, counter, 17u + 2u * k);
    const double u = u53(r.x, r.y);
    if (u < 1.0 - 0.0331 * (xn * xn) * (xn * xn) ||
        log(u) < 0.5 * xn * xn + d * (1.0 - v + log(v)))
      return d * v * boost;
  }
  return d * boost;
}

// CSVR factor lambda from the kinetic energy (as sum p^2/m) of a system with nf
// degrees of freedom; r1 and g from `noise` when given, else drawn
__device__ inline double vrescale_lambda(double sum_p2m, double nf, double kt, double dt,
                                         double tau, const double *noise, uint64_t seed,
                                         int64_t s, uint64_t counter) {
  const double ke_old = nf * (sum_p2m / nf) / 2.0;  // dof * current kT / 2
  const double ke_new = nf * kt / 2.0;
  double r1, g;
  if (noise) {
    r1 = noise[0];
    g = noise[1];
  } else {
    r1 = thermo_normal(seed, s, counter, 0u);
    g = gamma_deviate((nf - 1.0) / 2.0, seed, s, counter);
  }
  const double c1 = exp(-dt / tau);
  const double c2 = (1.0 - c1) * ke_new / ke_old / nf;
  return sqrt(c1 + c2 * (r1 * r1 + 2.0 * g) + 2.0 * r1 * sqrt(c1 * c2));
}

}  // namespace tsb
