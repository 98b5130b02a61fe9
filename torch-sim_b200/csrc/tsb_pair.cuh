// Pair-potential arithmetic shared by the fused-search force kernel and the
// persistent MD kernel.
//
// Parameter rows (derived on the device from the caller's (p0,p1,p2,rc,eshift)):
//   LJ    (lennard_jones.py:23-47):  a0=sigma^2 a1=4eps a2=24eps
//   MORSE (morse.py:23-47):          a0=sigma  a1=eps  a2=alpha a5=2*alpha*eps
//   SOFT  (soft_sphere.py:35-59):    a0=sigma  a1=1/sigma a2=alpha a5=eps/alpha a6=eps/sigma
//   PLIFE (particle_life.py:24-54):  a0=beta a1=A a5=1-beta a6=sigma a7=1+beta (force only)
//   a3 = effective cutoff^2 = min(cutoff, rc)^2 (SOFT also min with sigma), a4 = eshift
#pragma once

#include "tsb_common.cuh"

namespace tsb {

constexpr int kMaxSpecies = 16;

template <class R>
struct PairPrm {
  R a0, a1, a2, a3, a4, a5, a6, a7;
};

template <class R>
__device__ inline PairPrm<R> make_prm(int pot, const double *t, double cutoff) {
  // t = (p0, p1, p2, rc, eshift)
  PairPrm<R> q;
  double rc = fmin(cutoff, t[3]);
  q.a4 = (R)t[4];
  q.a7 = (R)0;
  if (pot == TSB_POT_LJ) {
    q.a0 = (R)(t[0] * t[0]);
    q.a1 = (R)(4.0 * t[1]);
    q.a2 = (R)(24.0 * t[1]);
    q.a5 = q.a6 = (R)0;
  } else if (pot == TSB_POT_MORSE) {
    q.a0 = (R)t[0];
    q.a1 = (R)t[1];
    q.a2 = (R)t[2];
    q.a5 = (R)(2.0 * t[2] * t[1]);
    q.a6 = (R)0;
  } else if (pot == TSB_POT_PLIFE) {
    q.a0 = (R)t[2];
    q.a1 = (R)t[1];
    q.a2 = (R)0;
    q.a5 = (R)(1.0 - t[2]);
    q.a6 = (R)t[0];
    q.a7 = (R)(1.0 + t[2]);
  } else {
    rc = fmin(rc, t[0]);
    q.a0 = (R)t[0];
    q.a1 = (R)(1.0 / t[0]);
    q.a2 = (R)t[2];
    q.a5 = (R)(t[1] / t[2]);
    q.a6 = (R)(t[1] / t[0]);
  }
  q.a3 = (R)(rc * rc);
  return q;
}

// FP64 effective cutoff^2 of a parameter row (the in/out decision of a pair is
// made on the FP64 squared distance against this, as the FP64 reference does).
__device__ inline double pair_rc2(int pot, const double *t, double cutoff) {
  double rc = fmin(cutoff, t[3]);
  if (pot == TSB_POT_SOFT) rc = fmin(rc, t[0]);
  return rc * rc;
}

__device__ inline float rsqrt_r(float x) { return rsqrtf(x); }
__device__ inline double rsqrt_r(double x) { return rsqrt(x); }
__device__ inline float exp_r(float x) { return expf(x); }
__device__ inline double exp_r(double x) { return exp(x); }
__device__ inline float pow_r(float x, float y) { return powf(x, y); }
__device__ inline double pow_r(double x, double y) { return pow(x, y); }

// Returns pair energy e and fr = -(dV/dr)/r, so that the force on j due to i is
// fr * (r_j - r_i) (pair_potential.py:426-428).  Caller guarantees r2 < a3.
template <int POT, class R>
__device__ __forceinline__ void pair_eval(const PairPrm<R> &q, R r2, R &e, R &fr) {
  if (POT == TSB_POT_LJ) {
    if (r2 > R(0)) {
      R ir2 = R(1) / r2;
      R s2 = q.a0 * ir2;
      R s6 = s2 * s2 * s2;
      e = q.a1 * (s6 * s6 - s6) - q.a4;
      fr = q.a2 * (R(2) * s6 * s6 - s6) * ir2;
    } else {
      e = R(0) - q.a4;
      fr = R(0);
    }
  } else if (POT == TSB_POT_MORSE) {
    if (r2 > R(0)) {
      R ir = rsqrt_r(r2);
      R r = r2 * ir;
      R ex = exp_r(-q.a2 * (r - q.a0));
      R om = R(1) - ex;
      e = q.a1 * om * om - q.a1 - q.a4;
      fr = -q.a5 * ex * om * ir;
    } else {
      e = R(0) - q.a4;
      fr = R(0);
    }
  } else if (POT == TSB_POT_PLIFE) {
    // force-defined: magnitude f(r) = r/beta - 1 (r < beta), A (1 - |2r - 1 - beta| /
    // (1 - beta)) (beta <= r < sigma); fr = f / r, no energy
    const R r = sqrt(r2);
    const R f = r < q.a0 ? r / q.a0 - R(1)
                         : (r < q.a6 ? q.a1 * (R(1) - fabs(R(2) * r - q.a7) / q.a5) : R(0));
    e = R(0);
    fr = r > R(0) ? f / r : R(0);
  } else {  // SOFT: V = eps/alpha (1 - r/sigma)^alpha for r < sigma
    R r = (r2 > R(0)) ? r2 * rsqrt_r(r2) : R(0);
    R base = R(1) - r * q.a1;
    R bam1 = (q.a2 == R(2)) ? base : pow_r(base, q.a2 - R(1));
    e = q.a5 * bam1 * base - q.a4;
    fr = (r2 > R(0)) ? q.a6 * bam1 / r : R(0);
  }
}

// PTX approximate instructions (relative error ~2^-22 .. 2^-23, denormals
// flushed: r^2 > 1e-30 and the exponents here are far from the denormal range).
__device__ __forceinline__ float ex2_ftz(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_ftz(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Morse rows used with pair_eval_fast also carry the exponent as one FMA in base 2:
// a6 = -alpha log2(e), a7 = alpha r0 log2(e), so exp(-alpha (r - r0)) =
// 2^(a6 r + a7).
__device__ inline void prm_fast_extra(int pot, const double *t, PairPrm<float> &q) {
  if (pot == TSB_POT_MORSE) {
    const double log2e = 1.4426950408889634;
    q.a6 = (float)(-t[2] * log2e);
    q.a7 = (float)(t[2] * t[0] * log2e);
  }
}

// Fast FP32 pair evaluation (same e and fr = -V'(r)/r as pair_eval, fewer
// instructions; rows need prm_fast_extra).
template <int POT>
__device__ __forceinline__ void pair_eval_fast(const PairPrm<float> &q, float r2, float &e,
                                               float &fr) {
  if (POT == TSB_POT_MORSE) {
    // V = D (1 - x)^2 - D - shift = D x (x - 2) - shift, x = exp(-alpha (r - r0))
    const float ir = rsqrt_ftz(r2);
    const float r = r2 * ir;
    const float x = ex2_ftz(fmaf(q.a6, r, q.a7));
    e = q.a1 * x * (x - 2.0f) - q.a4;
    fr = -q.a5 * fmaf(-x, x, x) * ir;  // -2 alpha D x (1 - x) / r
  } else if (POT == TSB_POT_LJ) {
    // V = 4 eps (s6^2 - s6) - shift, s6 = (sigma^2 / r^2)^3
    const float ir2 = rcp_ftz(r2);
    const float s2 = q.a0 * ir2;
    const float s6 = s2 * s2 * s2;
    e = q.a1 * s6 * (s6 - 1.0f) - q.a4;
    fr = q.a2 * s6 * fmaf(2.0f, s6, -1.0f) * ir2;
  } else {
    pair_eval<POT, float>(q, r2, e, fr);
  }
}

}  // namespace tsb
