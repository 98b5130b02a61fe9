// Elementwise integrator steps with per-system dt / kT / gamma.
//   kick : p += F * (scale*dt)                 torch_sim/integrators/md.py:169-187
//   drift: q += (p / m) * (scale*dt)           md.py:190-208
//   baoab_boa: B(dt/2) A(dt/2) O(dt) A(dt/2)   torch_sim/integrators/nvt.py:144-240,
//              O-step p <- c1 p + c2 sqrt(m) xi, c1 = exp(-gamma dt),
//              c2 = sqrt(kT (1 - c1^2))        nvt.py:27-86
// The floating-point operation order follows the reference expressions so a
// float64 step with the same noise agrees to the last bits.
#include "tsb_common.cuh"
#include "tsb_rng.cuh"

namespace tsb {

template <class P>
__global__ void k_kick(P *p, const P *f, const int64_t *sys, const double *dt, double scale,
                       int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const P h = (P)(scale * dt[sys[i]]);
#pragma unroll
  for (int k = 0; k < 3; ++k) p[3 * i + k] = p[3 * i + k] + f[3 * i + k] * h;
}

template <class P>
__global__ void k_drift(P *q, const P *p, const P *m, const int64_t *sys, const double *dt,
                        double scale, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const P h = (P)(scale * dt[sys[i]]);
  const P mi = m[i];
#pragma unroll
  for (int k = 0; k < 3; ++k) q[3 * i + k] = q[3 * i + k] + (p[3 * i + k] / mi) * h;
}

template <class P>
__global__ void k_baoab_boa(P *q, P *p, const P *f, const P *m, const int64_t *sys,
                            const double *dt_s, const double *kT_s, const double *g_s,
                            const P *noise, uint64_t seed, uint64_t counter,
                            const uint64_t *counter_dev, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (counter_dev) counter += *counter_dev;
  const int64_t s = sys[i];
  const P dt = (P)dt_s[s];
  const P half = dt / (P)2;
  const P mi = m[i];
  P pp[3], qq[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    pp[k] = p[3 * i + k] + f[3 * i + k] * half;
    qq[k] = q[3 * i + k] + (pp[k] / mi) * half;
  }
  const P c1 = (P)exp(-(double)((P)g_s[s] * dt));
  const P c2 = (P)sqrt((double)((P)kT_s[s] * ((P)1 - c1 * c1)));
  const P c2m = c2 * (P)sqrt((double)mi);
  double z[4];
  if (!noise) normal4(seed, (uint64_t)i, counter, z);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const P xi = noise ? noise[3 * i + k] : (P)z[k];
    pp[k] = c1 * pp[k] + c2m * xi;
    q[3 * i + k] = qq[k] + (pp[k] / mi) * half;
    p[3 * i + k] = pp[k];
  }
}

// advances the device-resident noise counter by one step (after the kernel that
// read it, in stream order)
__global__ void k_advance_step_counter(uint64_t *counter_dev) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *counter_dev += 1ull;
}

}  // namespace tsb

using namespace tsb;

extern "C" int tsb_md_kick(void *momenta, const void *forces, const int64_t *system_idx,
                           const double *dt_sys, double scale, int64_t n_atoms, int dtype,
                           void *stream) {
  if (n_atoms < 0 || (n_atoms > 0 && (!momenta || !forces || !system_idx || !dt_sys)))
    return TSB_ERR_INVALID_ARG;
  if (n_atoms == 0) return TSB_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == TSB_F64)
    k_kick<double><<<grid_for(n_atoms), kBlock, 0, st>>>(
        (double *)momenta, (const double *)forces, system_idx, dt_sys, scale, n_atoms);
  else if (dtype == TSB_F32)
    k_kick<float><<<grid_for(n_atoms), kBlock, 0, st>>>(
        (float *)momenta, (const float *)forces, system_idx, dt_sys, scale, n_atoms);
  else
    return TSB_ERR_INVALID_ARG;
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_md_drift(void *positions, const void *momenta, const void *masses,
                            const int64_t *system_idx, const double *dt_sys, double scale,
                            int64_t n_atoms, int dtype, void *stream) {
  if (n_atoms < 0 ||
      (n_atoms > 0 && (!positions || !momenta || !masses || !system_idx || !dt_sys)))
    return TSB_ERR_INVALID_ARG;
  if (n_atoms == 0) return TSB_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == TSB_F64)
    k_drift<double><<<grid_for(n_atoms), kBlock, 0, st>>>(
        (double *)positions, (const double *)momenta, (const double *)masses, system_idx,
        dt_sys, scale, n_atoms);
  else if (dtype == TSB_F32)
    k_drift<float><<<grid_for(n_atoms), kBlock, 0, st>>>(
        (float *)positions, (const float *)momenta, (const float *)masses, system_idx,
        dt_sys, scale, n_atoms);
  else
    return TSB_ERR_INVALID_ARG;
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_md_baoab_boa(void *positions, void *momenta, const void *forces,
                                const void *masses, const int64_t *system_idx,
                                const double *dt_sys, const double *kT_sys,
                                const double *gamma_sys, const void *noise, uint64_t seed,
                                uint64_t counter, uint64_t *counter_dev, int64_t n_atoms,
                                int dtype, void *stream) {
  if (n_atoms < 0 || (n_atoms > 0 && (!positions || !momenta || !forces || !masses ||
                                      !system_idx || !dt_sys || !kT_sys || !gamma_sys)))
    return TSB_ERR_INVALID_ARG;
  if (n_atoms == 0) return TSB_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == TSB_F64)
    k_baoab_boa<double><<<grid_for(n_atoms), kBlock, 0, st>>>(
        (double *)positions, (double *)momenta, (const double *)forces,
        (const double *)masses, system_idx, dt_sys, kT_sys, gamma_sys,
        (const double *)noise, seed, counter, counter_dev, n_atoms);
  else if (dtype == TSB_F32)
    k_baoab_boa<float><<<grid_for(n_atoms), kBlock, 0, st>>>(
        (float *)positions, (float *)momenta, (const float *)forces, (const float *)masses,
        system_idx, dt_sys, kT_sys, gamma_sys, (const float *)noise, seed, counter, counter_dev,
        n_atoms);
  else
    return TSB_ERR_INVALID_ARG;
  if (counter_dev) k_advance_step_counter<<<1, 32, 0, st>>>(counter_dev);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}
