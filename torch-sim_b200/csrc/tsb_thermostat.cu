// Deterministic and stochastic velocity thermostats of the NVT step functions:
// Nose-Hoover chains and V-rescale (CSVR).  Both act on each system's momenta by
// one per-system factor, so one block owns one system: it sums the system's
// kinetic energy in FP64 (fixed order), its first thread advances the
// per-system thermostat scalars, and all threads rescale the momenta.
//
// * Nose-Hoover chain half step (torch_sim/integrators/md.py:388-514, Martyna,
//   Tuckerman, Tobias & Klein 1996): chain_steps x sy_steps Suzuki-Yoshida
//   sub-steps of the chain; chain masses Q_j = kT tau^2, Q_1 = N_f kT tau^2
//   recomputed on every call (md.py:534-559, nvt.py:466).
// * V-rescale factor (torch_sim/integrators/nvt.py:594-654, Bussi, Donadio &
//   Parrinello 2007, Eq. A7) with r1 ~ N(0,1) and a Gamma((N_f - 1)/2) deviate
//   drawn on the device (Marsaglia & Tsang 2000, from counter-based
//   Philox4x32-10 streams) or supplied by the caller.
#include <math.h>

#include "tsb_common.cuh"
#include "tsb_thermostat.cuh"

namespace tsb {

constexpr int kThBlock = 256;

struct ThermoWork {
  int64_t *lo, *hi;  // [S] atom range of each system
};

static void carve_thermo(Carver &c, ThermoWork &w, int64_t ns) {
  w.lo = c.take<int64_t>(ns);
  w.hi = c.take<int64_t>(ns);
}

__global__ void k_thermo_bounds(const int64_t *sys, int64_t n, int64_t *lo, int64_t *hi) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = sys[i];
  if (i == 0 || sys[i - 1] != s) lo[s] = i;
  if (i == n - 1 || sys[i + 1] != s) hi[s] = i + 1;
}

// sum of p^2 / m over a system's atoms (FP64, fixed order: strided per thread,
// shuffles inside each warp, warps in order); valid in every thread
template <class P>
__device__ double sys_p2m(const P *p, const P *m, int64_t a0, int64_t a1, double *sh) {
  double acc = 0.0;
  for (int64_t i = a0 + threadIdx.x; i < a1; i += blockDim.x) {
    const double px = p[3 * i], py = p[3 * i + 1], pz = p[3 * i + 2];
    acc += (px * px + py * py + pz * pz) / (double)m[i];
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
  __syncthreads();
  return t;
}

template <class P>
__device__ void scale_momenta(P *p, int64_t a0, int64_t a1, double s) {
  for (int64_t i = a0 + threadIdx.x; i < a1; i += blockDim.x)
    for (int c = 0; c < 3; ++c) p[3 * i + c] = (P)((double)p[3 * i + c] * s);
}

template <class P>
__global__ void __launch_bounds__(kThBlock)
    k_nhc_half(P *p, const P *m, const int64_t *lo, const int64_t *hi, double *xi,
               double *p_xi, double *Q, double *ke, const double *dof, const double *kT,
               const double *tau, const double *dt, int M, int nc, int nsy, int recompute) {
  __shared__ double sh[kThBlock / 32];
  __shared__ double s_scale;
  const int64_t s = blockIdx.x;
  const int64_t a0 = lo[s], a1 = hi[s];
  double k2 = 0.0;
  if (recompute) k2 = sys_p2m(p, m, a0, a1, sh);
  if (threadIdx.x == 0) {
    const double kt = kT[s], t = tau[s], nf = dof[s], h = dt[s];
    double q[kMaxChain], x[kMaxChain], v[kMaxChain];
    for (int j = 0; j < M; ++j) {
      q[j] = kt * (t * t);
      x[j] = xi[s * M + j];
      v[j] = p_xi[s * M + j];
    }
    q[0] *= nf;
    double k = recompute ? 0.5 * k2 : ke[s];
    const double tot = nhc_half(h, M, nc, nsy, q, x, v, k, nf, kt);
    for (int j = 0; j < M; ++j) {
      xi[s * M + j] = x[j];
      p_xi[s * M + j] = v[j];
      Q[s * M + j] = q[j];
    }
    ke[s] = k;
    s_scale = tot;
  }
  __syncthreads();
  scale_momenta(p, a0, a1, s_scale);
}

template <class P>
__global__ void __launch_bounds__(kThBlock)
    k_kinetic(const P *p, const P *m, const int64_t *lo, const int64_t *hi, double *ke) {
  __shared__ double sh[kThBlock / 32];
  const int64_t s = blockIdx.x;
  const double t = sys_p2m(p, m, lo[s], hi[s], sh);
  if (threadIdx.x == 0) ke[s] = 0.5 * t;
}

template <class P>
__global__ void __launch_bounds__(kThBlock)
    k_vrescale(P *p, const P *m, const int64_t *lo, const int64_t *hi, const double *dof,
               const double *kT, const double *tau, const double *dt, const double *noise,
               uint64_t seed, uint64_t counter, double *lam_out) {
  __shared__ double sh[kThBlock / 32];
  __shared__ double s_lam;
  const int64_t s = blockIdx.x;
  const int64_t a0 = lo[s], a1 = hi[s];
  const double sum = sys_p2m(p, m, a0, a1, sh);
  if (threadIdx.x == 0) {
    s_lam = vrescale_lambda(sum, dof[s], kT[s], dt[s], tau[s], noise ? noise + 2 * s : nullptr,
                            seed, s, counter);
    if (lam_out) lam_out[s] = s_lam;
  }
  __syncthreads();
  scale_momenta(p, a0, a1, s_lam);
}

static int thermo_prepare(const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                          void *workspace, size_t ws_bytes, ThermoWork &w, cudaStream_t st) {
  Carver c(workspace, ws_bytes);
  carve_thermo(c, w, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaMemsetAsync(w.lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(w.hi, 0, sizeof(int64_t) * n_systems, st);
  k_thermo_bounds<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, w.lo, w.hi);
  return TSB_OK;
}

}  // namespace tsb

using namespace tsb;

extern "C" size_t tsb_thermostat_workspace_size(int64_t n_systems) {
  Carver c(nullptr, (size_t)-1);
  ThermoWork w;
  carve_thermo(c, w, n_systems);
  return c.off + 256;
}

extern "C" int tsb_kinetic_energy(const void *momenta, const void *masses,
                                  const int64_t *system_idx, int64_t n_atoms,
                                  int64_t n_systems, int dtype, double *ke, void *workspace,
                                  size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !momenta || !masses || !system_idx || !ke)
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  ThermoWork w;
  TSB_TRY(thermo_prepare(system_idx, n_atoms, n_systems, workspace, workspace_bytes, w, st));
  if (dtype == TSB_F64)
    k_kinetic<double><<<(unsigned)n_systems, kThBlock, 0, st>>>(
        (const double *)momenta, (const double *)masses, w.lo, w.hi, ke);
  else
    k_kinetic<float><<<(unsigned)n_systems, kThBlock, 0, st>>>(
        (const float *)momenta, (const float *)masses, w.lo, w.hi, ke);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_nhc_half_step(void *momenta, const void *masses, const int64_t *system_idx,
                                 int64_t n_atoms, int64_t n_systems, int dtype, double *xi,
                                 double *p_xi, double *Q, double *ke, const double *dof,
                                 const double *kT, const double *tau, const double *dt,
                                 int chain_length, int chain_steps, int sy_steps,
                                 int recompute_ke, void *workspace, size_t workspace_bytes,
                                 void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !momenta || !masses || !system_idx || !xi || !p_xi ||
      !Q || !ke || !dof || !kT || !tau || !dt)
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  if (chain_length < 1 || chain_length > kMaxChain || chain_steps < 1) return TSB_ERR_INVALID_ARG;
  if (sy_steps != 1 && sy_steps != 3 && sy_steps != 5 && sy_steps != 7) return TSB_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  ThermoWork w;
  TSB_TRY(thermo_prepare(system_idx, n_atoms, n_systems, workspace, workspace_bytes, w, st));
  if (dtype == TSB_F64)
    k_nhc_half<double><<<(unsigned)n_systems, kThBlock, 0, st>>>(
        (double *)momenta, (const double *)masses, w.lo, w.hi, xi, p_xi, Q, ke, dof, kT, tau,
        dt, chain_length, chain_steps, sy_steps, recompute_ke);
  else
    k_nhc_half<float><<<(unsigned)n_systems, kThBlock, 0, st>>>(
        (float *)momenta, (const float *)masses, w.lo, w.hi, xi, p_xi, Q, ke, dof, kT, tau,
        dt, chain_length, chain_steps, sy_steps, recompute_ke);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_vrescale(void *momenta, const void *masses, const int64_t *system_idx,
                            int64_t n_atoms, int64_t n_systems, int dtype, const double *dof,
                            const double *kT, const double *tau, const double *dt,
                            const double *noise, uint64_t seed, uint64_t counter,
                            double *lam, void *workspace, size_t workspace_bytes,
                            void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !momenta || !masses || !system_idx || !dof || !kT ||
      !tau || !dt)
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  ThermoWork w;
  TSB_TRY(thermo_prepare(system_idx, n_atoms, n_systems, workspace, workspace_bytes, w, st));
  if (dtype == TSB_F64)
    k_vrescale<double><<<(unsigned)n_systems, kThBlock, 0, st>>>(
        (double *)momenta, (const double *)masses, w.lo, w.hi, dof, kT, tau, dt, noise, seed,
        counter, lam);
  else
    k_vrescale<float><<<(unsigned)n_systems, kThBlock, 0, st>>>(
        (float *)momenta, (const float *)masses, w.lo, w.hi, dof, kT, tau, dt, noise, seed,
        counter, lam);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}
