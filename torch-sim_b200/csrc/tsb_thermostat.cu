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
#include "tsb_rng.cuh"

namespace tsb {

constexpr int kThBlock = 256;
constexpr int kMaxChain = 16;

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

// One chain sub-step of length `delta` (chain masses q, positions x, momenta v,
// M = chain length); returns the particle-momentum factor and updates ke.
__device__ double nhc_substep(double delta, int M, const double *q, double *x, double *v,
                              double &ke, double nf, double kt) {
  const double d2 = delta / 2.0, d4 = d2 / 2.0, d8 = d4 / 2.0;
  const int m = M - 1;
  if (m > 0) v[m] += d4 * (v[m - 1] * v[m - 1] / q[m - 1] - kt);
  for (int j = m - 1; j > 0; --j) {
    const double g = v[j - 1] * v[j - 1] / q[j - 1] - kt;
    const double s = exp(-d8 * v[j + 1] / q[j + 1]);
    v[j] = s * (s * v[j] + d4 * g);
  }
  {
    const double g = 2.0 * ke - nf * kt;
    const double s = m > 0 ? exp(-d8 * v[1] / q[1]) : 1.0;
    v[0] = s * (s * v[0] + d4 * g);
  }
  const double scale = exp(-d2 * v[0] / q[0]);
  ke = ke * (scale * scale);
  for (int j = 0; j < M; ++j) x[j] = x[j] + d2 * v[j] / q[j];
  double g = 2.0 * ke - nf * kt;
  for (int j = 0; j < m; ++j) {
    const double s = exp(-d8 * v[j + 1] / q[j + 1]);
    v[j] = s * (s * v[j] + d4 * g);
    g = v[j] * v[j] / q[j] - kt;
  }
  v[m] += d4 * g;
  return scale;
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
    double tot = 1.0;
    if (nc == 1 && nsy == 1) {
      tot = nhc_substep(h, M, q, x, v, k, nf, kt);
    } else {
      const double delta = h / nc;
      for (int sub = 0; sub < nc * nsy; ++sub)
        tot *= nhc_substep(delta * sy_weight(nsy, sub % nsy), M, q, x, v, k, nf, kt);
    }
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
__device__ double gamma_deviate(double a, uint64_t seed, int64_t s, uint64_t counter) {
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
    const double nf = dof[s];
    const double ke_old = nf * (sum / nf) / 2.0;  // dof * current kT / 2
    const double ke_new = nf * kT[s] / 2.0;
    double r1, g;
    if (noise) {
      r1 = noise[2 * s];
      g = noise[2 * s + 1];
    } else {
      r1 = thermo_normal(seed, s, counter, 0u);
      g = gamma_deviate((nf - 1.0) / 2.0, seed, s, counter);
    }
    const double c1 = exp(-dt[s] / tau[s]);
    const double c2 = (1.0 - c1) * ke_new / ke_old / nf;
    const double sc = c1 + c2 * (r1 * r1 + 2.0 * g) + 2.0 * r1 * sqrt(c1 * c2);
    s_lam = sqrt(sc);
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
