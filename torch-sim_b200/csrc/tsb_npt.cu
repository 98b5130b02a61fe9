// Isotropic NPT Langevin step (torch_sim/integrators/npt.py:653-1107): the cell
// degree of freedom is the logarithmic strain eps = ln(V/V0)/3, integrated with
// particle and strain positions/velocities by the Gronbech-Jensen-Farago
// Langevin scheme.  The step is split around the force call:
//
//   pre:  per system, strain force F_eps = 3 V (P_avg - P_ext) with
//         P_avg = -tr(stress)/3 + N kT / V (npt.py:704-749), barostat mass
//         Q = (N + 1) kT b_tau^2, strain position step (:769-798), new cell
//         exp(eps) h0 (:690-697); per atom, the GJF position step with the box
//         scaled by exp(eps_new - eps_old) (:838-885)
//   post: per system, the strain velocity step with the new strain force
//         (:801-835); per atom, the GJF velocity step (:316-367)
//
// The same noise realisation enters both halves: it is read from the caller's
// arrays, or drawn twice from the same counter-based Philox4x32-10 streams
// (particle: key seed, counter (atom, step); strain: (system, step)).
#include <math.h>

#include "tsb_common.cuh"
#include "tsb_rng.cuh"
#include "tsb_thermostat.cuh"
#include "tsb_mat3.cuh"

namespace tsb {

struct NptWork {
  int64_t *lo, *hi;  // [S] atom range of each system
  double *scale;     // [S] exp(eps_new - eps_old), or the isotropic C-rescale factor
  double *scale3;    // [3S] per-axis C-rescale factors
  double *kin6;      // [6S] sum_i p p^T / m per system (xx, yy, zz, xy, xz, yz)
  double *rv;        // [18S] triclinic C-rescale: R and the momentum matrix per system
};

static void carve_npt(Carver &c, NptWork &w, int64_t ns) {
  w.lo = c.take<int64_t>(ns);
  w.hi = c.take<int64_t>(ns);
  w.scale = c.take<double>(ns);
  w.scale3 = c.take<double>(3 * ns);
  w.kin6 = c.take<double>(6 * ns);
  w.rv = c.take<double>(18 * ns);
}

__global__ void k_npt_bounds(const int64_t *sys, int64_t n, int64_t *lo, int64_t *hi) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = sys[i];
  if (i == 0 || sys[i - 1] != s) lo[s] = i;
  if (i == n - 1 || sys[i + 1] != s) hi[s] = i + 1;
}

__device__ inline double det3(const double *a) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
         a[2] * (a[3] * a[7] - a[4] * a[6]);
}

template <class P>
__device__ inline double strain_force(const P *stress, double vol, double n_at, double kt,
                                      double p_ext) {
  const double tr = (double)stress[0] + (double)stress[4] + (double)stress[8];
  const double p_avg = -tr / 3.0 + n_at * kt / vol;
  return 3.0 * vol * (p_avg - p_ext);
}

__device__ inline double cell_noise_of(const double *cell_noise, uint64_t seed, int64_t s,
                                       uint64_t counter) {
  return cell_noise ? cell_noise[s] : thermo_normal(seed, s, counter, 2u);
}

__device__ inline void particle_noise_of(const double *pn, uint64_t seed, int64_t i,
                                         uint64_t counter, double *z) {
  if (pn) {
    z[0] = pn[3 * i];
    z[1] = pn[3 * i + 1];
    z[2] = pn[3 * i + 2];
  } else {
    normal4(seed, (uint64_t)i, counter, z);
  }
}

template <class P>
__global__ void k_npt_cell_pre(int64_t ns, const int64_t *lo, const int64_t *hi,
                               const P *stress, const double *ref_cell, P *cell, double *eps,
                               const double *eps_dot, double *Q, double *f_eps, double *scale,
                               const double *cell_alpha, const double *b_tau, const double *kT,
                               const double *p_ext, const double *dt, const double *cell_noise,
                               uint64_t seed, uint64_t counter) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const double n_at = (double)(hi[s] - lo[s]), kt = kT[s], h = dt[s], ac = cell_alpha[s];
  const double q = (n_at + 1.0) * kt * (b_tau[s] * b_tau[s]);
  const double v0 = det3(ref_cell + 9 * s);
  const double e0 = eps[s];
  const double f = strain_force(stress + 9 * s, v0 * exp(3.0 * e0), n_at, kt, p_ext[s]);
  const double beta = sqrt(2.0 * ac * kt * h) * cell_noise_of(cell_noise, seed, s, counter);
  const double q2 = 2.0 * q;
  const double cb = 1.0 / (1.0 + (ac * h) / q2);
  const double e1 = e0 + cb * h * eps_dot[s] + cb * h * h * f / q2 + cb * h * beta / q2;
  Q[s] = q;
  f_eps[s] = f;
  eps[s] = e1;
  scale[s] = exp(e1 - e0);
  const double g = exp(e1);
  for (int k = 0; k < 9; ++k) cell[9 * s + k] = (P)(g * ref_cell[9 * s + k]);
}

template <class P>
__global__ void k_npt_atom_pre(int64_t n, P *x, const P *p, const P *f, const P *m,
                               const int64_t *sys, const double *scale, const double *alpha,
                               const double *kT, const double *dt, const double *pn,
                               uint64_t seed, uint64_t counter) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = sys[i];
  double z[4];
  particle_noise_of(pn, seed, i, counter, z);
  const double a = alpha[s], h = dt[s], mi = m[i], sc = scale[s];
  const double pre = sqrt(2.0 * a * kT[s] * h);
  const double b = 1.0 / (1.0 + (a * h) / (2.0 * mi));
  const double c2 = (2.0 * sc / (sc + 1.0)) * b * h;
  for (int c = 0; c < 3; ++c) {
    const double c3 = (double)p[3 * i + c] / mi + h * (double)f[3 * i + c] / (2.0 * mi) +
                      pre * z[c] / (2.0 * mi);
    x[3 * i + c] = (P)(sc * (double)x[3 * i + c] + c2 * c3);
  }
}

template <class P>
__global__ void k_npt_cell_post(int64_t ns, const int64_t *lo, const int64_t *hi,
                                const P *stress, const double *ref_cell, const double *eps,
                                double *eps_dot, const double *Q, const double *f_eps,
                                const double *cell_alpha, const double *kT,
                                const double *p_ext, const double *dt, const double *cell_noise,
                                uint64_t seed, uint64_t counter) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const double n_at = (double)(hi[s] - lo[s]), kt = kT[s], h = dt[s], ac = cell_alpha[s];
  const double q = Q[s];
  const double v = det3(ref_cell + 9 * s) * exp(3.0 * eps[s]);
  const double f1 = strain_force(stress + 9 * s, v, n_at, kt, p_ext[s]);
  const double beta = sqrt(2.0 * ac * kt * h) * cell_noise_of(cell_noise, seed, s, counter);
  const double a = (1.0 - (ac * h) / (2.0 * q)) / (1.0 + (ac * h) / (2.0 * q));
  const double b = 1.0 / (1.0 + (ac * h) / (2.0 * q));
  eps_dot[s] = a * eps_dot[s] + h * ((a * f_eps[s]) + f1) / (2.0 * q) + b * beta / q;
}

template <class P>
__global__ void k_npt_atom_post(int64_t n, P *p, const P *m, const P *f_old, const P *f_new,
                                const int64_t *sys, const double *alpha, const double *kT,
                                const double *dt, const double *pn, uint64_t seed,
                                uint64_t counter) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = sys[i];
  double z[4];
  particle_noise_of(pn, seed, i, counter, z);
  const double al = alpha[s], h = dt[s], mi = m[i];
  const double pre = sqrt(2.0 * al * kT[s] * h);
  const double m2 = 2.0 * mi;
  const double a = (1.0 - (al * h) / m2) / (1.0 + (al * h) / m2);
  const double b = 1.0 / (1.0 + (al * h) / m2);
  for (int c = 0; c < 3; ++c) {
    const double v = (double)p[3 * i + c] / mi;
    const double vn = a * v + h * ((a * (double)f_old[3 * i + c]) + (double)f_new[3 * i + c]) / m2 +
                      b * (pre * z[c]) / mi;
    p[3 * i + c] = (P)(vn * mi);
  }
}

// Anisotropic NPT Langevin (npt.py:62-650): per-axis strains eps_k = ln(L_k/L0_k),
// cell row k = exp(eps_k) row k of the reference cell (:123-127), strain forces
// F_k = V (-sigma_kk + N kT / V - P_k) with V = det(cell) (:370-406), the GJF
// strain steps per axis with the shared mass Q = (N + 1) kT b_tau^2 (:201-264),
// positions scaled per component by exp(eps_new_k - eps_old_k) (:267-313); the
// particle velocity step is the isotropic one.  Cell noise [S, 3] (Philox slots
// 3..5 by default) and particle noise are shared by both halves.
template <class P>
__device__ inline void aniso_strain_force(const P *stress, const double *C, double n_at,
                                          double kt, const double *p_ext, double *f) {
  const double vol = det3(C);
  for (int k = 0; k < 3; ++k)
    f[k] = vol * ((-(double)stress[4 * k] + n_at * kt / vol) - p_ext[k]);
}

__device__ inline double aniso_cell_noise(const double *cn, uint64_t seed, int64_t s, int k,
                                          uint64_t counter) {
  return cn ? cn[3 * s + k] : thermo_normal(seed, s, counter, 3u + (uint32_t)k);
}

template <class P>
__global__ void k_npt_aniso_cell_pre(int64_t ns, const int64_t *lo, const int64_t *hi,
                                     const P *stress, const double *ref_cell, P *cell,
                                     double *eps, const double *eps_dot, double *Q,
                                     double *f_eps, double *scale3, const double *cell_alpha,
                                     const double *b_tau, const double *kT, const double *p_ext,
                                     const double *dt, const double *cell_noise, uint64_t seed,
                                     uint64_t counter) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const double n_at = (double)(hi[s] - lo[s]), kt = kT[s], h = dt[s], ac = cell_alpha[s];
  const double q = (n_at + 1.0) * kt * (b_tau[s] * b_tau[s]);
  double C[9];
  for (int k = 0; k < 9; ++k) C[k] = (double)cell[9 * s + k];
  double f[3];
  aniso_strain_force(stress + 9 * s, C, n_at, kt, p_ext + 3 * s, f);
  const double q2 = 2.0 * q;
  const double cb = 1.0 / (1.0 + (ac * h) / q2);
  const double sc = sqrt(2.0 * ac * kt * h);
  for (int k = 0; k < 3; ++k) {
    const double beta = sc * aniso_cell_noise(cell_noise, seed, s, k, counter);
    const double e0 = eps[3 * s + k];
    const double e1 = e0 + cb * h * eps_dot[3 * s + k] + cb * h * h * f[k] / q2 + cb * h * beta / q2;
    eps[3 * s + k] = e1;
    f_eps[3 * s + k] = f[k];
    scale3[3 * s + k] = exp(e1 - e0);
    const double g = exp(e1);
    for (int m = 0; m < 3; ++m) cell[9 * s + 3 * k + m] = (P)(g * ref_cell[9 * s + 3 * k + m]);
  }
  Q[s] = q;
}

template <class P>
__global__ void k_npt_aniso_atom_pre(int64_t n, P *x, const P *p, const P *f, const P *m,
                                     const int64_t *sys, const double *scale3,
                                     const double *alpha, const double *kT, const double *dt,
                                     const double *pn, uint64_t seed, uint64_t counter) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = sys[i];
  double z[4];
  particle_noise_of(pn, seed, i, counter, z);
  const double a = alpha[s], h = dt[s], mi = m[i];
  const double pre = sqrt(2.0 * a * kT[s] * h);
  const double b = 1.0 / (1.0 + (a * h) / (2.0 * mi));
  for (int c = 0; c < 3; ++c) {
    const double sc = scale3[3 * s + c];
    const double c2 = (2.0 * sc / (sc + 1.0)) * b * h;
    const double c3 = (double)p[3 * i + c] / mi + h * (double)f[3 * i + c] / (2.0 * mi) +
                      pre * z[c] / (2.0 * mi);
    x[3 * i + c] = (P)(sc * (double)x[3 * i + c] + c2 * c3);
  }
}

template <class P>
__global__ void k_npt_aniso_cell_post(int64_t ns, const int64_t *lo, const int64_t *hi,
                                      const P *stress, const P *cell, double *eps_dot,
                                      const double *Q, const double *f_eps,
                                      const double *cell_alpha, const double *kT,
                                      const double *p_ext, const double *dt,
                                      const double *cell_noise, uint64_t seed,
                                      uint64_t counter) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const double n_at = (double)(hi[s] - lo[s]), kt = kT[s], h = dt[s], ac = cell_alpha[s];
  const double q = Q[s];
  double C[9];
  for (int k = 0; k < 9; ++k) C[k] = (double)cell[9 * s + k];
  double f1[3];
  aniso_strain_force(stress + 9 * s, C, n_at, kt, p_ext + 3 * s, f1);
  const double a = (1.0 - (ac * h) / (2.0 * q)) / (1.0 + (ac * h) / (2.0 * q));
  const double b = 1.0 / (1.0 + (ac * h) / (2.0 * q));
  const double sc = sqrt(2.0 * ac * kt * h);
  for (int k = 0; k < 3; ++k) {
    const double beta = sc * aniso_cell_noise(cell_noise, seed, s, k, counter);
    eps_dot[3 * s + k] = a * eps_dot[3 * s + k] + h * ((a * f_eps[3 * s + k]) + f1[k]) / (2.0 * q) +
                         b * beta / q;
  }
}

// Isotropic NPT Nose-Hoover (Martyna-Tuckerman-Klein; npt.py:1110-1965): the
// inner step around the force call, between the chain half steps (which run on
// the thermostat kernel).  Log-volume coordinate eps = ln(V/V0)/3, cell momentum
// p_eps with mass W; alpha = 1 + 3/(3N - 3); cell force
// F = alpha 2 KE - tr(stress) V - 3 P V (:1460-1529).  pre: p_eps += F dt/2,
// v = p_eps / W, momenta by exp(iL2) (:1402-1457), eps += v dt, cell =
// (V/V0)^(1/3) ref, positions by exp(iL1) (:1346-1399); post: momenta by exp(iL2)
// with the new forces, p_eps += F(new stress, new V) dt/2 (:1532-1639).
__device__ inline double mtk_sinhx_x(double x) {
  const double x2 = x * x, x4 = x2 * x2, x6 = x4 * x2, x8 = x4 * x4, x10 = x8 * x2;
  return 1.0 + x2 / 6.0 + x4 / 120.0 + x6 / 5040.0 + x8 / 362880.0 + x10 / 39916800.0;
}

// per system: 2 KE = sum p^2 / m over the block, fixed order (thread 0 gets it)
template <class P>
__device__ inline double block_two_ke(int64_t lo, int64_t hi, const P *p, const P *m,
                                      double *sh) {
  double acc = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const double mi = (double)m[i];
    for (int c = 0; c < 3; ++c) {
      const double pc = (double)p[3 * i + c];
      acc += pc * pc / mi;
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
  return t;
}

__device__ inline double mtk_alpha(int64_t lo, int64_t hi) {
  return 1.0 + 3.0 / (3.0 * (double)(hi - lo) - 3.0);
}

template <class P>
__global__ void __launch_bounds__(256)
    k_mtk_pre_cell(const int64_t *lo, const int64_t *hi, const P *p, const P *m,
                   const P *stress, const double *ref_cell, P *cell, double *eps,
                   double *p_eps, const double *W, const double *p_ext, const double *dt,
                   double *v_eps) {
  __shared__ double sh[256 / 32];
  const int64_t s = blockIdx.x;
  const double two_ke = block_two_ke(lo[s], hi[s], p, m, sh);
  if (threadIdx.x != 0) return;
  const double ke = 0.5 * two_ke;
  const double al = mtk_alpha(lo[s], hi[s]), h = dt[s];
  const double v0 = det3(ref_cell + 9 * s);
  const double vol = v0 * exp(3.0 * eps[s]);
  const P *st = stress + 9 * s;
  const double tr = (double)st[0] + (double)st[4] + (double)st[8];
  const double f = (al * 2.0 * ke) - (tr * vol) - (p_ext[s] * vol * 3.0);
  const double pe = p_eps[s] + (h / 2.0) * f;
  const double v = pe / W[s];
  const double e1 = eps[s] + v * h;
  const double vol1 = v0 * exp(3.0 * e1);
  const double sc = pow(vol1 / v0, 1.0 / 3.0);
  for (int k = 0; k < 9; ++k) cell[9 * s + k] = (P)(sc * ref_cell[9 * s + k]);
  p_eps[s] = pe;
  eps[s] = e1;
  v_eps[s] = v;
}

template <class P>
__global__ void k_mtk_pre_atoms(int64_t n, P *x, P *p, const P *f, const P *m,
                                const int64_t *sys, const int64_t *lo, const int64_t *hi,
                                const double *v_eps, const double *dt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = sys[i];
  const double h = dt[s], h2 = h / 2.0, v = v_eps[s], mi = (double)m[i];
  const double x2 = mtk_alpha(lo[s], hi[s]) * v * h2, x2h = x2 / 2.0;
  const double e2 = exp(-x2), e2h = exp(-x2h), s2 = mtk_sinhx_x(x2h);
  const double x1 = v * h, x1h = x1 / 2.0;
  const double e1m = exp(x1) - 1.0, e1h = exp(x1h), s1 = mtk_sinhx_x(x1h);
  for (int c = 0; c < 3; ++c) {
    const double pn = (double)p[3 * i + c] * e2 + h2 * (double)f[3 * i + c] * s2 * e2h;
    p[3 * i + c] = (P)pn;
    const double r = (double)x[3 * i + c];
    const double vel = (double)(P)pn / mi;
    x[3 * i + c] = (P)(r + (r * e1m + h * vel * e1h * s1));
  }
}

template <class P>
__global__ void k_mtk_post_atoms(int64_t n, P *p, const P *f, const int64_t *sys,
                                 const int64_t *lo, const int64_t *hi, const double *v_eps,
                                 const double *dt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = sys[i];
  const double h2 = dt[s] / 2.0;
  const double x2 = mtk_alpha(lo[s], hi[s]) * v_eps[s] * h2, x2h = x2 / 2.0;
  const double e2 = exp(-x2), e2h = exp(-x2h), s2 = mtk_sinhx_x(x2h);
  for (int c = 0; c < 3; ++c)
    p[3 * i + c] = (P)((double)p[3 * i + c] * e2 + h2 * (double)f[3 * i + c] * s2 * e2h);
}

template <class P>
__global__ void __launch_bounds__(256)
    k_mtk_post_cell(const int64_t *lo, const int64_t *hi, const P *p, const P *m,
                    const P *stress, const double *ref_cell, const double *eps, double *p_eps,
                    const double *p_ext, const double *dt) {
  __shared__ double sh[256 / 32];
  const int64_t s = blockIdx.x;
  const double two_ke = block_two_ke(lo[s], hi[s], p, m, sh);
  if (threadIdx.x != 0) return;
  const double ke = 0.5 * two_ke;
  const double al = mtk_alpha(lo[s], hi[s]), h = dt[s];
  const double vol = det3(ref_cell + 9 * s) * exp(3.0 * eps[s]);
  const P *st = stress + 9 * s;
  const double tr = (double)st[0] + (double)st[4] + (double)st[8];
  const double f = (al * 2.0 * ke) - (tr * vol) - (p_ext[s] * vol * 3.0);
  p_eps[s] = p_eps[s] + (h / 2.0) * f;
}

// Isotropic stochastic cell rescaling (C-rescale, Bernetti & Bussi 2020;
// torch_sim/integrators/npt.py:2455-2492).  One block per system: the trace of
// the instantaneous pressure tensor P = (sum_i p_i p_i^T / m_i) / V - stress
// (quantities.py:156-198), summed in FP64 in a fixed order, then the Euler step
// of lambda = sqrt(V):
//   d lambda = -(beta_T lambda / (2 tau_p)) (P0 - tr P / 3 - kT / (2 V)) dt
//              + sqrt(2) sqrt(kT beta_T dt / (4 tau_p)) z,
// the factor mu = (lambda' / lambda)^(2/3) and the cell scaled by mu.
template <class P>
__global__ void __launch_bounds__(256)
    k_crescale_iso_cell(const int64_t *lo, const int64_t *hi, const P *p, const P *m,
                        const P *stress, P *cell, const double *beta_t, const double *tau_p,
                        const double *kT, const double *p_ext, const double *dt,
                        const double *noise, uint64_t seed, uint64_t counter, double *mu) {
  __shared__ double sh[256 / 32];
  const int64_t s = blockIdx.x;
  double acc = 0.0;
  for (int64_t i = lo[s] + threadIdx.x; i < hi[s]; i += blockDim.x) {
    const double mi = (double)m[i];
    for (int c = 0; c < 3; ++c) {
      const double pc = (double)p[3 * i + c];
      acc += pc * pc / mi;
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x != 0) return;
  double two_k = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) two_k += sh[w];
  double C[9];
  for (int k = 0; k < 9; ++k) C[k] = (double)cell[9 * s + k];
  const double vol = det3(C);
  const P *st = stress + 9 * s;
  const double tr_p = two_k / vol - ((double)st[0] + (double)st[4] + (double)st[8]);
  const double kt = kT[s], h = dt[s], bt = beta_t[s], tp = tau_p[s];
  const double sqrt_vol = sqrt(vol);
  const double pre_random = sqrt(kt * bt * h / (4.0 * tp));
  const double pre = bt * sqrt_vol / (2.0 * tp);
  const double z = noise ? noise[s] : thermo_normal(seed, s, counter, 3u);
  const double change =
      -pre * (p_ext[s] - tr_p / 3.0 - kt / (2.0 * vol)) * h + sqrt(2.0) * pre_random * z;
  const double f = pow((sqrt_vol + change) / sqrt_vol, 2.0 / 3.0);
  mu[s] = f;
  for (int k = 0; k < 9; ++k) cell[9 * s + k] = (P)(f * C[k]);
}

// per atom: r <- mu r + (mu + 1/mu) p dt / (2 m), p <- p / mu
template <class P>
__global__ void k_crescale_iso_atoms(int64_t n, P *x, P *p, const P *m, const int64_t *sys,
                                     const double *dt, const double *mu) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = sys[i];
  const double f = mu[s], fi = 1.0 / f, h = dt[s], mi = (double)m[i];
  for (int c = 0; c < 3; ++c) {
    const double pc = (double)p[3 * i + c];
    x[3 * i + c] = (P)(f * (double)x[3 * i + c] + (f + fi) * pc * (0.5 * h) / mi);
    p[3 * i + c] = (P)(fi * pc);
  }
}

// Anisotropic C-rescale (npt.py:2282-2343): the volume half step, a traceless
// random per-axis deformation exp(a~ dt + c z~) with a~_k = beta_T / (3 tau_p)
// (P_kk - tr P / 3) and c = sqrt(2 beta_T kT dt / (3 tau_p)) / lambda', a second
// volume half step, and per-axis factors mu_k = d_k (lambda'' / lambda)^(2/3).
// noise [S, 5] = (volume normal, z_x, z_y, z_z, volume normal) in the reference's
// order of draws, or Philox slots 3..7.
template <class P>
__global__ void __launch_bounds__(256)
    k_crescale_aniso_cell(const int64_t *lo, const int64_t *hi, const P *p, const P *m,
                          const P *stress, P *cell, const double *beta_t, const double *tau_p,
                          const double *kT, const double *p_ext, const double *dt,
                          const double *noise, uint64_t seed, uint64_t counter, double *mu3) {
  __shared__ double sh[3][256 / 32];
  const int64_t s = blockIdx.x;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int64_t i = lo[s] + threadIdx.x; i < hi[s]; i += blockDim.x) {
    const double mi = (double)m[i];
    for (int c = 0; c < 3; ++c) {
      const double pc = (double)p[3 * i + c];
      acc[c] += pc * pc / mi;
    }
  }
  for (int c = 0; c < 3; ++c) {
    for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    if ((threadIdx.x & 31) == 0) sh[c][threadIdx.x >> 5] = acc[c];
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double two_k[3] = {0.0, 0.0, 0.0};
  for (int c = 0; c < 3; ++c)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) two_k[c] += sh[c][w];
  double C[9];
  for (int k = 0; k < 9; ++k) C[k] = (double)cell[9 * s + k];
  const double vol = det3(C);
  const P *st = stress + 9 * s;
  double pd[3];
  for (int c = 0; c < 3; ++c) pd[c] = two_k[c] / vol - (double)st[4 * c];
  const double tr_p = pd[0] + pd[1] + pd[2];
  const double kt = kT[s], h = dt[s], bt = beta_t[s], tp = tau_p[s];
  double z[5];
  for (int k = 0; k < 5; ++k)
    z[k] = noise ? noise[5 * s + k] : thermo_normal(seed, s, counter, 3u + (uint32_t)k);
  const double sqrt_vol = sqrt(vol);
  const double pre_random = sqrt(kt * bt * h / (4.0 * tp));
  const double pre = bt * sqrt_vol / (2.0 * tp);
  const double drift = -pre * (p_ext[s] - tr_p / 3.0 - kt / (2.0 * vol)) * h / 2.0;
  double lam = sqrt_vol + (drift + pre_random * z[0]);
  const double c_rand = sqrt(2.0 * bt * kt * h / (3.0 * tp)) / lam;
  const double zm = (z[1] + z[2] + z[3]) / 3.0;
  double d[3];
  for (int c = 0; c < 3; ++c)
    d[c] = exp((bt / (3.0 * tp)) * (pd[c] - tr_p / 3.0) * h + c_rand * (z[1 + c] - zm));
  lam += drift + pre_random * z[4];
  const double f = pow(lam / sqrt_vol, 2.0 / 3.0);
  for (int c = 0; c < 3; ++c) {
    const double mu = d[c] * f;
    mu3[3 * s + c] = mu;
    for (int k = 0; k < 3; ++k) cell[9 * s + 3 * c + k] = (P)(mu * C[3 * c + k]);
  }
}

// per atom and axis: r_k <- mu_k r_k + (mu_k + 1/mu_k) p_k dt / (2 m), p_k <- p_k / mu_k
template <class P>
__global__ void k_crescale_aniso_atoms(int64_t n, P *x, P *p, const P *m, const int64_t *sys,
                                       const double *dt, const double *mu3) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = sys[i];
  const double h = dt[s], mi = (double)m[i];
  for (int c = 0; c < 3; ++c) {
    const double f = mu3[3 * s + c], fi = 1.0 / f;
    const double pc = (double)p[3 * i + c];
    x[3 * i + c] = (P)(f * (double)x[3 * i + c] + (f + fi) * pc * h / (2.0 * mi));
    p[3 * i + c] = (P)(fi * pc);
  }
}

// Triclinic C-rescale (npt.py:2186-2280; average variant :2376-2452) in three
// launches: (a) one block per system sums the kinetic tensor sum_i p p^T / m in
// FP64 in a fixed order; (b) one thread per system does the 3x3 algebra
// (pressure tensor, deviatoric correction for a tensor external pressure,
// sqrt(V) half steps, matrix exponential of the traceless drive plus noise,
// Gram-Schmidt rotation to lower-triangular form, R and the momentum matrix
// inv(R)^T, cell <- cell R^T); (c) one thread per atom applies
// r <- R r + (M + R) p dt / (2 m), p <- M p.  The average variant uses the
// average kinetic pressure (3N - 3)/3 kT / V and M = I (momenta unscaled).
// noise [S, 11] = (volume normal, 3x3 normals row-major, volume normal) in the
// reference's order of draws, or Philox slots 3..13.
template <class P>
__global__ void __launch_bounds__(256)
    k_crescale_kinetic(const int64_t *lo, const int64_t *hi, const P *p, const P *m,
                       double *kin6) {
  __shared__ double sh[6][256 / 32];
  const int64_t s = blockIdx.x;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t i = lo[s] + threadIdx.x; i < hi[s]; i += blockDim.x) {
    const double mi = (double)m[i];
    const double px = (double)p[3 * i], py = (double)p[3 * i + 1], pz = (double)p[3 * i + 2];
    acc[0] += px * px / mi;
    acc[1] += py * py / mi;
    acc[2] += pz * pz / mi;
    acc[3] += px * py / mi;
    acc[4] += px * pz / mi;
    acc[5] += py * pz / mi;
  }
  for (int c = 0; c < 6; ++c) {
    for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    if ((threadIdx.x & 31) == 0) sh[c][threadIdx.x >> 5] = acc[c];
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[threadIdx.x][w];
    kin6[6 * s + threadIdx.x] = t;
  }
}

__device__ inline M3 gram_schmidt_lower(const M3 &D) {
  // columns a, b, c of D -> lower-triangular box (npt.py:2093-2126)
  double a[3], b[3], c[3];
  for (int r = 0; r < 3; ++r) {
    a[r] = D(r, 0);
    b[r] = D(r, 1);
    c[r] = D(r, 2);
  }
  auto dot = [](const double *x, const double *y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
  M3 o = m3_zero();
  o(0, 0) = sqrt(dot(a, a));
  o(1, 0) = dot(a, b) / o(0, 0);
  o(1, 1) = sqrt(dot(b, b) - o(1, 0) * o(1, 0));
  o(2, 0) = dot(a, c) / o(0, 0);
  o(2, 1) = (dot(b, c) - o(2, 0) * o(1, 0)) / o(1, 1);
  o(2, 2) = sqrt(dot(c, c) - o(2, 0) * o(2, 0) - o(2, 1) * o(2, 1));
  return o;
}

template <class P>
__global__ void k_crescale_tri_cell(int64_t ns, const int64_t *lo, const int64_t *hi,
                                    const double *kin6, const P *stress, P *cell,
                                    const double *beta_t, const double *tau_p, const double *kT,
                                    const double *p_ext, const double *p_ext_t,
                                    const double *cell0_inv, const double *vol0, const double *dt,
                                    int average, const double *noise, uint64_t seed,
                                    uint64_t counter, double *rv) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  M3 C;
  for (int k = 0; k < 9; ++k) C.a[k] = (double)cell[9 * s + k];
  const double vol = m3_det(C);
  const double kt = kT[s], h = dt[s], bt = beta_t[s], tp = tau_p[s];
  M3 Pint;
  if (average) {
    const double pref = ((3.0 * (double)(hi[s] - lo[s]) - 3.0) / 3.0) * kt / vol;
    for (int k = 0; k < 9; ++k) Pint.a[k] = (k % 4 == 0 ? pref : 0.0) - (double)stress[9 * s + k];
  } else {
    const double *q = kin6 + 6 * s;
    const double K[9] = {q[0], q[3], q[4], q[3], q[1], q[5], q[4], q[5], q[2]};
    for (int k = 0; k < 9; ++k) Pint.a[k] = K[k] / vol - (double)stress[9 * s + k];
  }
  const double trP = Pint.a[0] + Pint.a[4] + Pint.a[8];
  const double sqrt_vol = sqrt(vol);
  const double pre_random = sqrt(kt * bt * h / (4.0 * tp));
  const double pre = bt * sqrt_vol / (2.0 * tp);
  double eff = average || !p_ext_t ? p_ext[s] : 0.0;
  M3 Pdrive = Pint;
  if (!average && p_ext_t) {
    // deviatoric correction (npt.py:2145-2183)
    M3 T;
    for (int k = 0; k < 9; ++k) T.a[k] = p_ext_t[9 * s + k];
    const double hydro = (T.a[0] + T.a[4] + T.a[8]) / 3.0;
    M3 Sd = T;
    Sd.a[0] -= hydro;
    Sd.a[4] -= hydro;
    Sd.a[8] -= hydro;
    M3 Ci;
    for (int k = 0; k < 9; ++k) Ci.a[k] = cell0_inv[9 * s + k];
    const M3 sig = m3_scale(m3_mul(m3_mul(m3_T(Ci), Sd), Ci), vol0[s]);
    const M3 sym = m3_scale(m3_add(sig, m3_T(sig)), 0.5);
    const M3 Pdev = m3_scale(m3_mul(m3_mul(m3_T(C), sym), C), 1.0 / vol);
    eff = hydro + (Pdev.a[0] + Pdev.a[4] + Pdev.a[8]) / 3.0;
    Pdrive = m3_add(Pint, Pdev, 1.0, -1.0);
  }
  double z[11];
  for (int k = 0; k < 11; ++k)
    z[k] = noise ? noise[11 * s + k] : thermo_normal(seed, s, counter, 3u + (uint32_t)k);
  const double drift = -pre * (eff - trP / 3.0 - kt / (2.0 * vol)) * h / 2.0;
  double lam = sqrt_vol + (drift + pre_random * z[0]);
  const double prm = sqrt(2.0 * bt * kt * h / (3.0 * tp)) / lam;
  const double trD = Pdrive.a[0] + Pdrive.a[4] + Pdrive.a[8];
  const double trZ = z[1] + z[5] + z[9];
  M3 X;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      const double a_t = (bt / (3.0 * tp)) * (Pdrive(r, c) - (r == c ? trD / 3.0 : 0.0));
      const double zt = z[1 + 3 * r + c] - (r == c ? trZ / 3.0 : 0.0);
      X(r, c) = a_t * h + prm * zt;
    }
  const M3 D = gram_schmidt_lower(m3_expm(X));
  lam += drift + pre_random * z[10];
  const double f = pow(lam / sqrt_vol, 2.0 / 3.0);
  const M3 R = m3_scale(D, f);
  const M3 Mp = average ? m3_eye() : m3_T(m3_inv(R));
  for (int k = 0; k < 9; ++k) {
    rv[18 * s + k] = R.a[k];
    rv[18 * s + 9 + k] = Mp.a[k];
  }
  const M3 Cn = m3_mul(C, m3_T(R));
  for (int k = 0; k < 9; ++k) cell[9 * s + k] = (P)Cn.a[k];
}

template <class P>
__global__ void k_crescale_tri_atoms(int64_t n, P *x, P *p, const P *m, const int64_t *sys,
                                     const double *dt, const double *rv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = sys[i];
  const double *R = rv + 18 * s, *M = rv + 18 * s + 9;
  const double h = dt[s], mi = (double)m[i];
  const double r0[3] = {(double)x[3 * i], (double)x[3 * i + 1], (double)x[3 * i + 2]};
  const double p0[3] = {(double)p[3 * i], (double)p[3 * i + 1], (double)p[3 * i + 2]};
  for (int a = 0; a < 3; ++a) {
    double rr = 0.0, mp = 0.0, np = 0.0;
    for (int b = 0; b < 3; ++b) {
      rr += R[3 * a + b] * r0[b];
      mp += (M[3 * a + b] + R[3 * a + b]) * p0[b];
      np += M[3 * a + b] * p0[b];
    }
    x[3 * i + a] = (P)(rr + mp * h / (2.0 * mi));
    p[3 * i + a] = (P)np;
  }
}

}  // namespace tsb

using namespace tsb;

extern "C" size_t tsb_npt_workspace_size(int64_t n_systems) {
  Carver c(nullptr, (size_t)-1);
  NptWork w;
  carve_npt(c, w, n_systems);
  return c.off + 256;
}

extern "C" int tsb_npt_langevin_iso_pre(
    void *positions, const void *momenta, const void *forces, const void *masses,
    const int64_t *system_idx, int64_t n_atoms, int64_t n_systems, int dtype,
    const void *stress, const double *reference_cell, void *cell, double *eps,
    const double *eps_dot, double *cell_masses, double *f_eps, const double *alpha,
    const double *cell_alpha, const double *b_tau, const double *kT, const double *p_ext,
    const double *dt, const double *cell_noise, const double *particle_noise, uint64_t seed,
    uint64_t counter, void *workspace, size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !positions || !momenta || !forces || !masses ||
      !system_idx || !stress || !reference_cell || !cell || !eps || !eps_dot || !cell_masses ||
      !f_eps || !alpha || !cell_alpha || !b_tau || !kT || !p_ext || !dt)
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  NptWork w;
  carve_npt(c, w, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(w.lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(w.hi, 0, sizeof(int64_t) * n_systems, st);
  k_npt_bounds<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, w.lo, w.hi);
#define TSB_NPT_PRE(P)                                                                        \
  k_npt_cell_pre<P><<<grid_for(n_systems), kBlock, 0, st>>>(                                 \
      n_systems, w.lo, w.hi, (const P *)stress, reference_cell, (P *)cell, eps, eps_dot,      \
      cell_masses, f_eps, w.scale, cell_alpha, b_tau, kT, p_ext, dt, cell_noise, seed,         \
      counter);                                                                              \
  k_npt_atom_pre<P><<<grid_for(n_atoms), kBlock, 0, st>>>(                                   \
      n_atoms, (P *)positions, (const P *)momenta, (const P *)forces, (const P *)masses,     \
      system_idx, w.scale, alpha, kT, dt, particle_noise, seed, counter);
  if (dtype == TSB_F64) {
    TSB_NPT_PRE(double)
  } else {
    TSB_NPT_PRE(float)
  }
#undef TSB_NPT_PRE
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_npt_langevin_iso_post(
    void *momenta, const void *masses, const void *forces_old, const void *forces,
    const int64_t *system_idx, int64_t n_atoms, int64_t n_systems, int dtype,
    const void *stress, const double *reference_cell, const double *eps, double *eps_dot,
    const double *cell_masses, const double *f_eps, const double *alpha,
    const double *cell_alpha, const double *kT, const double *p_ext, const double *dt,
    const double *cell_noise, const double *particle_noise, uint64_t seed, uint64_t counter,
    void *workspace, size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !momenta || !masses || !forces_old || !forces ||
      !system_idx || !stress || !reference_cell || !eps || !eps_dot || !cell_masses ||
      !f_eps || !alpha || !cell_alpha || !kT || !p_ext || !dt)
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  NptWork w;
  carve_npt(c, w, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(w.lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(w.hi, 0, sizeof(int64_t) * n_systems, st);
  k_npt_bounds<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, w.lo, w.hi);
#define TSB_NPT_POST(P)                                                                       \
  k_npt_cell_post<P><<<grid_for(n_systems), kBlock, 0, st>>>(                                \
      n_systems, w.lo, w.hi, (const P *)stress, reference_cell, eps, eps_dot, cell_masses,    \
      f_eps, cell_alpha, kT, p_ext, dt, cell_noise, seed, counter);                          \
  k_npt_atom_post<P><<<grid_for(n_atoms), kBlock, 0, st>>>(                                  \
      n_atoms, (P *)momenta, (const P *)masses, (const P *)forces_old, (const P *)forces,    \
      system_idx, alpha, kT, dt, particle_noise, seed, counter);
  if (dtype == TSB_F64) {
    TSB_NPT_POST(double)
  } else {
    TSB_NPT_POST(float)
  }
#undef TSB_NPT_POST
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_npt_crescale_iso(void *positions, void *momenta, const void *masses,
                                    const int64_t *system_idx, int64_t n_atoms,
                                    int64_t n_systems, int dtype, const void *stress,
                                    void *cell, const double *compressibility,
                                    const double *tau_p, const double *kT, const double *p_ext,
                                    const double *dt, const double *noise, uint64_t seed,
                                    uint64_t counter, void *workspace, size_t workspace_bytes,
                                    void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !positions || !momenta || !masses || !system_idx ||
      !stress || !cell || !compressibility || !tau_p || !kT || !p_ext || !dt)
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  NptWork w;
  carve_npt(c, w, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(w.lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(w.hi, 0, sizeof(int64_t) * n_systems, st);
  k_npt_bounds<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, w.lo, w.hi);
#define TSB_CRESCALE(P)                                                                      \
  k_crescale_iso_cell<P><<<(unsigned)n_systems, 256, 0, st>>>(                               \
      w.lo, w.hi, (const P *)momenta, (const P *)masses, (const P *)stress, (P *)cell,       \
      compressibility, tau_p, kT, p_ext, dt, noise, seed, counter, w.scale);                 \
  k_crescale_iso_atoms<P><<<grid_for(n_atoms), kBlock, 0, st>>>(                             \
      n_atoms, (P *)positions, (P *)momenta, (const P *)masses, system_idx, dt, w.scale);
  if (dtype == TSB_F64) {
    TSB_CRESCALE(double)
  } else {
    TSB_CRESCALE(float)
  }
#undef TSB_CRESCALE
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_npt_crescale_aniso(void *positions, void *momenta, const void *masses,
                                      const int64_t *system_idx, int64_t n_atoms,
                                      int64_t n_systems, int dtype, const void *stress,
                                      void *cell, const double *compressibility,
                                      const double *tau_p, const double *kT,
                                      const double *p_ext, const double *dt, const double *noise,
                                      uint64_t seed, uint64_t counter, void *workspace,
                                      size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !positions || !momenta || !masses || !system_idx ||
      !stress || !cell || !compressibility || !tau_p || !kT || !p_ext || !dt)
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  NptWork w;
  carve_npt(c, w, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(w.lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(w.hi, 0, sizeof(int64_t) * n_systems, st);
  k_npt_bounds<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, w.lo, w.hi);
#define TSB_CRESCALE_A(P)                                                                    \
  k_crescale_aniso_cell<P><<<(unsigned)n_systems, 256, 0, st>>>(                             \
      w.lo, w.hi, (const P *)momenta, (const P *)masses, (const P *)stress, (P *)cell,       \
      compressibility, tau_p, kT, p_ext, dt, noise, seed, counter, w.scale3);                \
  k_crescale_aniso_atoms<P><<<grid_for(n_atoms), kBlock, 0, st>>>(                           \
      n_atoms, (P *)positions, (P *)momenta, (const P *)masses, system_idx, dt, w.scale3);
  if (dtype == TSB_F64) {
    TSB_CRESCALE_A(double)
  } else {
    TSB_CRESCALE_A(float)
  }
#undef TSB_CRESCALE_A
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_npt_crescale_tri(void *positions, void *momenta, const void *masses,
                                    const int64_t *system_idx, int64_t n_atoms,
                                    int64_t n_systems, int dtype, const void *stress,
                                    void *cell, const double *compressibility,
                                    const double *tau_p, const double *kT, const double *p_ext,
                                    const double *p_ext_tensor, const double *initial_cell_inv,
                                    const double *initial_volume, const double *dt, int average,
                                    const double *noise, uint64_t seed, uint64_t counter,
                                    void *workspace, size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !positions || !momenta || !masses || !system_idx ||
      !stress || !cell || !compressibility || !tau_p || !kT || !p_ext || !dt)
    return TSB_ERR_INVALID_ARG;
  if (p_ext_tensor && (average || !initial_cell_inv || !initial_volume))
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  NptWork w;
  carve_npt(c, w, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(w.lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(w.hi, 0, sizeof(int64_t) * n_systems, st);
  k_npt_bounds<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, w.lo, w.hi);
#define TSB_CRESCALE_T(P)                                                                    \
  if (!average)                                                                              \
    k_crescale_kinetic<P><<<(unsigned)n_systems, 256, 0, st>>>(                              \
        w.lo, w.hi, (const P *)momenta, (const P *)masses, w.kin6);                          \
  k_crescale_tri_cell<P><<<grid_for(n_systems, 64), 64, 0, st>>>(                            \
      n_systems, w.lo, w.hi, w.kin6, (const P *)stress, (P *)cell, compressibility, tau_p,   \
      kT, p_ext, p_ext_tensor, initial_cell_inv, initial_volume, dt, average, noise, seed,   \
      counter, w.rv);                                                                        \
  k_crescale_tri_atoms<P><<<grid_for(n_atoms), kBlock, 0, st>>>(                             \
      n_atoms, (P *)positions, (P *)momenta, (const P *)masses, system_idx, dt, w.rv);
  if (dtype == TSB_F64) {
    TSB_CRESCALE_T(double)
  } else {
    TSB_CRESCALE_T(float)
  }
#undef TSB_CRESCALE_T
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_npt_langevin_aniso_pre(
    void *positions, const void *momenta, const void *forces, const void *masses,
    const int64_t *system_idx, int64_t n_atoms, int64_t n_systems, int dtype,
    const void *stress, const double *reference_cell, void *cell, double *eps,
    const double *eps_dot, double *cell_masses, double *f_eps, const double *alpha,
    const double *cell_alpha, const double *b_tau, const double *kT, const double *p_ext,
    const double *dt, const double *cell_noise, const double *particle_noise, uint64_t seed,
    uint64_t counter, void *workspace, size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !positions || !momenta || !forces || !masses ||
      !system_idx || !stress || !reference_cell || !cell || !eps || !eps_dot || !cell_masses ||
      !f_eps || !alpha || !cell_alpha || !b_tau || !kT || !p_ext || !dt)
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  NptWork w;
  carve_npt(c, w, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(w.lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(w.hi, 0, sizeof(int64_t) * n_systems, st);
  k_npt_bounds<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, w.lo, w.hi);
#define TSB_NPTA_PRE(P)                                                                       \
  k_npt_aniso_cell_pre<P><<<grid_for(n_systems), kBlock, 0, st>>>(                           \
      n_systems, w.lo, w.hi, (const P *)stress, reference_cell, (P *)cell, eps, eps_dot,      \
      cell_masses, f_eps, w.scale3, cell_alpha, b_tau, kT, p_ext, dt, cell_noise, seed,       \
      counter);                                                                              \
  k_npt_aniso_atom_pre<P><<<grid_for(n_atoms), kBlock, 0, st>>>(                             \
      n_atoms, (P *)positions, (const P *)momenta, (const P *)forces, (const P *)masses,     \
      system_idx, w.scale3, alpha, kT, dt, particle_noise, seed, counter);
  if (dtype == TSB_F64) {
    TSB_NPTA_PRE(double)
  } else {
    TSB_NPTA_PRE(float)
  }
#undef TSB_NPTA_PRE
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_npt_langevin_aniso_post(
    void *momenta, const void *masses, const void *forces_old, const void *forces,
    const int64_t *system_idx, int64_t n_atoms, int64_t n_systems, int dtype,
    const void *stress, const void *cell, double *eps_dot, const double *cell_masses,
    const double *f_eps, const double *alpha, const double *cell_alpha, const double *kT,
    const double *p_ext, const double *dt, const double *cell_noise,
    const double *particle_noise, uint64_t seed, uint64_t counter, void *workspace,
    size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !momenta || !masses || !forces_old || !forces ||
      !system_idx || !stress || !cell || !eps_dot || !cell_masses || !f_eps || !alpha ||
      !cell_alpha || !kT || !p_ext || !dt)
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  NptWork w;
  carve_npt(c, w, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(w.lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(w.hi, 0, sizeof(int64_t) * n_systems, st);
  k_npt_bounds<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, w.lo, w.hi);
#define TSB_NPTA_POST(P)                                                                      \
  k_npt_aniso_cell_post<P><<<grid_for(n_systems), kBlock, 0, st>>>(                          \
      n_systems, w.lo, w.hi, (const P *)stress, (const P *)cell, eps_dot, cell_masses, f_eps, \
      cell_alpha, kT, p_ext, dt, cell_noise, seed, counter);                                 \
  k_npt_atom_post<P><<<grid_for(n_atoms), kBlock, 0, st>>>(                                  \
      n_atoms, (P *)momenta, (const P *)masses, (const P *)forces_old, (const P *)forces,    \
      system_idx, alpha, kT, dt, particle_noise, seed, counter);
  if (dtype == TSB_F64) {
    TSB_NPTA_POST(double)
  } else {
    TSB_NPTA_POST(float)
  }
#undef TSB_NPTA_POST
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_npt_nh_iso_pre(void *positions, void *momenta, const void *forces,
                                  const void *masses, const int64_t *system_idx,
                                  int64_t n_atoms, int64_t n_systems, int dtype,
                                  const void *stress, const double *reference_cell, void *cell,
                                  double *eps, double *p_eps, const double *cell_mass,
                                  const double *p_ext, const double *dt, double *v_eps,
                                  void *workspace, size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !positions || !momenta || !forces || !masses ||
      !system_idx || !stress || !reference_cell || !cell || !eps || !p_eps || !cell_mass ||
      !p_ext || !dt || !v_eps)
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  NptWork w;
  carve_npt(c, w, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(w.lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(w.hi, 0, sizeof(int64_t) * n_systems, st);
  k_npt_bounds<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, w.lo, w.hi);
#define TSB_MTK_PRE(P)                                                                       \
  k_mtk_pre_cell<P><<<(unsigned)n_systems, 256, 0, st>>>(                                    \
      w.lo, w.hi, (const P *)momenta, (const P *)masses, (const P *)stress, reference_cell,  \
      (P *)cell, eps, p_eps, cell_mass, p_ext, dt, v_eps);                                   \
  k_mtk_pre_atoms<P><<<grid_for(n_atoms), kBlock, 0, st>>>(                                  \
      n_atoms, (P *)positions, (P *)momenta, (const P *)forces, (const P *)masses,           \
      system_idx, w.lo, w.hi, v_eps, dt);
  if (dtype == TSB_F64) {
    TSB_MTK_PRE(double)
  } else {
    TSB_MTK_PRE(float)
  }
#undef TSB_MTK_PRE
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_npt_nh_iso_post(void *momenta, const void *forces, const void *masses,
                                   const int64_t *system_idx, int64_t n_atoms,
                                   int64_t n_systems, int dtype, const void *stress,
                                   const double *reference_cell, const double *eps,
                                   double *p_eps, const double *p_ext, const double *dt,
                                   const double *v_eps, void *workspace,
                                   size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !momenta || !forces || !masses || !system_idx ||
      !stress || !reference_cell || !eps || !p_eps || !p_ext || !dt || !v_eps)
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  NptWork w;
  carve_npt(c, w, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(w.lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(w.hi, 0, sizeof(int64_t) * n_systems, st);
  k_npt_bounds<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, w.lo, w.hi);
#define TSB_MTK_POST(P)                                                                      \
  k_mtk_post_atoms<P><<<grid_for(n_atoms), kBlock, 0, st>>>(                                 \
      n_atoms, (P *)momenta, (const P *)forces, system_idx, w.lo, w.hi, v_eps, dt);          \
  k_mtk_post_cell<P><<<(unsigned)n_systems, 256, 0, st>>>(                                   \
      w.lo, w.hi, (const P *)momenta, (const P *)masses, (const P *)stress, reference_cell,  \
      eps, p_eps, p_ext, dt);
  if (dtype == TSB_F64) {
    TSB_MTK_POST(double)
  } else {
    TSB_MTK_POST(float)
  }
#undef TSB_MTK_POST
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}
