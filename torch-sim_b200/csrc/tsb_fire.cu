// Batched FIRE (ASE and velocity-Verlet flavours) with the Frechet cell filter.
//
//   tsb_fire_ase_pre   <- torch_sim/optimizers/fire.py:288-485 (_ase_fire_step up to
//                         the model call), with the Frechet position/cell update of
//                         fire.py:400-483 and _clamp_deform_grad_log
//                         (cell_filters.py:26-60)
//   tsb_fire_vv_pre / tsb_fire_vv_post <- fire.py:179-285 (_vv_fire_step)
//   tsb_frechet_cell_forces <- cell_filters.py:353-391 (Frechet branch) and the
//                         initial cell forces of frechet_cell_filter_init (:230-284)
//   tsb_fire_converged <- runners.py:501-538 + quantities.py:327-342, as a device
//                         mask: converged systems are frozen (skipped by every
//                         kernel, including the force kernel's sys_active input)
//
// One block per system for the per-system reductions (FP64), one thread per
// system for the 3x3 cell algebra.  The contraction of the nine Frechet
// directions with the cell gradient, sum_ab L(A, E_mn)_ab G_ab, equals the
// adjoint derivative L(A^T, G)_mn, so one Frechet evaluation replaces nine.
#include "tsb_common.cuh"
#include "tsb_mat3.cuh"

namespace tsb {

constexpr int kFireThreads = 256;
constexpr int kFireScr = 21;  // per-system scratch: drs, sc, fac, Finv[9], Fa[9]

struct FireHyper {
  double dt_max, f_inc, f_dec, alpha_start, f_alpha, max_step, eps;
  int n_min;
};

template <class P>
struct FireArgs {
  int cell_filter;  // 0 none, 1 Frechet
  P *x, *v;
  const P *f, *m;
  P *dt, *alpha;
  int32_t *n_pos;
  P *cell;                 // [S,9] column-vector cell (state.cell)
  const P *ref_cell;       // [S,9] column-vector reference cell
  const P *cell_factor;    // [S]
  P *cell_pos, *cell_vel;  // [S,9]
  const P *cell_force;     // [S,9]
  const P *cell_mass;      // [S]
  const uint8_t *active;   // [S] or null
  const int64_t *lo, *hi;
  FireHyper h;
};

__device__ inline void block_sum3(double &a, double &b, double &c, double *sh) {
  // sh: >= 3 * 32 doubles
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (l == 0) {
    sh[w] = a;
    sh[32 + w] = b;
    sh[64 + w] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0, y = 0, z = 0;
    for (int k = 0; k < nw; ++k) {
      x += sh[k];
      y += sh[32 + k];
      z += sh[64 + k];
    }
    sh[96] = x;
    sh[97] = y;
    sh[98] = z;
  }
  __syncthreads();
  a = sh[96];
  b = sh[97];
  c = sh[98];
  __syncthreads();
}

template <class P>
__device__ inline M3 load_m3(const P *p) {
  M3 m;
#pragma unroll
  for (int k = 0; k < 9; ++k) m.a[k] = (double)p[k];
  return m;
}

template <class P>
__device__ inline void store_m3(P *p, const M3 &m) {
#pragma unroll
  for (int k = 0; k < 9; ++k) p[k] = (P)m.a[k];
}

// does any atom have a velocity without NaN?  (the ASE step skips mixing on the
// first step, when every velocity of the batch is NaN: fire.py:303-310)  Warps
// stride over the atoms and stop as soon as one of them has found one, so the
// usual case (finite velocities) costs one load per warp.
template <class P>
__global__ void k_any_finite_v(const P *v, int64_t n, int32_t *found) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i - threadIdx.x % 32 < n;
       i += stride) {
    if (*(volatile int32_t *)found) return;
    const bool fin = i < n && !(isnan((double)v[3 * i]) || isnan((double)v[3 * i + 1]) ||
                                isnan((double)v[3 * i + 2]));
    if (__any_sync(0xffffffffu, fin)) {
      if ((threadIdx.x & 31) == 0) atomicExch(found, 1);
      return;
    }
  }
}

// ASE-FIRE step in three launches: (a) one block per system for the power,
// mixing and velocity step with its FP64 sums, (b) one thread per system for the
// cell velocity, the max_step factor and the Frechet cell update (3x3 algebra,
// kept out of (a) so that the per-system blocks stay light on registers), (c) one
// thread per atom for the position update.  (a) reads the system's atoms twice:
// once for the power and norms (velocities with NaN read as 0), once for the
// mixing, the Euler step and the step-length sum.
template <class P>
__global__ void __launch_bounds__(kFireThreads) k_fire_ase_vel(FireArgs<P> A,
                                                               const int32_t *any_finite,
                                                               double *scr) {
  __shared__ double sh[100];
  __shared__ double s_alpha, s_vs, s_fs, s_dt;
  __shared__ int s_pos;
  const int s = blockIdx.x;
  if (A.active && !A.active[s]) return;
  const int64_t a0 = A.lo[s], a1 = A.hi[s];
  const int tid = threadIdx.x;
  const bool cellf = A.cell_filter != 0;
  const FireHyper &h = A.h;
  // NaN velocities read as 0 (nan_to_num_, fire.py:304-307)
  auto vel = [&](int64_t j) {
    const double x = (double)A.v[j];
    return isnan(x) ? 0.0 : x;
  };
  const bool all_nan = (*any_finite == 0);
  if (!all_nan) {
    double pw = 0, vv = 0, ff = 0;
    for (int64_t i = a0 + tid; i < a1; i += blockDim.x)
      for (int k = 0; k < 3; ++k) {
        const double fk = (double)A.f[3 * i + k], vk = vel(3 * i + k);
        pw += fk * vk;
        vv += vk * vk;
        ff += fk * fk;
      }
    block_sum3(pw, vv, ff, sh);
    if (tid == 0) {
      if (cellf)
        for (int k = 0; k < 9; ++k) {
          if (isnan((double)A.cell_vel[9 * s + k])) A.cell_vel[9 * s + k] = (P)0;
          const double cf = (double)A.cell_force[9 * s + k], cv = (double)A.cell_vel[9 * s + k];
          pw += cf * cv;
          vv += cv * cv;
          ff += cf * cf;
        }
      const bool pos = pw > 0.0;
      double dt = (double)A.dt[s], alpha = (double)A.alpha[s];
      int np = A.n_pos[s];
      // ASE ordering (fire.py:339-346): increase test before counting
      if (np > h.n_min && pos) {
        dt = fmin((double)(P)(dt * h.f_inc), h.dt_max);
        alpha = alpha * h.f_alpha;
      }
      if (pos) np += 1;
      if (!pos) {
        dt = dt * h.f_dec;
        alpha = h.alpha_start;
        np = 0;
      }
      A.dt[s] = (P)dt;
      A.alpha[s] = (P)alpha;
      A.n_pos[s] = np;
      const double vsc = sqrt(vv), fsc = sqrt(ff);
      if (cellf)
        for (int k = 0; k < 9; ++k) {
          const double cv = (double)A.cell_vel[9 * s + k];
          const double mix = (double)A.cell_force[9 * s + k] / (fsc + h.eps) * vsc;
          A.cell_vel[9 * s + k] = (P)(pos ? (1.0 - (double)(P)alpha) * cv + (double)(P)alpha * mix
                                          : 0.0);
        }
      s_pos = pos;
      s_alpha = (double)(P)alpha;
      s_vs = vsc;
      s_fs = fsc;
      s_dt = (double)(P)dt;
    }
  } else if (tid == 0) {
    if (cellf)
      for (int k = 0; k < 9; ++k)
        if (isnan((double)A.cell_vel[9 * s + k])) A.cell_vel[9 * s + k] = (P)0;
    s_dt = (double)A.dt[s];
  }
  __syncthreads();
  // mixing (fire.py:348-367), then the Euler step (no mass, ASE) and the sum for
  // the max_step clamp (fire.py:369-391)
  const double al = all_nan ? 0.0 : s_alpha;
  const double ratio = all_nan ? 0.0 : s_vs / (s_fs + h.eps);
  const bool pos = all_nan ? false : s_pos;
  const double dts = s_dt;
  double drs = 0, dummy1 = 0, dummy2 = 0;
  for (int64_t i = a0 + tid; i < a1; i += blockDim.x)
    for (int k = 0; k < 3; ++k) {
      const double fk = (double)A.f[3 * i + k];
      double vk = vel(3 * i + k);
      if (!all_nan) vk = (double)(P)(pos ? (1.0 - al) * vk + al * (fk * ratio) : 0.0);
      vk = (double)(P)(vk + fk * dts);
      A.v[3 * i + k] = (P)vk;
      const double d = (double)(P)(vk * dts);
      drs += d * d;
    }
  __syncthreads();
  block_sum3(drs, dummy1, dummy2, sh);
  if (tid == 0) scr[kFireScr * s] = drs;
}

template <class P>
__global__ void k_fire_ase_cell(FireArgs<P> A, int64_t ns, double *scr) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns || (A.active && !A.active[s])) return;
  const bool cellf = A.cell_filter != 0;
  const FireHyper &h = A.h;
  const double dts = (double)A.dt[s];
  double drs = scr[kFireScr * s];
  double *o = scr + kFireScr * s;
  {
    double dc[9];
    if (cellf)
      for (int k = 0; k < 9; ++k) {
        const double cv = (double)(P)((double)A.cell_vel[9 * s + k] +
                                      (double)A.cell_force[9 * s + k] * dts);
        A.cell_vel[9 * s + k] = (P)cv;
        dc[k] = (double)(P)(cv * dts);
        drs += dc[k] * dc[k];
      }
    const double sc = sqrt(drs);
    o[1] = sc;
    o[2] = sc > h.max_step ? h.max_step / (sc + h.eps) : 1.0;
    if (cellf) {
      // Frechet cell update (fire.py:400-470)
      const M3 ref = load_m3(A.ref_cell + 9 * s);
      const M3 cell = load_m3(A.cell + 9 * s);
      const M3 refi = m3_inv(ref);
      const M3 Fd = m3_mul(cell, refi);  // deform_grad(ref^T, cell^T)
      const M3 Finv = m3_inv(Fd);
      const double cf = (double)A.cell_factor[s];
      M3 cp, lg;
      bool big = false;
      for (int k = 0; k < 9; ++k) {
        const double d = sc > h.max_step ? h.max_step * dc[k] / (sc + h.eps) : dc[k];
        cp.a[k] = (double)A.cell_pos[9 * s + k] + d;
        lg.a[k] = cp.a[k] / cf;
        big = big || fabs(lg.a[k]) > 2.0;
      }
      if (big)
        for (int k = 0; k < 9; ++k) {
          lg.a[k] = fmin(fmax(lg.a[k], -2.0), 2.0);
          cp.a[k] = lg.a[k] * cf;
        }
      const M3 Fn = m3_expm(lg);
      const M3 new_cell = m3_mul(Fn, ref);
      store_m3(A.cell + 9 * s, new_cell);
      const M3 Fa = m3_mul(load_m3(A.cell + 9 * s), refi);
      store_m3(A.cell_pos + 9 * s, m3_scale(m3_logm(Fa), cf));
      for (int k = 0; k < 9; ++k) {
        o[3 + k] = Finv.a[k];
        o[12 + k] = Fa.a[k];
      }
    }
  }
}

template <class P>
__global__ void k_fire_ase_pos(FireArgs<P> A, int64_t n, const int64_t *system_idx,
                               const double *scr) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = system_idx[i];
  if (A.active && !A.active[s]) return;
  const bool cellf = A.cell_filter != 0;
  const FireHyper &h = A.h;
  const double *o = scr + kFireScr * s;
  const double fac = o[2];
  const double dtu = (double)A.dt[s];
  const double *s_Finv = o + 3, *s_Fa = o + 12;
  const double s_sc = o[1];
  {
    double d[3], x[3];
    for (int k = 0; k < 3; ++k) {
      const double dk = (double)(P)((double)A.v[3 * i + k] * dtu);
      d[k] = fac != 1.0 ? h.max_step * dk / (s_sc + h.eps) : dk;
      x[k] = (double)A.x[3 * i + k];
    }
    if (cellf) {
      double fr[3];
      for (int r = 0; r < 3; ++r)
        fr[r] = s_Finv[3 * r] * x[0] + s_Finv[3 * r + 1] * x[1] + s_Finv[3 * r + 2] * x[2] + d[r];
      for (int r = 0; r < 3; ++r)
        A.x[3 * i + r] = (P)(s_Fa[3 * r] * fr[0] + s_Fa[3 * r + 1] * fr[1] + s_Fa[3 * r + 2] * fr[2]);
    } else {
      for (int k = 0; k < 3; ++k) A.x[3 * i + k] = (P)(x[k] + d[k]);
    }
  }
}

// VV-FIRE first half: NaN rows -> 0, half kick, drift (fire.py:196-219)
template <class P>
__global__ void k_fire_vv_pre(FireArgs<P> A, int64_t n_atoms, const int64_t *system_idx) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_atoms) return;
  const int64_t s = system_idx[i];
  if (A.active && !A.active[s]) return;
  P *v = A.v + 3 * i;
  if (isnan((double)v[0]) || isnan((double)v[1]) || isnan((double)v[2])) v[0] = v[1] = v[2] = 0;
  const double dt = (double)A.dt[s];
  const double m = (double)A.m[i];
  for (int k = 0; k < 3; ++k) {
    const double vk = (double)(P)((double)v[k] + (double)(P)(0.5 * dt) * (double)A.f[3 * i + k] / m);
    v[k] = (P)vk;
    A.x[3 * i + k] = (P)((double)A.x[3 * i + k] + dt * vk);
  }
}

// VV-FIRE second half after the model call: half kick, power, dt/alpha/n_pos,
// mixing (fire.py:228-285)
template <class P>
__global__ void __launch_bounds__(kFireThreads) k_fire_vv_post(FireArgs<P> A) {
  __shared__ double sh[100];
  __shared__ double s_alpha, s_ratio;
  __shared__ int s_pos;
  const int s = blockIdx.x;
  if (A.active && !A.active[s]) return;
  const int64_t a0 = A.lo[s], a1 = A.hi[s];
  const int tid = threadIdx.x;
  const bool cellf = A.cell_filter != 0;
  const FireHyper &h = A.h;
  const double dt = (double)A.dt[s];
  double pw = 0, vv = 0, ff = 0;
  for (int64_t i = a0 + tid; i < a1; i += blockDim.x) {
    const double m = (double)A.m[i];
    for (int k = 0; k < 3; ++k) {
      const double fk = (double)A.f[3 * i + k];
      const double vk = (double)(P)((double)A.v[3 * i + k] + (double)(P)(0.5 * dt) * fk / m);
      A.v[3 * i + k] = (P)vk;
      pw += fk * vk;
      vv += vk * vk;
      ff += fk * fk;
    }
  }
  block_sum3(pw, vv, ff, sh);
  if (tid == 0) {
    double cvn[9];
    if (cellf) {
      bool any_nan = false;
      for (int k = 0; k < 9; ++k) any_nan = any_nan || isnan((double)A.cell_vel[9 * s + k]);
      const double cm = (double)A.cell_mass[s];
      for (int k = 0; k < 9; ++k) {
        const double cf = (double)A.cell_force[9 * s + k];
        const double cv0 = any_nan ? 0.0 : (double)A.cell_vel[9 * s + k];
        cvn[k] = (double)(P)(cv0 + (double)(P)(0.5 * dt) * cf / cm);
        pw += cf * cvn[k];
      }
    }
    const bool pos = pw > 0.0;
    double dtn = dt, alpha = (double)A.alpha[s];
    int np = A.n_pos[s];
    // VV ordering (fire.py:231-240): count first, then the increase test
    if (pos) np += 1;
    if (np > h.n_min && pos) {
      dtn = fmin((double)(P)(dtn * h.f_inc), h.dt_max);
      alpha = alpha * h.f_alpha;
    }
    if (!pos) {
      dtn = dtn * h.f_dec;
      alpha = h.alpha_start;
      np = 0;
    }
    A.dt[s] = (P)dtn;
    A.alpha[s] = (P)alpha;
    A.n_pos[s] = np;
    if (cellf)
      for (int k = 0; k < 9; ++k) {
        const double cf = (double)A.cell_force[9 * s + k];
        vv += cvn[k] * cvn[k];
        ff += cf * cf;
      }
    const double vsc = sqrt(vv), fsc = sqrt(ff);
    const double al = (double)(P)alpha;
    if (cellf)
      for (int k = 0; k < 9; ++k) {
        const double mix = (double)A.cell_force[9 * s + k] / (fsc + h.eps) * vsc;
        A.cell_vel[9 * s + k] = (P)(pos ? (1.0 - al) * cvn[k] + al * mix : 0.0);
      }
    s_pos = pos;
    s_alpha = al;
    s_ratio = vsc / (fsc + h.eps);
  }
  __syncthreads();
  const bool pos = s_pos;
  const double al = s_alpha, ratio = s_ratio;
  for (int64_t i = a0 + tid; i < a1; i += blockDim.x)
    for (int k = 0; k < 3; ++k) {
      const double vk = (double)A.v[3 * i + k];
      const double mix = (double)A.f[3 * i + k] * ratio;
      A.v[3 * i + k] = (P)(pos ? (1.0 - al) * vk + al * mix : 0.0);
    }
}

// Frechet cell forces, one thread per system (cell_filters.py:353-391; with
// `init`, the initial cell forces of frechet_cell_filter_init, :255-269)
template <class P>
__global__ void k_frechet_cell_forces(P *cell_force, const P *stress, const P *cell,
                                      const P *ref_cell, const P *pressure,
                                      const P *cell_factor, int64_t ns, int init,
                                      const uint8_t *active) {
  int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  if (active && !active[s]) return;
  const M3 C = load_m3(cell + 9 * s);
  const M3 R = load_m3(ref_cell + 9 * s);
  const double vol = m3_det(C);  // torch.linalg.det(state.cell): signed
  const M3 virial = m3_scale(m3_add(load_m3(stress + 9 * s), load_m3(pressure + 9 * s)), -vol);
  const M3 Fd = m3_mul(C, m3_inv(R));
  const M3 ucf = m3_mul(virial, m3_inv(m3_T(Fd)));
  const double cf = (double)cell_factor[s];
  M3 out;
  if (init) {
    out = m3_scale(ucf, 1.0 / cf);
  } else {
    M3 lg = m3_logm(Fd);
    for (int k = 0; k < 9; ++k) lg.a[k] = fmin(fmax(lg.a[k], -2.0), 2.0);
    M3 E_unused, L;
    m3_expm_frechet(m3_T(lg), ucf, &E_unused, &L);
    out = m3_scale(L, 1.0 / cf);
  }
  store_m3(cell_force + 9 * s, out);
}

// max |F_i| per system below fmax (and, with cell forces, the row norms of the
// cell force): freeze converged systems and count the still-active ones.
template <class P>
__global__ void k_fire_converged(const P *f, const int64_t *lo, const int64_t *hi,
                                 const P *cell_force, double f_tol, uint8_t *active,
                                 int32_t *n_active) {
  __shared__ double sh[100];
  const int s = blockIdx.x;
  if (!active[s]) return;
  double mx = 0.0;
  for (int64_t i = lo[s] + threadIdx.x; i < hi[s]; i += blockDim.x) {
    const double a = (double)f[3 * i], b = (double)f[3 * i + 1], c = (double)f[3 * i + 2];
    mx = fmax(mx, sqrt(a * a + b * b + c * c));
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x != 0) return;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) mx = fmax(mx, sh[k]);
  bool conv = mx < f_tol;
  if (cell_force) {
    double cm = 0.0;
    for (int r = 0; r < 3; ++r) {
      const P *q = cell_force + 9 * s + 3 * r;
      cm = fmax(cm, sqrt((double)q[0] * q[0] + (double)q[1] * q[1] + (double)q[2] * q[2]));
    }
    conv = conv && cm < f_tol;
  }
  if (conv) active[s] = 0;
  else atomicAdd(n_active, 1);
}

__global__ void k_bounds(const int64_t *sys, int64_t n, int64_t *lo, int64_t *hi) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t s = sys[i];
  if (i == 0 || sys[i - 1] != s) lo[s] = i;
  if (i == n - 1 || sys[i + 1] != s) hi[s] = i + 1;
}

struct FireWork {
  int64_t *lo, *hi;
  int32_t *counter;
  double *scr;  // [kFireScr * S] per-system values passed between the ASE launches
};

static void carve_fire(Carver &c, FireWork &w, int64_t ns) {
  w.lo = c.take<int64_t>(ns);
  w.hi = c.take<int64_t>(ns);
  w.counter = c.take<int32_t>(4);
  w.scr = c.take<double>(kFireScr * ns);
}

// grid of the finite-velocity probe: up to 4 blocks per SM
static unsigned fire_probe_grid(int64_t n) {
  int dev = 0, n_sm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  const int64_t g = (n + kBlock - 1) / kBlock;
  return (unsigned)(g < 4 * (int64_t)n_sm ? (g > 0 ? g : 1) : 4 * (int64_t)n_sm);
}

static int prep_bounds(FireWork &w, const int64_t *sys, int64_t n, int64_t ns,
                       cudaStream_t st) {
  cudaMemsetAsync(w.lo, 0, sizeof(int64_t) * ns, st);
  cudaMemsetAsync(w.hi, 0, sizeof(int64_t) * ns, st);
  cudaMemsetAsync(w.counter, 0, sizeof(int32_t) * 4, st);
  if (n > 0) k_bounds<<<grid_for(n), kBlock, 0, st>>>(sys, n, w.lo, w.hi);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

}  // namespace tsb

using namespace tsb;

extern "C" size_t tsb_fire_workspace_size(int64_t n_systems) {
  Carver c(nullptr, (size_t)-1);
  FireWork w;
  carve_fire(c, w, n_systems);
  return c.off + 256;
}

template <class P>
static int fire_call(int which, int cell_filter, void *positions, void *velocities,
                     const void *forces, const void *masses, const int64_t *system_idx,
                     int64_t n_atoms, int64_t n_systems, void *dt, void *alpha,
                     int32_t *n_pos, void *cell, const void *reference_cell,
                     const void *cell_factor, void *cell_positions, void *cell_velocities,
                     const void *cell_forces, const void *cell_masses, const uint8_t *active,
                     const FireHyper &h, void *workspace, size_t ws_bytes, cudaStream_t st) {
  Carver c(workspace, ws_bytes);
  FireWork w;
  carve_fire(c, w, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  TSB_TRY(prep_bounds(w, system_idx, n_atoms, n_systems, st));
  FireArgs<P> A{cell_filter, (P *)positions, (P *)velocities, (const P *)forces,
                (const P *)masses, (P *)dt, (P *)alpha, n_pos, (P *)cell,
                (const P *)reference_cell, (const P *)cell_factor, (P *)cell_positions,
                (P *)cell_velocities, (const P *)cell_forces, (const P *)cell_masses, active,
                w.lo, w.hi, h};
  if (which == 0) {
    if (n_atoms > 0)
      k_any_finite_v<P><<<fire_probe_grid(n_atoms), kBlock, 0, st>>>((const P *)velocities,
                                                                      n_atoms, w.counter);
    k_fire_ase_vel<P><<<(unsigned)n_systems, kFireThreads, 0, st>>>(A, w.counter, w.scr);
    k_fire_ase_cell<P><<<grid_for(n_systems, 128), 128, 0, st>>>(A, n_systems, w.scr);
    if (n_atoms > 0)
      k_fire_ase_pos<P><<<grid_for(n_atoms), kBlock, 0, st>>>(A, n_atoms, system_idx, w.scr);
  } else if (which == 1) {
    if (n_atoms > 0)
      k_fire_vv_pre<P><<<grid_for(n_atoms), kBlock, 0, st>>>(A, n_atoms, system_idx);
  } else {
    k_fire_vv_post<P><<<(unsigned)n_systems, kFireThreads, 0, st>>>(A);
  }
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

static int fire_entry(int which, int cell_filter, void *positions, void *velocities,
                      const void *forces, const void *masses, const int64_t *system_idx,
                      int64_t n_atoms, int64_t n_systems, void *dt, void *alpha,
                      int32_t *n_pos, void *cell, const void *reference_cell,
                      const void *cell_factor, void *cell_positions, void *cell_velocities,
                      const void *cell_forces, const void *cell_masses, const uint8_t *active,
                      double dt_max, int n_min, double f_inc, double f_dec, double alpha_start,
                      double f_alpha, double max_step, double eps, int dtype, void *workspace,
                      size_t ws_bytes, void *stream) {
  if (n_atoms < 0 || n_systems < 1 || !system_idx || !dt || !alpha || !n_pos)
    return TSB_ERR_INVALID_ARG;
  if (n_atoms > 0 && (!positions || !velocities || !forces || !masses))
    return TSB_ERR_INVALID_ARG;
  if (cell_filter != 0 && cell_filter != 1) return TSB_ERR_INVALID_ARG;
  if (cell_filter && (!cell || !reference_cell || !cell_factor || !cell_positions ||
                      !cell_velocities || !cell_forces))
    return TSB_ERR_INVALID_ARG;
  if (cell_filter && which != 0 && !cell_masses) return TSB_ERR_INVALID_ARG;
  FireHyper h{dt_max, f_inc, f_dec, alpha_start, f_alpha, max_step, eps, n_min};
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == TSB_F64)
    return fire_call<double>(which, cell_filter, positions, velocities, forces, masses,
                             system_idx, n_atoms, n_systems, dt, alpha, n_pos, cell,
                             reference_cell, cell_factor, cell_positions, cell_velocities,
                             cell_forces, cell_masses, active, h, workspace, ws_bytes, st);
  if (dtype == TSB_F32)
    return fire_call<float>(which, cell_filter, positions, velocities, forces, masses,
                            system_idx, n_atoms, n_systems, dt, alpha, n_pos, cell,
                            reference_cell, cell_factor, cell_positions, cell_velocities,
                            cell_forces, cell_masses, active, h, workspace, ws_bytes, st);
  return TSB_ERR_INVALID_ARG;
}

#define TSB_FIRE_ARGS                                                                        \
  int cell_filter, void *positions, void *velocities, const void *forces,                   \
      const void *masses, const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,    \
      void *dt, void *alpha, int32_t *n_pos, void *cell, const void *reference_cell,        \
      const void *cell_factor, void *cell_positions, void *cell_velocities,                 \
      const void *cell_forces, const void *cell_masses, const uint8_t *active,              \
      double dt_max, int n_min, double f_inc, double f_dec, double alpha_start,             \
      double f_alpha, double max_step, double eps, int dtype, void *workspace,              \
      size_t workspace_bytes, void *stream
#define TSB_FIRE_PASS                                                                        \
  cell_filter, positions, velocities, forces, masses, system_idx, n_atoms, n_systems, dt,   \
      alpha, n_pos, cell, reference_cell, cell_factor, cell_positions, cell_velocities,     \
      cell_forces, cell_masses, active, dt_max, n_min, f_inc, f_dec, alpha_start, f_alpha,  \
      max_step, eps, dtype, workspace, workspace_bytes, stream

extern "C" int tsb_fire_ase_pre(TSB_FIRE_ARGS) { return fire_entry(0, TSB_FIRE_PASS); }
extern "C" int tsb_fire_vv_pre(TSB_FIRE_ARGS) { return fire_entry(1, TSB_FIRE_PASS); }
extern "C" int tsb_fire_vv_post(TSB_FIRE_ARGS) { return fire_entry(2, TSB_FIRE_PASS); }

extern "C" int tsb_frechet_cell_forces(void *cell_forces, const void *stress, const void *cell,
                                       const void *reference_cell, const void *pressure,
                                       const void *cell_factor, int64_t n_systems, int init,
                                       const uint8_t *active, int dtype, void *stream) {
  if (n_systems < 1 || !cell_forces || !stress || !cell || !reference_cell || !pressure ||
      !cell_factor)
    return TSB_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == TSB_F64)
    k_frechet_cell_forces<double><<<grid_for(n_systems, 64), 64, 0, st>>>(
        (double *)cell_forces, (const double *)stress, (const double *)cell,
        (const double *)reference_cell, (const double *)pressure,
        (const double *)cell_factor, n_systems, init, active);
  else if (dtype == TSB_F32)
    k_frechet_cell_forces<float><<<grid_for(n_systems, 64), 64, 0, st>>>(
        (float *)cell_forces, (const float *)stress, (const float *)cell,
        (const float *)reference_cell, (const float *)pressure, (const float *)cell_factor,
        n_systems, init, active);
  else
    return TSB_ERR_INVALID_ARG;
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_fire_converged(const void *forces, const int64_t *system_idx,
                                  int64_t n_atoms, int64_t n_systems,
                                  const void *cell_forces, double fmax, uint8_t *active,
                                  int32_t *n_active, int dtype, void *workspace,
                                  size_t workspace_bytes, void *stream) {
  if (n_systems < 1 || !active || !n_active || !system_idx || (n_atoms > 0 && !forces))
    return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  FireWork w;
  carve_fire(c, w, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  TSB_TRY(prep_bounds(w, system_idx, n_atoms, n_systems, st));
  cudaMemsetAsync(n_active, 0, sizeof(int32_t), st);
  if (dtype == TSB_F64)
    k_fire_converged<double><<<(unsigned)n_systems, kFireThreads, 0, st>>>(
        (const double *)forces, w.lo, w.hi, (const double *)cell_forces, fmax, active,
        n_active);
  else if (dtype == TSB_F32)
    k_fire_converged<float><<<(unsigned)n_systems, kFireThreads, 0, st>>>(
        (const float *)forces, w.lo, w.hi, (const float *)cell_forces, fmax, active, n_active);
  else
    return TSB_ERR_INVALID_ARG;
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}
