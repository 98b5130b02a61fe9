// Persistent fused batched MD: neighbour list + pair forces + integrator for
// thousands of small periodic systems in one launch.
//
// Replaces, per step and per system, the reference chain
//   nvt_langevin_step / nve_step (torch_sim/integrators/nvt.py:144-240,
//   nve.py:74-130) -> model(state) -> PairPotentialModel.forward
//   (torch_sim/models/pair_potential.py:351-464) -> torch_nl_linked_cell
//   (torch_sim/neighbors/torch_nl.py:156-215)
// which rebuilds the neighbour list and launches dozens of kernels per step.
//
// Design (B200, sm_100a):
//   * One CTA (512 threads) owns one system at a time and runs all n_steps for
//     it before taking the next system from a global work counter (systems are
//     independent; no grid-wide synchronisation, no host round trips).
//   * Shared memory holds the system's atoms and the periodic images ("ghosts")
//     that lie within cutoff+skin of the cell, as float4 (x, y, z, species) in
//     cell-centre-relative FP32 coordinates, plus FP64 copies of the positions.
//     FP64 master positions/momenta live in registers of the owning threads.
//   * The Verlet list (cutoff + skin) is an ELL table of uint16 indices into the
//     atom+ghost array in per-CTA global scratch; it is written and read only by
//     the owning thread, so it stays in L1/L2.  It is rebuilt on the device when
//     any atom moved more than skin/2 since the last build.
//   * Small systems use 2..16 threads per atom (lanes split the neighbour list
//     and reduce with warp shuffles), so a 512-thread CTA stays busy for any
//     system size.  Summation orders are fixed: results are deterministic and a
//     system's trajectory does not depend on the rest of the batch.
//   * Pair arithmetic is FP32; positions, momenta and the per-system energy are
//     FP64.
#include <math.h>

#include "tsb_pair.cuh"
#include "tsb_rng.cuh"

namespace tsb {

constexpr int kFusedThreads = 512;
constexpr int kFusedMaxAtoms = 512;
constexpr int kExtMax = 4096;   // atoms + ghost images per system
constexpr int kListLen = 192;   // Verlet-list slots per thread
constexpr int kMaxGrid = 296;   // upper bound on persistent CTAs (scratch sizing)
constexpr size_t kFusedSmem = (size_t)kExtMax * sizeof(float4) +      // ext
                              (size_t)kExtMax * sizeof(uint32_t) +    // ghost records
                              (size_t)kFusedMaxAtoms * 3 * sizeof(double) +  // xd
                              (size_t)kFusedMaxAtoms * sizeof(int4);  // wrap

struct FusedArgs {
  int integrator, potential, n_species;
  const double *table;
  const int32_t *species;
  double *x, *p, *f;
  const double *m;
  const double *cell_row;
  const int64_t *lo, *hi;
  int64_t n_sys;
  const int32_t *order;
  double cutoff, skin;
  int64_t n_steps;
  const double *dt, *kT, *gamma;
  uint64_t seed, counter;
  double *energy;
  int32_t *n_rebuilds;
  uint16_t *lists;
  int32_t *queue;
  int32_t *status;
};

__device__ inline int64_t block_excl_scan_i(int v, int *total, int *sh) {
  // sh: >= 32 ints
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) sh[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    int w = lane < nw ? sh[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < nw) sh[lane] = wi - w;
    if (lane == nw - 1) sh[32] = wi;
  }
  __syncthreads();
  int r = inc - v + sh[warp];
  *total = sh[32];
  __syncthreads();
  return r;
}

__device__ inline void report(int32_t *status, int code, int64_t sys) {
  if (atomicCAS(status, 0, code) == 0) status[1] = (int32_t)sys;
}

template <int POT>
__global__ void __launch_bounds__(kFusedThreads, 1) k_fused_md(FusedArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  float4 *ext = (float4 *)smem;
  uint32_t *ghost = (uint32_t *)(ext + kExtMax);
  double *xd = (double *)(ghost + kExtMax);
  int4 *wrapW = (int4 *)(xd + 3 * kFusedMaxAtoms);
  __shared__ PairPrm<float> prm[kMaxSpecies * kMaxSpecies];
  __shared__ int s_scan[33];
  __shared__ int s_work;
  __shared__ double s_red[kFusedThreads / 32];

  const int tid = threadIdx.x;
  for (int k = tid; k < A.n_species * A.n_species; k += blockDim.x)
    prm[k] = make_prm<float>(POT, A.table + 5 * k, A.cutoff);
  uint16_t *mylist = A.lists + (size_t)blockIdx.x * kListLen * kFusedThreads;
  const double rcs = A.cutoff + A.skin;
  const float rcs2_build = (float)(rcs * rcs) * (1.0f + 1e-5f);
  const double half_skin2 = 0.25 * A.skin * A.skin;

  for (;;) {
    __syncthreads();
    if (tid == 0) s_work = atomicAdd(A.queue, 1);
    __syncthreads();
    const int64_t w = s_work;
    if (w >= A.n_sys) break;
    const int64_t s = A.order ? A.order[w] : w;
    const int64_t start = A.lo[s];
    const int n = (int)(A.hi[s] - start);
    if (n <= 0) {
      if (tid == 0) {
        A.energy[s] = 0.0;
        if (A.n_rebuilds) A.n_rebuilds[s] = 0;
      }
      continue;
    }
    if (n > kFusedMaxAtoms) {
      if (tid == 0) report(A.status, TSB_ERR_UNSUPPORTED, s);
      continue;
    }
    // ---- per-system geometry (every thread, FP64) ----
    double C[9], T[9], h[3], ctr[3];
    for (int k = 0; k < 9; ++k) C[k] = A.cell_row[9 * s + k];
    {
      const double d = C[0] * (C[4] * C[8] - C[5] * C[7]) - C[1] * (C[3] * C[8] - C[5] * C[6]) +
                       C[2] * (C[3] * C[7] - C[4] * C[6]);
      const double id = 1.0 / d;
      // T = inv(C)^T: fractional coordinates u = T r
      T[0] = (C[4] * C[8] - C[5] * C[7]) * id;
      T[3] = (C[2] * C[7] - C[1] * C[8]) * id;
      T[6] = (C[1] * C[5] - C[2] * C[4]) * id;
      T[1] = (C[5] * C[6] - C[3] * C[8]) * id;
      T[4] = (C[0] * C[8] - C[2] * C[6]) * id;
      T[7] = (C[2] * C[3] - C[0] * C[5]) * id;
      T[2] = (C[3] * C[7] - C[4] * C[6]) * id;
      T[5] = (C[1] * C[6] - C[0] * C[7]) * id;
      T[8] = (C[0] * C[4] - C[1] * C[3]) * id;
    }
    int rep[3];
    for (int k = 0; k < 3; ++k) {
      h[k] = rcs * sqrt(T[3 * k] * T[3 * k] + T[3 * k + 1] * T[3 * k + 1] +
                        T[3 * k + 2] * T[3 * k + 2]) * (1.0 + 1e-9);
      rep[k] = (int)ceil(h[k]);
      ctr[k] = 0.5 * (C[k] + C[3 + k] + C[6 + k]);
    }
    if (rep[0] > 15 || rep[1] > 15 || rep[2] > 15) {
      if (tid == 0) report(A.status, TSB_ERR_UNSUPPORTED, s);
      continue;
    }
    int tpa = 1;
    while (tpa < 32 && n * tpa * 2 <= kFusedThreads) tpa *= 2;
    const int a = tid / tpa, lane = tid - a * tpa;
    const bool own = a < n;
    const bool lead = own && lane == 0;
    const int64_t gi = start + a;
    double x[3] = {0, 0, 0}, pm[3] = {0, 0, 0}, F[3] = {0, 0, 0}, xr[3] = {0, 0, 0};
    double mass = 1.0;
    int sp = 0;
    if (own) {
      for (int k = 0; k < 3; ++k) {
        x[k] = A.x[3 * gi + k];
        pm[k] = A.p[3 * gi + k];
        F[k] = A.f[3 * gi + k];
      }
      mass = A.m[gi];
      sp = A.species ? min(max(A.species[gi], 0), A.n_species - 1) : 0;
    }
    const double dt = A.dt[s];
    const double half = dt / 2.0;
    double c1 = 1.0, c2m = 0.0;
    if (A.integrator == TSB_INT_LANGEVIN) {
      c1 = exp(-(A.gamma[s] * dt));
      c2m = sqrt(A.kT[s] * (1.0 - c1 * c1)) * sqrt(mass);
    }
    int Wx = 0, Wy = 0, Wz = 0;
    int n_ext = n, n_ghost = 0, cnt = 0, rebuilds = 0;
    bool failed = false;
    float ei = 0.0f;

    // ---------------------------------------------------------------- rebuild
    auto rebuild = [&]() {
      int gcount = 0;
      double f0 = 0, f1 = 0, f2 = 0;
      if (own) {
        const double u0 = T[0] * x[0] + T[1] * x[1] + T[2] * x[2];
        const double u1 = T[3] * x[0] + T[4] * x[1] + T[5] * x[2];
        const double u2 = T[6] * x[0] + T[7] * x[1] + T[8] * x[2];
        const double w0 = floor(u0), w1 = floor(u1), w2 = floor(u2);
        f0 = u0 - w0;
        f1 = u1 - w1;
        f2 = u2 - w2;
        Wx = (int)w0;
        Wy = (int)w1;
        Wz = (int)w2;
        for (int k = 0; k < 3; ++k) xr[k] = x[k];
        if (lead) {
          wrapW[a] = make_int4(Wx, Wy, Wz, 0);
          for (int k = 0; k < 3; ++k) xd[3 * a + k] = x[k];
          float4 e;
          e.x = (float)(x[0] - (Wx * C[0] + Wy * C[3] + Wz * C[6]) - ctr[0]);
          e.y = (float)(x[1] - (Wx * C[1] + Wy * C[4] + Wz * C[7]) - ctr[1]);
          e.z = (float)(x[2] - (Wx * C[2] + Wy * C[5] + Wz * C[8]) - ctr[2]);
          e.w = __int_as_float(sp);
          ext[a] = e;
          for (int sx = -rep[0]; sx <= rep[0]; ++sx) {
            const double g0 = f0 + sx;
            if (g0 < -h[0] || g0 >= 1.0 + h[0]) continue;
            for (int sy = -rep[1]; sy <= rep[1]; ++sy) {
              const double g1 = f1 + sy;
              if (g1 < -h[1] || g1 >= 1.0 + h[1]) continue;
              for (int sz = -rep[2]; sz <= rep[2]; ++sz) {
                const double g2 = f2 + sz;
                if (g2 < -h[2] || g2 >= 1.0 + h[2]) continue;
                if ((sx | sy | sz) != 0) ++gcount;
              }
            }
          }
        }
      }
      int total;
      int off = (int)block_excl_scan_i(gcount, &total, s_scan);
      n_ghost = total;
      n_ext = n + total;
      if (n_ext > kExtMax) {
        failed = true;
        return;
      }
      if (lead && gcount) {
        int g = n + off;
        for (int sx = -rep[0]; sx <= rep[0]; ++sx) {
          const double g0 = f0 + sx;
          if (g0 < -h[0] || g0 >= 1.0 + h[0]) continue;
          for (int sy = -rep[1]; sy <= rep[1]; ++sy) {
            const double g1 = f1 + sy;
            if (g1 < -h[1] || g1 >= 1.0 + h[1]) continue;
            for (int sz = -rep[2]; sz <= rep[2]; ++sz) {
              const double g2 = f2 + sz;
              if (g2 < -h[2] || g2 >= 1.0 + h[2]) continue;
              if ((sx | sy | sz) == 0) continue;
              const int ex = sx - Wx, ey = sy - Wy, ez = sz - Wz;
              float4 e;
              e.x = (float)(x[0] + (ex * C[0] + ey * C[3] + ez * C[6]) - ctr[0]);
              e.y = (float)(x[1] + (ex * C[1] + ey * C[4] + ez * C[7]) - ctr[1]);
              e.z = (float)(x[2] + (ex * C[2] + ey * C[5] + ez * C[8]) - ctr[2]);
              e.w = __int_as_float(sp);
              ext[g] = e;
              ghost[g - n] = (uint32_t)a | ((uint32_t)(sx & 31) << 16) |
                             ((uint32_t)(sy & 31) << 21) | ((uint32_t)(sz & 31) << 26);
              ++g;
            }
          }
        }
      }
      __syncthreads();
      cnt = 0;
      if (own) {
        const float4 xi = ext[a];
        for (int e = lane; e < n_ext; e += tpa) {
          const float4 q = ext[e];
          const float dx = q.x - xi.x, dy = q.y - xi.y, dz = q.z - xi.z;
          const float d2 = dx * dx + dy * dy + dz * dz;
          if (d2 < rcs2_build && e != a) {
            if (cnt < kListLen) mylist[(size_t)cnt * kFusedThreads + tid] = (uint16_t)e;
            ++cnt;
          }
        }
      }
      if (__syncthreads_or(cnt > kListLen)) failed = true;
      ++rebuilds;
    };

    // ------------------------------------------------- refresh positions only
    auto refresh = [&]() {
      if (lead) {
        for (int k = 0; k < 3; ++k) xd[3 * a + k] = x[k];
        float4 e;
        e.x = (float)(x[0] - (Wx * C[0] + Wy * C[3] + Wz * C[6]) - ctr[0]);
        e.y = (float)(x[1] - (Wx * C[1] + Wy * C[4] + Wz * C[7]) - ctr[1]);
        e.z = (float)(x[2] - (Wx * C[2] + Wy * C[5] + Wz * C[8]) - ctr[2]);
        e.w = __int_as_float(sp);
        ext[a] = e;
      }
      __syncthreads();
      for (int g = tid; g < n_ghost; g += blockDim.x) {
        const uint32_t r = ghost[g];
        const int src = (int)(r & 0xFFFFu);
        const int sx = ((int)(r << 11)) >> 27;
        const int sy = ((int)(r << 6)) >> 27;
        const int sz = ((int)(r << 1)) >> 27;
        const int4 W = wrapW[src];
        const int ex = sx - W.x, ey = sy - W.y, ez = sz - W.z;
        const double *xs = xd + 3 * src;
        float4 e;
        e.x = (float)(xs[0] + (ex * C[0] + ey * C[3] + ez * C[6]) - ctr[0]);
        e.y = (float)(xs[1] + (ex * C[1] + ey * C[4] + ez * C[7]) - ctr[1]);
        e.z = (float)(xs[2] + (ex * C[2] + ey * C[5] + ez * C[8]) - ctr[2]);
        e.w = ext[src].w;
        ext[n + g] = e;
      }
      __syncthreads();
    };

    // ------------------------------------------------------------------ force
    auto forces = [&]() {
      float fx = 0.f, fy = 0.f, fz = 0.f, en = 0.f;
      if (own) {
        const float4 xi = ext[a];
        const PairPrm<float> *row = prm + sp * A.n_species;
        for (int k = 0; k < cnt; ++k) {
          const int e = mylist[(size_t)k * kFusedThreads + tid];
          const float4 q = ext[e];
          const float rx = q.x - xi.x, ry = q.y - xi.y, rz = q.z - xi.z;
          const float r2 = rx * rx + ry * ry + rz * rz;
          const PairPrm<float> &pq = row[__float_as_int(q.w)];
          if (r2 < pq.a3) {
            float ep, fr;
            pair_eval<POT, float>(pq, r2, ep, fr);
            fx -= fr * rx;
            fy -= fr * ry;
            fz -= fr * rz;
            en += ep;
          }
        }
      }
      // reduce over the tpa lanes of this atom (lanes are aligned inside a warp)
      for (int o = 1; o < tpa; o <<= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
        en += __shfl_xor_sync(0xffffffffu, en, o);
      }
      F[0] = fx;
      F[1] = fy;
      F[2] = fz;
      ei = en;
    };

    rebuild();
    if (failed) {
      if (tid == 0) report(A.status, TSB_ERR_CAPACITY, s);
      continue;
    }
    for (int64_t step = 0; step < A.n_steps; ++step) {
      if (own) {
        for (int k = 0; k < 3; ++k) pm[k] = pm[k] + F[k] * half;
        if (A.integrator == TSB_INT_LANGEVIN) {
          for (int k = 0; k < 3; ++k) x[k] = x[k] + (pm[k] / mass) * half;
          double z[4];
          normal4(A.seed, (uint64_t)gi, A.counter + (uint64_t)step, z);
          for (int k = 0; k < 3; ++k) {
            pm[k] = c1 * pm[k] + c2m * z[k];
            x[k] = x[k] + (pm[k] / mass) * half;
          }
        } else {
          for (int k = 0; k < 3; ++k) x[k] = x[k] + (pm[k] / mass) * dt;
        }
      }
      bool moved = false;
      if (own) {
        const double d0 = x[0] - xr[0], d1 = x[1] - xr[1], d2 = x[2] - xr[2];
        moved = d0 * d0 + d1 * d1 + d2 * d2 > half_skin2;
      }
      if (__syncthreads_or(moved)) {
        rebuild();
        if (failed) break;
      } else {
        refresh();
      }
      forces();
      if (own)
        for (int k = 0; k < 3; ++k) pm[k] = pm[k] + F[k] * half;
    }
    if (failed) {
      if (tid == 0) report(A.status, TSB_ERR_CAPACITY, s);
      continue;
    }
    if (A.n_steps == 0) forces();
    // ---- write back + FP64 energy reduction (each pair seen from both ends)
    if (lead) {
      for (int k = 0; k < 3; ++k) {
        A.x[3 * gi + k] = x[k];
        A.p[3 * gi + k] = pm[k];
        A.f[3 * gi + k] = F[k];
      }
    }
    double ev = lead ? 0.5 * (double)ei : 0.0;
    for (int o = 16; o > 0; o >>= 1) ev += __shfl_xor_sync(0xffffffffu, ev, o);
    if ((tid & 31) == 0) s_red[tid >> 5] = ev;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int k = 0; k < kFusedThreads / 32; ++k) t += s_red[k];
      A.energy[s] = t;
      if (A.n_rebuilds) A.n_rebuilds[s] = rebuilds;
    }
  }
}

}  // namespace tsb

using namespace tsb;

extern "C" int tsb_fused_max_atoms(void) { return kFusedMaxAtoms; }

extern "C" size_t tsb_fused_workspace_size(int64_t n_atoms, int64_t n_systems) {
  Carver c(nullptr, (size_t)-1);
  c.take<int64_t>(n_systems);      // lo
  c.take<int64_t>(n_systems);      // hi
  c.take<int32_t>(4);              // queue
  c.take<uint16_t>((int64_t)kMaxGrid * kListLen * kFusedThreads);
  (void)n_atoms;
  return c.off + 256;
}

__global__ void k_bounds_fused(const int64_t *sys, int64_t n, int64_t *lo, int64_t *hi) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t s = sys[i];
  if (i == 0 || sys[i - 1] != s) lo[s] = i;
  if (i == n - 1 || sys[i + 1] != s) hi[s] = i + 1;
}

extern "C" int tsb_fused_md(int integrator, int potential, const double *table,
                            int n_species, const int32_t *species, double *positions,
                            double *momenta, double *forces, const double *masses,
                            const double *cell_row, const int64_t *system_idx,
                            int64_t n_atoms, int64_t n_systems, const int32_t *order,
                            double cutoff, double skin, int64_t n_steps,
                            const double *dt_sys, const double *kT_sys,
                            const double *gamma_sys, uint64_t seed, uint64_t counter,
                            double *energy, int32_t *n_rebuilds, int32_t *status,
                            void *workspace, size_t workspace_bytes, void *stream) {
  if (integrator != TSB_INT_NVE && integrator != TSB_INT_LANGEVIN) return TSB_ERR_INVALID_ARG;
  if (potential < TSB_POT_LJ || potential > TSB_POT_SOFT) return TSB_ERR_INVALID_ARG;
  if (n_species < 1 || n_species > kMaxSpecies || !table || (n_species > 1 && !species))
    return TSB_ERR_INVALID_ARG;
  if (n_atoms < 1 || n_systems < 1 || !(cutoff > 0.0) || !(skin >= 0.0) || n_steps < 0)
    return TSB_ERR_INVALID_ARG;
  if (!positions || !momenta || !forces || !masses || !cell_row || !system_idx || !dt_sys ||
      !energy || !status)
    return TSB_ERR_INVALID_ARG;
  if (integrator == TSB_INT_LANGEVIN && (!kT_sys || !gamma_sys)) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  int64_t *lo = c.take<int64_t>(n_systems);
  int64_t *hi = c.take<int64_t>(n_systems);
  int32_t *queue = c.take<int32_t>(4);
  uint16_t *lists = c.take<uint16_t>((int64_t)kMaxGrid * kListLen * kFusedThreads);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, n_sm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  int64_t grid = n_sm;
  if (grid > kMaxGrid) grid = kMaxGrid;
  if (grid > n_systems) grid = n_systems;
  cudaMemsetAsync(lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(hi, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(queue, 0, sizeof(int32_t) * 4, st);
  cudaMemsetAsync(status, 0, sizeof(int32_t) * 2, st);
  k_bounds_fused<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, lo, hi);
  FusedArgs A{integrator, potential, n_species, table, species, positions, momenta, forces,
              masses, cell_row, lo, hi, n_systems, order, cutoff, skin, n_steps, dt_sys,
              kT_sys, gamma_sys, seed, counter, energy, n_rebuilds, lists, queue, status};
  const size_t smem = kFusedSmem;
#define TSB_FUSED(POT)                                                                   \
  cudaFuncSetAttribute(k_fused_md<POT>, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                       (int)smem);                                                       \
  k_fused_md<POT><<<(unsigned)grid, kFusedThreads, smem, st>>>(A);
  if (potential == TSB_POT_LJ) {
    TSB_FUSED(TSB_POT_LJ)
  } else if (potential == TSB_POT_MORSE) {
    TSB_FUSED(TSB_POT_MORSE)
  } else {
    TSB_FUSED(TSB_POT_SOFT)
  }
#undef TSB_FUSED
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}
