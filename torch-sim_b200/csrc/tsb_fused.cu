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
//     independent: no grid-wide synchronisation, no host round trips).
//   * Everything the step loop touches lives in shared memory: the system's
//     atoms and the periodic images ("ghosts") within cutoff+skin of the cell as
//     float4 (x, y, z, species) in cell-centre-relative FP32 coordinates, FP64
//     copies of the positions for refreshing the ghosts, and the Verlet list
//     (cutoff + skin) as a uint16 ELL table [slot group][thread] that each thread
//     reads four entries per 64-bit load.  FP64 positions/momenta live in the
//     registers of the owning threads.
//   * The list is rebuilt on the device when any atom of the system moved more
//     than skin/2 since the last build.
//   * Small systems use 2..32 threads per atom (lanes split the list and reduce
//     with warp shuffles).  Summation orders are fixed: results are
//     deterministic and a system's trajectory does not depend on the batch.
//   * Pair arithmetic FP32; positions, momenta and per-system energy FP64.
#include <math.h>

#include <mutex>

#include "tsb_pair.cuh"
#include "tsb_rng.cuh"

namespace tsb {

constexpr int kFusedThreads = 512;
constexpr int kFusedMaxAtoms = 512;
constexpr int kExtMax = 3328;        // atoms + ghost images per system
constexpr int kListLen = 152;        // Verlet-list slots per thread (multiple of 4)
constexpr int kListGroups = kListLen / 4;
constexpr int kFusedMaxSpecies = 4;
constexpr int kMaxGrid = 296;        // upper bound on persistent CTAs
constexpr size_t kSmemList = (size_t)kListGroups * kFusedThreads * sizeof(uint2);
constexpr size_t kSmemExt = (size_t)kExtMax * sizeof(float4);
constexpr size_t kSmemGhost = (size_t)kExtMax * sizeof(uint32_t);
constexpr size_t kFusedSmem = kSmemList + kSmemExt + kSmemGhost;

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
  const uint64_t *counter_dev;  // optional device-resident counter added to `counter`
  double *energy;
  int32_t *n_rebuilds;
  int32_t *queue;
  int32_t *status;
};

// per-system geometry, computed once by thread 0 into shared memory
struct FusedGeom {
  double C[9];    // row-vector cell
  double T[9];    // inv(C)^T: fractional coordinates u = T r
  double ctr[3];  // cell centre
  double tn[3];   // |row k of T|
  double h[3];    // (cutoff + skin) * |row k of T|
  double skin;    // this system's current Verlet skin
  int rep[3];
  int n, tpa, ok;
  int64_t start;
};

// margins of the ghost region for the current skin (thread 0 only)
__device__ inline bool set_margins(FusedGeom &g, double cutoff) {
  bool ok = true;
  for (int k = 0; k < 3; ++k) {
    g.h[k] = (cutoff + g.skin) * g.tn[k] * (1.0 + 1e-9);
    g.rep[k] = (int)ceil(g.h[k]);
    ok = ok && g.rep[k] <= 15;
  }
  return ok;
}

// status[0] = code, [1] = system, [2] = what (1 image slots, 2 list slots), [3] = size
__device__ inline void report(int32_t *status, int code, int64_t sys, int what, int size) {
  if (atomicCAS(status, 0, code) == 0) {
    status[1] = (int32_t)sys;
    status[2] = what;
    status[3] = size;
  }
}

// Block-wide exclusive scan of one int per thread (512 threads).
__device__ inline int block_excl_scan_i(int v, int *total, int *sh) {
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
    const int nw = kFusedThreads / 32;
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

// FP32 standard normals for the O-step (Philox4x32-10 + Box-Muller).
__device__ inline void normal3f(uint64_t seed, uint64_t atom, uint64_t counter, float *z) {
  U4 c{(uint32_t)atom, (uint32_t)(atom >> 32), (uint32_t)counter, (uint32_t)(counter >> 32)};
  U4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const float k24 = 5.9604644775390625e-8f;  // 2^-24
  const float u1 = (float)((r.x >> 8) + 1u) * k24;  // (0, 1]
  const float u2 = (float)((r.z >> 8) + 1u) * k24;
  const float r1 = sqrtf(-2.0f * logf(u1));
  const float r2 = sqrtf(-2.0f * logf(u2));
  float s1, c1, s2, c2;
  sincospif((float)(r.y >> 8) * (2.0f * k24), &s1, &c1);
  sincospif((float)(r.w >> 8) * (2.0f * k24), &s2, &c2);
  z[0] = r1 * c1;
  z[1] = r1 * s1;
  z[2] = r2 * c2;
  (void)s2;
}

__device__ __forceinline__ float4 make_ext(const FusedGeom &g, double x0, double x1, double x2,
                                           int ex, int ey, int ez, int sp) {
  // position x + (ex, ey, ez) @ C relative to the cell centre, rounded to FP32
  float4 e;
  e.x = (float)(x0 + (ex * g.C[0] + ey * g.C[3] + ez * g.C[6]) - g.ctr[0]);
  e.y = (float)(x1 + (ex * g.C[1] + ey * g.C[4] + ez * g.C[7]) - g.ctr[1]);
  e.z = (float)(x2 + (ex * g.C[2] + ey * g.C[5] + ez * g.C[8]) - g.ctr[2]);
  e.w = __int_as_float(sp);
  return e;
}

__device__ __forceinline__ bool in_margin(const FusedGeom &g, double f, int k) {
  return f >= -g.h[k] && f < 1.0 + g.h[k];
}

// Fast FP32 pair evaluation for the fused kernel (exp via ex2.approx).
template <int POT>
__device__ __forceinline__ void pair_eval_fast(const PairPrm<float> &q, float r2, float &e,
                                               float &fr) {
  if (POT == TSB_POT_MORSE) {
    const float ir = rsqrtf(r2);
    const float r = r2 * ir;
    const float ex = __expf(-q.a2 * (r - q.a0));
    const float om = 1.0f - ex;
    e = q.a1 * om * om - q.a1 - q.a4;
    fr = -q.a5 * ex * om * ir;
  } else {
    pair_eval<POT, float>(q, r2, e, fr);
  }
}

template <int POT, bool MULTI>
__global__ void __launch_bounds__(kFusedThreads, 1) k_fused_md(FusedArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint2 *s_list = (uint2 *)smem;
  float4 *s_ext = (float4 *)(smem + kSmemList);
  uint32_t *s_gshift = (uint32_t *)(smem + kSmemList + kSmemExt);
  uint16_t *list16 = (uint16_t *)s_list;
  __shared__ FusedGeom g;
  __shared__ PairPrm<float> prm[kFusedMaxSpecies * kFusedMaxSpecies];
  __shared__ int s_scan[33];
  __shared__ int s_work;
  __shared__ double s_red[kFusedThreads / 32];

  const int tid = threadIdx.x;
  for (int k = tid; k < A.n_species * A.n_species; k += blockDim.x)
    prm[k] = make_prm<float>(POT, A.table + 5 * k, A.cutoff);
  __syncthreads();
  const PairPrm<float> p0 = prm[0];  // single-species parameters in registers
  const uint64_t counter0 = A.counter + (A.counter_dev ? *A.counter_dev : 0ull);

  for (;;) {
    __syncthreads();
    if (tid == 0) s_work = atomicAdd(A.queue, 1);
    __syncthreads();
    const int64_t w = s_work;
    if (w >= A.n_sys) break;
    const int64_t s = A.order ? A.order[w] : w;
    if (tid == 0) {
      g.start = A.lo[s];
      g.n = (int)(A.hi[s] - g.start);
      g.ok = 1;
      double *C = g.C, *T = g.T;
      for (int k = 0; k < 9; ++k) C[k] = A.cell_row[9 * s + k];
      const double d = C[0] * (C[4] * C[8] - C[5] * C[7]) - C[1] * (C[3] * C[8] - C[5] * C[6]) +
                       C[2] * (C[3] * C[7] - C[4] * C[6]);
      const double id = 1.0 / d;
      T[0] = (C[4] * C[8] - C[5] * C[7]) * id;
      T[3] = (C[2] * C[7] - C[1] * C[8]) * id;
      T[6] = (C[1] * C[5] - C[2] * C[4]) * id;
      T[1] = (C[5] * C[6] - C[3] * C[8]) * id;
      T[4] = (C[0] * C[8] - C[2] * C[6]) * id;
      T[7] = (C[2] * C[3] - C[0] * C[5]) * id;
      T[2] = (C[3] * C[7] - C[4] * C[6]) * id;
      T[5] = (C[1] * C[6] - C[0] * C[7]) * id;
      T[8] = (C[0] * C[4] - C[1] * C[3]) * id;
      for (int k = 0; k < 3; ++k) {
        g.tn[k] = sqrt(T[3 * k] * T[3 * k] + T[3 * k + 1] * T[3 * k + 1] +
                       T[3 * k + 2] * T[3 * k + 2]);
        g.ctr[k] = 0.5 * (C[k] + C[3 + k] + C[6 + k]);
      }
      g.skin = A.skin;
      const bool rep_ok = set_margins(g, A.cutoff);
      int tpa = 1;
      while (tpa < 32 && g.n * tpa * 2 <= kFusedThreads) tpa *= 2;
      g.tpa = tpa;
      if (g.n <= 0) {
        g.ok = 0;
        A.energy[s] = 0.0;
        if (A.n_rebuilds) A.n_rebuilds[s] = 0;
      } else if (g.n > kFusedMaxAtoms || !rep_ok || !isfinite(d)) {
        g.ok = 0;
        report(A.status, TSB_ERR_UNSUPPORTED, s, 0, g.n);
      }
    }
    __syncthreads();
    if (!g.ok) continue;
    const int n = g.n, tpa = g.tpa;
    const int a = tid / tpa, lane = tid - a * tpa;
    const bool own = a < n;
    const bool lead = own && lane == 0;
    const int64_t gi = g.start + a;
    // owner state (every lane of the atom holds an identical copy)
    double x0 = 0, x1 = 0, x2 = 0, px = 0, py = 0, pz = 0, inv_m = 1.0, c2m = 0.0;
    float F0 = 0.f, F1 = 0.f, F2 = 0.f, xr0 = 0.f, xr1 = 0.f, xr2 = 0.f;
    int sp = 0;
    if (own) {
      x0 = A.x[3 * gi];
      x1 = A.x[3 * gi + 1];
      x2 = A.x[3 * gi + 2];
      px = A.p[3 * gi];
      py = A.p[3 * gi + 1];
      pz = A.p[3 * gi + 2];
      F0 = (float)A.f[3 * gi];
      F1 = (float)A.f[3 * gi + 1];
      F2 = (float)A.f[3 * gi + 2];
      const double mass = A.m[gi];
      inv_m = 1.0 / mass;
      sp = A.species ? min(max(A.species[gi], 0), A.n_species - 1) : 0;
      if (A.integrator == TSB_INT_LANGEVIN)
        c2m = sqrt(A.kT[s] * (1.0 - exp(-2.0 * (A.gamma[s] * A.dt[s])))) * sqrt(mass);
    }
    const double dt = A.dt[s];
    const double half = dt / 2.0;
    const double c1 = (A.integrator == TSB_INT_LANGEVIN) ? exp(-(A.gamma[s] * dt)) : 1.0;
    int Wx = 0, Wy = 0, Wz = 0;        // integer wrap of the owned atom at the last build
    int gbeg = 0, gcnt = 0;            // the owned atom's ghost slots [gbeg, gbeg + gcnt)
    int cnt = 0, rebuilds = 0;
    bool failed = false;
    float ei = 0.0f, half_skin2 = 0.f;

    // ------------------------------------------------------------- rebuild
    // Wrap the owned atom, create its periodic images inside the cutoff+skin
    // margin of the cell, then every atom scans all atoms + images.  If the
    // shared-memory tables overflow, the skin of this system is halved.
#define TSB_REBUILD()                                                                        \
  for (;;) {                                                                                 \
    const double rcs_ = A.cutoff + g.skin;                                                   \
    const float rcs2_build = (float)(rcs_ * rcs_) * (1.0f + 1e-5f);                          \
    half_skin2 = (float)(0.25 * g.skin * g.skin);                                            \
    int over = 0, over_size = 0;                                                             \
    int gcount = 0;                                                                          \
    double f0 = 0, f1 = 0, f2 = 0;                                                           \
    if (own) {                                                                               \
      const double u0 = g.T[0] * x0 + g.T[1] * x1 + g.T[2] * x2;                             \
      const double u1 = g.T[3] * x0 + g.T[4] * x1 + g.T[5] * x2;                             \
      const double u2 = g.T[6] * x0 + g.T[7] * x1 + g.T[8] * x2;                             \
      const double w0 = floor(u0), w1 = floor(u1), w2 = floor(u2);                           \
      f0 = u0 - w0;                                                                          \
      f1 = u1 - w1;                                                                          \
      f2 = u2 - w2;                                                                          \
      Wx = (int)fmin(fmax(w0, -1e8), 1e8);                                                   \
      Wy = (int)fmin(fmax(w1, -1e8), 1e8);                                                   \
      Wz = (int)fmin(fmax(w2, -1e8), 1e8);                                                   \
      xr0 = (float)x0;                                                                       \
      xr1 = (float)x1;                                                                       \
      xr2 = (float)x2;                                                                       \
      if (lead) {                                                                            \
        s_ext[a] = make_ext(g, x0, x1, x2, -Wx, -Wy, -Wz, sp);                               \
        for (int sx = -g.rep[0]; sx <= g.rep[0]; ++sx) {                                     \
          if (!in_margin(g, f0 + sx, 0)) continue;                                           \
          for (int sy = -g.rep[1]; sy <= g.rep[1]; ++sy) {                                   \
            if (!in_margin(g, f1 + sy, 1)) continue;                                         \
            for (int sz = -g.rep[2]; sz <= g.rep[2]; ++sz) {                                 \
              if (!in_margin(g, f2 + sz, 2)) continue;                                       \
              if ((sx | sy | sz) != 0) ++gcount;                                             \
            }                                                                                \
          }                                                                                  \
        }                                                                                    \
      }                                                                                      \
    }                                                                                        \
    int total;                                                                               \
    const int goff = block_excl_scan_i(gcount, &total, s_scan);                              \
    /* broadcast the lead's ghost range to the other lanes of its atom */                    \
    gbeg = __shfl_sync(0xffffffffu, n + goff, (threadIdx.x & 31) & ~(tpa - 1));              \
    gcnt = __shfl_sync(0xffffffffu, gcount, (threadIdx.x & 31) & ~(tpa - 1));                \
    const int n_ext = n + total;                                                             \
    if (n_ext > kExtMax) {                                                                   \
      over = 1;                                                                              \
      over_size = n_ext;                                                                     \
    } else {                                                                                 \
      if (lead && gcount) {                                                                  \
        int gg = gbeg;                                                                       \
        for (int sx = -g.rep[0]; sx <= g.rep[0]; ++sx) {                                     \
          if (!in_margin(g, f0 + sx, 0)) continue;                                           \
          for (int sy = -g.rep[1]; sy <= g.rep[1]; ++sy) {                                   \
            if (!in_margin(g, f1 + sy, 1)) continue;                                         \
            for (int sz = -g.rep[2]; sz <= g.rep[2]; ++sz) {                                 \
              if (!in_margin(g, f2 + sz, 2)) continue;                                       \
              if ((sx | sy | sz) == 0) continue;                                             \
              s_ext[gg] = make_ext(g, x0, x1, x2, sx - Wx, sy - Wy, sz - Wz, sp);            \
              s_gshift[gg - n] = ((uint32_t)(sx & 1023)) | ((uint32_t)(sy & 1023) << 10) |   \
                                 ((uint32_t)(sz & 1023) << 20);                              \
              ++gg;                                                                          \
            }                                                                                \
          }                                                                                  \
        }                                                                                    \
      }                                                                                      \
      __syncthreads();                                                                       \
      cnt = 0;                                                                               \
      if (own) {                                                                             \
        const float4 xi = s_ext[a];                                                          \
        for (int e = lane; e < n_ext; e += tpa) {                                            \
          const float4 q = s_ext[e];                                                         \
          const float dx = q.x - xi.x, dy = q.y - xi.y, dz = q.z - xi.z;                     \
          const float d2 = dx * dx + dy * dy + dz * dz;                                      \
          if (d2 < rcs2_build && e != a) {                                                   \
            if (cnt < kListLen)                                                              \
              list16[((size_t)(cnt >> 2) * kFusedThreads + tid) * 4 + (cnt & 3)] =           \
                  (uint16_t)e;                                                               \
            ++cnt;                                                                           \
          }                                                                                  \
        }                                                                                    \
      }                                                                                      \
      if (__syncthreads_or(cnt > kListLen)) {                                                \
        over = 2;                                                                            \
        over_size = kListLen;                                                                \
      }                                                                                      \
    }                                                                                        \
    ++rebuilds;                                                                              \
    if (!over) break;                                                                        \
    /* too many images / neighbours for this skin: shrink it (results unchanged) */          \
    __syncthreads();                                                                         \
    const bool zero_skin_ = g.skin == 0.0;                                                   \
    __syncthreads();                                                                         \
    if (zero_skin_) {                                                                        \
      failed = true;                                                                         \
      if (tid == 0) report(A.status, TSB_ERR_CAPACITY, s, over, over_size);                  \
      break;                                                                                 \
    }                                                                                        \
    if (tid == 0) {                                                                          \
      g.skin = g.skin > 0.05 ? 0.5 * g.skin : 0.0;                                           \
      set_margins(g, A.cutoff);                                                              \
    }                                                                                        \
    __syncthreads();                                                                         \
  }

    // ------------------------------------------------------------ pair loop
    // Four list entries per iteration, branch-free (out-of-range pairs are
    // evaluated and masked), so the loads and the math of the four pairs
    // overlap.
#define TSB_PAIR(E, WITH_E)                                                                  \
  {                                                                                          \
    const float4 q = s_ext[E];                                                               \
    const float rx = q.x - xi.x, ry = q.y - xi.y, rz = q.z - xi.z;                           \
    const float r2 = fmaxf(rx * rx + ry * ry + rz * rz, 1e-30f);                             \
    const PairPrm<float> &pq = MULTI ? row[__float_as_int(q.w)] : p0;                        \
    float ep, fr;                                                                            \
    pair_eval_fast<POT>(pq, r2, ep, fr);                                                     \
    const bool in_ = r2 < pq.a3;                                                             \
    fr = in_ ? fr : 0.f;                                                                     \
    fx -= fr * rx;                                                                           \
    fy -= fr * ry;                                                                           \
    fz -= fr * rz;                                                                           \
    if (WITH_E) en += in_ ? ep : 0.f;                                                        \
  }
#define TSB_FORCES(WITH_E)                                                                   \
  {                                                                                          \
    float fx = 0.f, fy = 0.f, fz = 0.f, en = 0.f;                                            \
    if (own) {                                                                               \
      const float4 xi = s_ext[a];                                                            \
      const PairPrm<float> *row = prm + sp * A.n_species;                                    \
      (void)row;                                                                             \
      const int full = cnt >> 2;                                                             \
      for (int k4 = 0; k4 < full; ++k4) {                                                    \
        const uint2 ge = s_list[k4 * kFusedThreads + tid];                                   \
        TSB_PAIR(ge.x & 0xFFFFu, WITH_E)                                                     \
        TSB_PAIR(ge.x >> 16, WITH_E)                                                         \
        TSB_PAIR(ge.y & 0xFFFFu, WITH_E)                                                     \
        TSB_PAIR(ge.y >> 16, WITH_E)                                                         \
      }                                                                                      \
      const int rem = cnt & 3;                                                               \
      if (rem) {                                                                             \
        const uint2 ge = s_list[full * kFusedThreads + tid];                                 \
        TSB_PAIR(ge.x & 0xFFFFu, WITH_E)                                                     \
        if (rem > 1) TSB_PAIR(ge.x >> 16, WITH_E)                                            \
        if (rem > 2) TSB_PAIR(ge.y & 0xFFFFu, WITH_E)                                        \
      }                                                                                      \
    }                                                                                        \
    for (int o = 1; o < tpa; o <<= 1) {                                                      \
      fx += __shfl_xor_sync(0xffffffffu, fx, o);                                             \
      fy += __shfl_xor_sync(0xffffffffu, fy, o);                                             \
      fz += __shfl_xor_sync(0xffffffffu, fz, o);                                             \
      if (WITH_E) en += __shfl_xor_sync(0xffffffffu, en, o);                                 \
    }                                                                                        \
    F0 = fx;                                                                                 \
    F1 = fy;                                                                                 \
    F2 = fz;                                                                                 \
    if (WITH_E) ei = en;                                                                     \
  }

    TSB_REBUILD()
    if (failed) continue;
    for (int64_t step = 0; step < A.n_steps; ++step) {
      if (own) {
        px += F0 * half;
        py += F1 * half;
        pz += F2 * half;
        if (A.integrator == TSB_INT_LANGEVIN) {
          x0 += (px * inv_m) * half;
          x1 += (py * inv_m) * half;
          x2 += (pz * inv_m) * half;
          float z[3];
          normal3f(A.seed, (uint64_t)gi, counter0 + (uint64_t)step, z);
          px = c1 * px + c2m * z[0];
          py = c1 * py + c2m * z[1];
          pz = c1 * pz + c2m * z[2];
          x0 += (px * inv_m) * half;
          x1 += (py * inv_m) * half;
          x2 += (pz * inv_m) * half;
        } else {
          x0 += (px * inv_m) * dt;
          x1 += (py * inv_m) * dt;
          x2 += (pz * inv_m) * dt;
        }
      }
      bool moved = false;
      if (own) {
        const float d0 = (float)x0 - xr0, d1 = (float)x1 - xr1, d2 = (float)x2 - xr2;
        moved = d0 * d0 + d1 * d1 + d2 * d2 > half_skin2;
      }
      // all warps are done reading the previous positions
      __syncthreads();
      // refresh: the lanes of each atom rewrite the atom and its own images
      if (own) {
        for (int it = lane; it <= gcnt; it += tpa) {
          if (it == 0) {
            s_ext[a] = make_ext(g, x0, x1, x2, -Wx, -Wy, -Wz, sp);
          } else {
            const int gg = gbeg + it - 1;
            const uint32_t r = s_gshift[gg - n];
            const int sx = ((int)(r << 22)) >> 22;
            const int sy = ((int)(r << 12)) >> 22;
            const int sz = ((int)(r << 2)) >> 22;
            s_ext[gg] = make_ext(g, x0, x1, x2, sx - Wx, sy - Wy, sz - Wz, sp);
          }
        }
      }
      if (__syncthreads_or(moved)) {
        TSB_REBUILD()
        if (failed) break;
      }
      if (step + 1 == A.n_steps) {
        TSB_FORCES(true)
      } else {
        TSB_FORCES(false)
      }
      if (own) {
        px += F0 * half;
        py += F1 * half;
        pz += F2 * half;
      }
    }
    if (failed) continue;
    if (A.n_steps == 0) TSB_FORCES(true)
#undef TSB_FORCES
#undef TSB_PAIR
#undef TSB_REBUILD
    // ---- write back + FP64 energy reduction (each pair seen from both ends)
    if (lead) {
      A.x[3 * gi] = x0;
      A.x[3 * gi + 1] = x1;
      A.x[3 * gi + 2] = x2;
      A.p[3 * gi] = px;
      A.p[3 * gi + 1] = py;
      A.p[3 * gi + 2] = pz;
      A.f[3 * gi] = F0;
      A.f[3 * gi + 1] = F1;
      A.f[3 * gi + 2] = F2;
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
  c.take<int64_t>(n_systems);  // lo
  c.take<int64_t>(n_systems);  // hi
  c.take<int32_t>(4);          // queue
  (void)n_atoms;
  return c.off + 256;
}

__global__ void k_advance_counter(uint64_t *counter_dev, int64_t n_steps) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *counter_dev += (uint64_t)n_steps;
}

__global__ void k_bounds_fused(const int64_t *sys, int64_t n, int64_t *lo, int64_t *hi) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t s = sys[i];
  if (i == 0 || sys[i - 1] != s) lo[s] = i;
  if (i == n - 1 || sys[i + 1] != s) hi[s] = i + 1;
}

template <int POT, bool MULTI>
static void launch_fused(const FusedArgs &A, int64_t grid, cudaStream_t st) {
  cudaFuncSetAttribute(k_fused_md<POT, MULTI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kFusedSmem);
  k_fused_md<POT, MULTI><<<(unsigned)grid, kFusedThreads, kFusedSmem, st>>>(A);
}

extern "C" int tsb_fused_md(int integrator, int potential, const double *table,
                            int n_species, const int32_t *species, double *positions,
                            double *momenta, double *forces, const double *masses,
                            const double *cell_row, const int64_t *system_idx,
                            int64_t n_atoms, int64_t n_systems, const int32_t *order,
                            double cutoff, double skin, int64_t n_steps,
                            const double *dt_sys, const double *kT_sys,
                            const double *gamma_sys, uint64_t seed, uint64_t counter,
                            uint64_t *counter_dev, double *energy, int32_t *n_rebuilds,
                            int32_t *status, void *workspace, size_t workspace_bytes,
                            void *stream) {
  if (integrator != TSB_INT_NVE && integrator != TSB_INT_LANGEVIN) return TSB_ERR_INVALID_ARG;
  if (potential < TSB_POT_LJ || potential > TSB_POT_SOFT) return TSB_ERR_INVALID_ARG;
  if (n_species < 1 || !table || (n_species > 1 && !species)) return TSB_ERR_INVALID_ARG;
  if (n_species > kFusedMaxSpecies) return TSB_ERR_UNSUPPORTED;
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
  cudaMemsetAsync(status, 0, sizeof(int32_t) * 4, st);
  k_bounds_fused<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, lo, hi);
  FusedArgs A{integrator, potential, n_species, table, species, positions, momenta, forces,
              masses, cell_row, lo, hi, n_systems, order, cutoff, skin, n_steps, dt_sys,
              kT_sys, gamma_sys, seed, counter, counter_dev, energy, n_rebuilds, queue,
              status};
  const bool multi = n_species > 1;
  if (potential == TSB_POT_LJ) {
    multi ? launch_fused<TSB_POT_LJ, true>(A, grid, st) : launch_fused<TSB_POT_LJ, false>(A, grid, st);
  } else if (potential == TSB_POT_MORSE) {
    multi ? launch_fused<TSB_POT_MORSE, true>(A, grid, st)
          : launch_fused<TSB_POT_MORSE, false>(A, grid, st);
  } else {
    multi ? launch_fused<TSB_POT_SOFT, true>(A, grid, st)
          : launch_fused<TSB_POT_SOFT, false>(A, grid, st);
  }
  if (counter_dev) k_advance_counter<<<1, 32, 0, st>>>(counter_dev, n_steps);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of tsb_fused_md.
//
// Some callers cannot hand us a workspace: host programs that own every byte of
// device memory through their own pool and do not let a library call
// cudaMalloc, programs that must not trigger the implicit device-wide
// synchronisation cudaMalloc/cudaFree can cause while other streams run, and
// programs with a fixed memory budget that cannot risk an allocation failing
// mid-run.  For them the scratch of the fused kernel (per-system atom ranges
// and the work counter) lives in this fixed array, compiled into the library.
// Every GPU that loads the library holds it until the process exits.
// ---------------------------------------------------------------------------
namespace tsb {
constexpr int kStaticMaxSystems = TSB_FUSED_STATIC_MAX_SYSTEMS;
constexpr size_t kStaticScratchBytes = 2 * sizeof(int64_t) * kStaticMaxSystems + 256;
static __device__ __align__(256) unsigned char g_fused_static_scratch[kStaticScratchBytes];

// Device address of the array on each device (host code may not use the
// symbol itself as a pointer); looked up once per device, with it current.
constexpr int kMaxDevices = 64;
static void *g_fused_static_ptr[kMaxDevices];
static std::mutex g_fused_static_mu;

static int fused_static_scratch(void **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TSB_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_fused_static_mu);
  if (!g_fused_static_ptr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_fused_static_scratch) != cudaSuccess || !p)
      return TSB_ERR_CUDA;
    g_fused_static_ptr[dev] = p;
  }
  *out = g_fused_static_ptr[dev];
  return TSB_OK;
}
}  // namespace tsb

extern "C" int tsb_fused_md_static(int integrator, int potential, const double *table,
                                   int n_species, const int32_t *species, double *positions,
                                   double *momenta, double *forces, const double *masses,
                                   const double *cell_row, const int64_t *system_idx,
                                   int64_t n_atoms, int64_t n_systems, const int32_t *order,
                                   double cutoff, double skin, int64_t n_steps,
                                   const double *dt_sys, const double *kT_sys,
                                   const double *gamma_sys, uint64_t seed, uint64_t counter,
                                   double *energy, int32_t *n_rebuilds, int32_t *status,
                                   void *stream) {
  if (integrator != TSB_INT_NVE && integrator != TSB_INT_LANGEVIN) return TSB_ERR_INVALID_ARG;
  if (potential < TSB_POT_LJ || potential > TSB_POT_SOFT) return TSB_ERR_INVALID_ARG;
  if (n_species < 1 || !table || (n_species > 1 && !species)) return TSB_ERR_INVALID_ARG;
  if (n_species > kFusedMaxSpecies) return TSB_ERR_UNSUPPORTED;
  if (n_atoms < 1 || n_systems < 1 || !(cutoff > 0.0) || !(skin >= 0.0) || n_steps < 0)
    return TSB_ERR_INVALID_ARG;
  if (!positions || !momenta || !forces || !masses || !cell_row || !system_idx || !dt_sys ||
      !energy || !status)
    return TSB_ERR_INVALID_ARG;
  if (integrator == TSB_INT_LANGEVIN && (!kT_sys || !gamma_sys)) return TSB_ERR_INVALID_ARG;
  // the fixed scratch holds the atom ranges of at most kStaticMaxSystems systems
  if (n_systems > kStaticMaxSystems) return TSB_ERR_CAPACITY;
  void *scratch = nullptr;
  TSB_TRY(fused_static_scratch(&scratch));
  char *base = (char *)scratch;
  int64_t *lo = (int64_t *)base;
  int64_t *hi = lo + kStaticMaxSystems;
  int32_t *queue = (int32_t *)(hi + kStaticMaxSystems);
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, n_sm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  int64_t grid = n_sm;
  if (grid > kMaxGrid) grid = kMaxGrid;
  if (grid > n_systems) grid = n_systems;
  // the array keeps the previous call's contents: clear what must start at zero
  cudaMemsetAsync(lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(hi, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(queue, 0, sizeof(int32_t) * 4, st);
  cudaMemsetAsync(status, 0, sizeof(int32_t) * 4, st);
  k_bounds_fused<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, lo, hi);
  FusedArgs A{integrator, potential, n_species, table, species, positions, momenta, forces,
              masses, cell_row, lo, hi, n_systems, order, cutoff, skin, n_steps, dt_sys,
              kT_sys, gamma_sys, seed, counter, nullptr, energy, n_rebuilds, queue, status};
  const bool multi = n_species > 1;
  if (potential == TSB_POT_LJ) {
    multi ? launch_fused<TSB_POT_LJ, true>(A, grid, st) : launch_fused<TSB_POT_LJ, false>(A, grid, st);
  } else if (potential == TSB_POT_MORSE) {
    multi ? launch_fused<TSB_POT_MORSE, true>(A, grid, st)
          : launch_fused<TSB_POT_MORSE, false>(A, grid, st);
  } else {
    multi ? launch_fused<TSB_POT_SOFT, true>(A, grid, st)
          : launch_fused<TSB_POT_SOFT, false>(A, grid, st);
  }
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}
