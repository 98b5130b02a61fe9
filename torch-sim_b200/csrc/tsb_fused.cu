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
//     float4 (x, y, z, species) in cell-centre-relative FP32 coordinates, and
//     the Verlet list (cutoff + skin) as a uint16 ELL table [slot group][thread]
//     of byte offsets into the image table, which each thread reads four
//     entries per 64-bit load.  FP64
//     positions/momenta live in the registers of the owning threads.
//   * The list is rebuilt on the device when any atom of the system moved more
//     than skin/2 since the last build.  A rebuild sorts atoms + images into
//     bins of half the list radius in fractional coordinates (counting sort in
//     shared memory, entries ordered by index inside a bin) and each atom scans
//     the 5 x 5 x 5 bins around its own, row by row over contiguous entries.
//   * The list has two parts: "core" pairs (slots from the bottom), closer at
//     the build than cutoff - skin, stay inside the cutoff for the list's whole
//     life and are evaluated without any cutoff test; "shell" pairs (slots from
//     the top) get the cutoff test.
//   * Small systems use 2..32 threads per atom (lanes split the candidates and
//     the list and reduce with warp shuffles).  Summation orders are fixed:
//     results are deterministic and a system's trajectory does not depend on
//     the batch.
//   * Pair arithmetic FP32; positions, momenta and per-system energy FP64.
//     Whether a pair is inside the cutoff is decided as in FP64: a shell pair
//     whose FP32 r^2 lies within the proven FP32 rounding bound of the
//     cutoff^2 is re-tested on FP64 positions.  Those live in the caller's
//     force array while the system runs (wrapped, cell-centre relative; the
//     forces are held in registers and written over them at the end).
#include <math.h>

#include <algorithm>
#include <mutex>

#include "tsb_pair.cuh"
#include "tsb_rng.cuh"
#include "tsb_thermostat.cuh"

namespace tsb {

constexpr int kFusedMaxAtoms = 512;
constexpr int kFusedMaxSpecies = 4;
constexpr int kMaxGrid = 296;        // upper bound on persistent CTAs

// Two block shapes.  Wide: 512 threads, one block per SM, any system of up to
// 512 atoms.  Narrow: 256 threads and half the shared memory, two blocks per
// SM, for systems of up to 256 atoms whose images fit its smaller table -- two
// independent systems per SM hide each other's barrier and latency stalls
// (1.4x the throughput of the wide shape on systems of up to 128 atoms).
template <int NT>
struct FusedShape;
template <>
struct FusedShape<512> {
  static constexpr int kThreads = 512, kMinBlocks = 1;
  static constexpr int kExtMax = 3328;   // atoms + ghost images per system
  static constexpr int kListLen = 144;   // Verlet-list slots per thread (multiple of 4)
  static constexpr int kMaxBins = 2048;  // spatial bins over the image region
};
template <>
struct FusedShape<256> {
  static constexpr int kThreads = 256, kMinBlocks = 2;
  static constexpr int kExtMax = 1968;
  static constexpr int kListLen = 128;
  static constexpr int kMaxBins = 1024;
};
template <int NT>
struct FusedSmem {
  using S = FusedShape<NT>;
  static constexpr size_t kList = (size_t)(S::kListLen / 4) * NT * sizeof(uint2);
  static constexpr size_t kExt = (size_t)S::kExtMax * sizeof(float4);
  static constexpr size_t kGhost = (size_t)S::kExtMax * sizeof(uint32_t);
  static constexpr size_t kSorted = (size_t)S::kExtMax * sizeof(uint16_t);
  static constexpr size_t kBins = (size_t)S::kMaxBins * sizeof(int);
  static constexpr size_t kTotal = kList + kExt + kGhost + kSorted + kBins;
  // the bin of every entry is kept in the list area while the list is rebuilt
  static_assert(S::kExtMax * sizeof(uint16_t) <= kList, "bin ids alias the list");
  static_assert(S::kMaxBins <= 4 * NT, "bin scan: four bins per thread");
  static_assert((S::kExtMax - 1) * sizeof(float4) <= 0xFFFF,
                "list entries are 16-bit byte offsets");
  static_assert(kList >= (size_t)S::kExtMax * (sizeof(float4) + sizeof(uint32_t)),
                "the bin-order copy of the table fits the list area");
  static_assert(kSorted + kBins >= (size_t)NT * 3 * sizeof(double),
                "atom positions alias the sort and bin tables");
  static_assert((kList + kExt + kGhost) % 8 == 0, "sort table 8-byte aligned");
};

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
  // Nose-Hoover chain / V-rescale (integrator TSB_INT_NOSE_HOOVER / TSB_INT_VRESCALE)
  double *cxi, *cpxi, *cQ, *cke;  // chain positions, momenta, masses [S, M]; carried KE [S]
  const double *tau, *cdt;        // thermostat time constant [S]; chain time step [S]
  int M, nc, nsy;                 // chain length, chain steps, Suzuki-Yoshida steps
  // trajectory frames (tsb_fused_md_ex): every rep_every steps, positions [N, 3]
  // (FP32) into frame_x and the potential energy of each system into frame_e
  float *frame_x;
  double *frame_e;
  int64_t rep_every, n_frames, n_atoms_total;
  // per-system stress [S, 3, 3] at the last step (optional): -W / V with the
  // virial W = sum over pairs of r (x) f, accumulated in FP64
  double *stress;
  // most lanes per atom (a power of two in 1..32; 0 means 32): small systems
  // get the largest lane count with atoms x lanes <= the block's threads
  int lanes_max;
  // systems this launch takes from `order` (order[0 .. n_work)); 0: all n_sys
  int64_t n_work;
  // dynamic pruning of the list's shell (0: off): between list builds only the
  // shell pairs within cutoff + prune are evaluated, and the shell is pruned
  // again whenever an atom moved more than prune / 2 since the last pruning
  double prune;
};

// per-system geometry, computed by thread 0 into shared memory
struct FusedGeom {
  double C[9];    // row-vector cell
  double T[9];    // inv(C)^T: fractional coordinates u = T r
  double ctr[3];  // cell centre
  double tn[3];   // |row k of T|
  double h[3];    // (cutoff + skin) * |row k of T|: image margin, fractional
  double iw[3];   // 1 / bin width, fractional
  double skin;    // this system's current Verlet skin
  double half_skin2;    // (skin / 2)^2: rebuild when an atom moved further
  double half_prune2;   // (prune / 2)^2: prune the shell again when an atom moved further
  float act2;     // FP32 r^2 below which a shell pair stays in the pruned shell
  int prune_on;   // 0 < prune < skin
  double dt, half, c1;  // time step, dt / 2, Langevin exp(-gamma dt)
  // thermostat scalars of this system (thread 0), and the momentum factor it
  // hands to all threads
  double cx[kMaxChain], cv[kMaxChain], cq[kMaxChain];
  double cke, nf, kt, tau, cdt, th_scale;
  float band;     // FP32 r^2 within +-band of cutoff^2: decide in FP64
  float build2;   // list radius^2 used by the FP32 build test
  float core2[kFusedMaxSpecies * kFusedMaxSpecies];  // core-pair bound^2 per pair type
  // search window of the list build, FP32: bin width and margin h in
  // fractional coordinates, 1 / width, plane window (list radius) |T_k| + eps,
  // |a_k|^2, and 1 / lambda with lambda a lower bound of the smallest
  // eigenvalue of D^-1 G D^-1 (G = C C^T, D = diag |a_k|), so that
  // |d|^2 >= lambda sum_k |a_k|^2 du_k^2 for any fractional offset du
  float sw[3], sh[3], siw[3], stw[3], alen2[3], ilam;
  int rep[3];
  int nb[3];
  int nbins;
  int n, tpa, ok;
  int64_t start;
  // potential energy and virial (xx, yy, zz, yz, xz, xy) of the system at the
  // last energy step, FP64 sums in a fixed order (thread 0)
  double esum7[7];
};

// Margins of the image region, bins, FP32 error bounds and core radii for the
// current skin (thread 0 only).
//
// Error bounds: every image y (FP64) is stored as fl32(y) with |y_m| <= Y (per
// coordinate, Y = max_m sum_k (1/2 + h_k) |C_km|), so each coordinate carries
// an error <= 2^-24 Y and a difference d_m one <= 2^-24 (2Y + |d_m|).
//   * band: for |d| ~ rc the FP32 r^2 differs from the exact one by at most
//     2^-24 (4 sqrt3 Y rc + 2 rc^2), plus 3 2^-24 rc^2 for the products and sums
//     and 2^-24 rc^2 for the rounding of cutoff^2 itself; the band is twice it.
//   * distances (list build) and displacements (rebuild test, against the FP32
//     build position) are off by less than 1e-7 (4Y + R) together,
//     R = cutoff + skin; `margin` = 10x that widens the build radius and
//     narrows the core radius.
// Bins: width >= R |T_k| / 2 in fractional coordinate k, so two points closer
// than R differ by at most 2 bins per axis; coarsened until <= kMaxBins.
template <int kMaxBins>
__device__ inline bool set_margins(FusedGeom &g, double cutoff, double prune, const double *rc2d,
                                   int nsp2) {
  bool ok = true;
  const double R = cutoff + g.skin;
  g.half_skin2 = 0.25 * g.skin * g.skin;
  for (int k = 0; k < 3; ++k) {
    g.h[k] = R * g.tn[k] * (1.0 + 1e-9);
    g.rep[k] = (int)ceil(g.h[k]);
    ok = ok && g.rep[k] <= 15;
  }
  double ymax = 0.0, ypmax = 0.0;
  for (int m = 0; m < 3; ++m) {
    double y = 0.0, yp = 0.0;
    for (int k = 0; k < 3; ++k) {
      y += (0.5 + g.h[k]) * fabs(g.C[3 * k + m]);
      yp += (0.5 + g.rep[k]) * fabs(g.C[3 * k + m]);
    }
    ymax = fmax(ymax, y);
    ypmax = fmax(ypmax, yp);
  }
  // Every table entry is fl32 of its FP64 value (atoms and images alike, at
  // the build and at every refresh), off by at most 2^-24 Y per coordinate.
  g.band = (float)(2.0 * 5.9604644775390625e-8 *
                   (4.0 * 1.7320508075688772 * ymax * cutoff + 6.0 * cutoff * cutoff));
  const double margin = 1e-6 * (4.0 * ymax + R);
  g.build2 = (float)((R + margin) * (R + margin));
  // Pruned shell: a pair whose FP32 distance at the pruning is at least
  // cutoff + prune + pm, pm = 1e-6 (8 Y' + R) (Y' = max_m sum_k (1/2 + rep_k)
  // |C_km| >= Y), is left out until the next pruning.  Until then no atom moves
  // more than prune / 2 from its position at the pruning (tested in FP64
  // against that position rounded to FP32), so the exact distance stays above
  // the cutoff: pm covers the FP32 distance error (each coordinate of both
  // entries off by <= 2^-24 Y, so |d| by <= 2 sqrt3 2^-24 Y, plus ~2^-23 R from
  // the arithmetic) and the FP32 rounding of both reference positions
  // (2 sqrt3 2^-24 Y), with a wide margin.
  const double pr = (prune > 0.0 && prune < g.skin) ? prune : 0.0;
  g.prune_on = pr > 0.0;
  g.half_prune2 = pr > 0.0 ? 0.25 * pr * pr : INFINITY;
  const double pm = 1e-6 * (8.0 * ypmax + R);
  g.act2 = (float)((cutoff + pr + pm) * (cutoff + pr + pm));
  for (int k = 0; k < nsp2; ++k) {
    const double cr = sqrt(rc2d[k]) - g.skin - margin;
    g.core2[k] = cr > 0.0 ? (float)(cr * cr) : -1.0f;
  }
  // one bin of the whole region (always valid) unless a finer grid fits
  g.nb[0] = g.nb[1] = g.nb[2] = 1;
  g.nbins = 1;
  for (int k = 0; k < 3; ++k) g.iw[k] = 0.0;
  double c = 1.0;
  for (int it = 0; it < 64; ++it, c *= 1.25) {
    double tot = 1.0, nbd[3], iw[3];
    for (int k = 0; k < 3; ++k) {
      const double w = c * 0.5 * R * g.tn[k] * (1.0 + 1e-6);
      nbd[k] = fmax(1.0, ceil((1.0 + 2.0 * g.h[k]) / w));
      iw[k] = 1.0 / w;
      tot *= nbd[k];
    }
    if (tot <= (double)kMaxBins) {
      for (int k = 0; k < 3; ++k) {
        g.nb[k] = (int)nbd[k];
        g.iw[k] = iw[k];
      }
      g.nbins = (int)tot;
      break;
    }
  }
  const double rb = sqrt((double)g.build2);
  for (int k = 0; k < 3; ++k) {
    g.sw[k] = g.iw[k] > 0.0 ? (float)(1.0 / g.iw[k]) : 1e30f;
    g.sh[k] = (float)g.h[k];
    g.siw[k] = (float)g.iw[k];
    g.stw[k] = (float)(rb * g.tn[k]) + 1e-5f;
  }
  return ok;
}

__device__ __forceinline__ int bin_coord(const FusedGeom &g, double f, int k) {
  const int b = (int)floor((f + g.h[k]) * g.iw[k]);
  return min(max(b, 0), g.nb[k] - 1);
}

// status[0] = code, [1] = system, [2] = what (1 image slots, 2 list slots), [3] = size
__device__ inline void report(int32_t *status, int code, int64_t sys, int what, int size) {
  if (atomicCAS(status, 0, code) == 0) {
    status[1] = (int32_t)sys;
    status[2] = what;
    status[3] = size;
  }
}

// Block-wide exclusive scan of one int per thread (NT threads).
template <int NT>
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
    const int nw = NT / 32;
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

// FP64 sum over the block in a fixed order (shuffles inside each warp, then the
// warps in order); the result is valid in thread 0 only
template <int NT>
__device__ inline double block_sum_to0(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < NT / 32; ++w) t += sh[w];
  return t;
}

// Warp sum of one FP64 value (fixed order), stored by lane 0 into sh[warp]
__device__ __forceinline__ void warp_sum_store(double t, double *sh) {
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
}

// Thread 0: out[c] = sum over warps of sh[c][warp], c < 7 (fixed order)
template <int NT>
__device__ __noinline__ void warps_sum7(const double (*sh)[NT / 32], double *out) {
  for (int c = 0; c < 7; ++c) {
    double t = 0.0;
    for (int w = 0; w < NT / 32; ++w) t += sh[c][w];
    out[c] = t;
  }
}

// PTX approximate base-2 logarithm, sine and cosine (hardware MUFU; absolute
// errors ~2^-22 for lg2 near 1 and ~2^-21 for sin / cos on [-pi, pi]).
__device__ __forceinline__ float lg2_ftz(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sin_ftz(float x) {
  float y;
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float cos_ftz(float x) {
  float y;
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// FP32 standard normals for the O-step (Philox4x32-10 + Box-Muller): radii
// sqrt(-2 ln u), u = (w >> 8 + 1) 2^-24 in (0, 1], and angles pi t,
// t = (w >> 8) 2^-23 in [0, 2), evaluated as -cos / -sin of pi (t - 1) (t - 1
// is exact) so that the hardware sine and cosine see arguments in [-pi, pi).
// The values agree with the FP64 Box-Muller of the same integers to a few
// 1e-6 absolute.
__device__ inline void normal3f(uint64_t seed, uint64_t atom, uint64_t counter, float *z) {
  U4 c{(uint32_t)atom, (uint32_t)(atom >> 32), (uint32_t)counter, (uint32_t)(counter >> 32)};
  U4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const float k24 = 5.9604644775390625e-8f;  // 2^-24
  const float m2ln2 = -1.3862943611198906f;   // -2 ln 2
  const float pi = 3.14159265358979f;
  const float u1 = (float)((r.x >> 8) + 1u) * k24;  // (0, 1]
  const float u2 = (float)((r.z >> 8) + 1u) * k24;
  const float r1 = sqrtf(fmaxf(m2ln2 * lg2_ftz(u1), 0.0f));
  const float r2 = sqrtf(fmaxf(m2ln2 * lg2_ftz(u2), 0.0f));
  const float a1 = pi * ((float)(r.y >> 8) * (2.0f * k24) - 1.0f);
  const float a2 = pi * ((float)(r.w >> 8) * (2.0f * k24) - 1.0f);
  z[0] = -r1 * cos_ftz(a1);
  z[1] = -r1 * sin_ftz(a1);
  z[2] = -r2 * cos_ftz(a2);
}

// ghost slot word: shift (sx, sy, sz) in [-15, 15] as 5-bit fields, owner atom above
__device__ __forceinline__ uint32_t pack_ghost(int owner, int sx, int sy, int sz) {
  return ((uint32_t)(sx & 31)) | ((uint32_t)(sy & 31) << 5) | ((uint32_t)(sz & 31) << 10) |
         ((uint32_t)owner << 15);
}
__device__ __forceinline__ void unpack_ghost(uint32_t r, int &owner, int &sx, int &sy, int &sz) {
  sx = ((int)(r << 27)) >> 27;
  sy = ((int)(r << 22)) >> 27;
  sz = ((int)(r << 17)) >> 27;
  owner = (int)(r >> 15);
}

// Exact (FP64) squared distance between the home image of atom a and table
// table entry e (owner atom + lattice shift @ C, from its descriptor), from the
// FP64 wrapped positions Y [n, 3] of the system.  Rarely called (pairs within
// the band).
__device__ __noinline__ double exact_r2(const double *Y, const uint32_t *s_desc,
                                        const FusedGeom &g, int a, int e) {
  int j, sx, sy, sz;
  unpack_ghost(s_desc[e], j, sx, sy, sz);
  const double s0 = sx * g.C[0] + sy * g.C[3] + sz * g.C[6];
  const double s1 = sx * g.C[1] + sy * g.C[4] + sz * g.C[7];
  const double s2 = sx * g.C[2] + sy * g.C[5] + sz * g.C[8];
  const double dx = (Y[3 * j] + s0) - Y[3 * a];
  const double dy = (Y[3 * j + 1] + s1) - Y[3 * a + 1];
  const double dz = (Y[3 * j + 2] + s2) - Y[3 * a + 2];
  return dx * dx + dy * dy + dz * dz;
}

// wrapped, cell-centre-relative FP64 position x - W @ C - ctr
__device__ __forceinline__ void wrapped(const FusedGeom &g, double x0, double x1, double x2,
                                        int wx, int wy, int wz, double &y0, double &y1,
                                        double &y2) {
  y0 = x0 - (wx * g.C[0] + wy * g.C[3] + wz * g.C[6]) - g.ctr[0];
  y1 = x1 - (wx * g.C[1] + wy * g.C[4] + wz * g.C[7]) - g.ctr[1];
  y2 = x2 - (wx * g.C[2] + wy * g.C[5] + wz * g.C[8]) - g.ctr[2];
}

// image y + s @ C rounded to FP32, species in w
__device__ __forceinline__ float4 image_of(const FusedGeom &g, double y0, double y1, double y2,
                                           int sx, int sy, int sz, int sp) {
  float4 e;
  e.x = (float)(y0 + (sx * g.C[0] + sy * g.C[3] + sz * g.C[6]));
  e.y = (float)(y1 + (sx * g.C[1] + sy * g.C[4] + sz * g.C[7]));
  e.z = (float)(y2 + (sx * g.C[2] + sy * g.C[5] + sz * g.C[8]));
  e.w = __int_as_float(sp);
  return e;
}

__device__ __forceinline__ bool in_margin(const FusedGeom &g, double f, int k) {
  return f >= -g.h[k] && f < 1.0 + g.h[k];
}

// Two pairs at once in FP32x2 arithmetic (sm_100 FFMA2 / FMUL2 / FADD2): the
// constants of one single-species parameter row duplicated into both halves.
struct Prm2 {
  float2 c0, c1, c2, c3;
};

template <int POT>
__device__ inline Prm2 make_prm2(const PairPrm<float> &q) {
  Prm2 k;
  if (POT == TSB_POT_MORSE) {
    k.c0 = make_float2(q.a6, q.a6);  // exponent slope (base 2)
    k.c1 = make_float2(q.a7, q.a7);  // exponent offset
    k.c2 = make_float2(q.a5, q.a5);  // 2 alpha D
  } else {
    k.c0 = make_float2(q.a0, q.a0);  // sigma^2
    k.c1 = make_float2(q.a2, q.a2);  // 24 eps
    k.c2 = make_float2(2.0f, 2.0f);
  }
  k.c3 = make_float2(-1.0f, -1.0f);
  return k;
}

// fr = -V'(r)/r of two pairs (LJ or Morse); energies only when WITH_E
template <int POT, bool WITH_E>
__device__ __forceinline__ float2 pair_fr2(const Prm2 &k, const PairPrm<float> &q, float2 r2,
                                           float2 &e) {
  if (POT == TSB_POT_MORSE) {
    const float2 ir = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
    const float2 r = __fmul2_rn(r2, ir);
    const float2 arg = __ffma2_rn(k.c0, r, k.c1);
    const float2 x = make_float2(ex2_ftz(arg.x), ex2_ftz(arg.y));
    if (WITH_E) {
      e.x = q.a1 * x.x * (x.x - 2.0f) - q.a4;
      e.y = q.a1 * x.y * (x.y - 2.0f) - q.a4;
    }
    // -2 alpha D x (1 - x) / r = (x x - x) (2 alpha D / r)
    return __fmul2_rn(__ffma2_rn(x, x, make_float2(-x.x, -x.y)), __fmul2_rn(k.c2, ir));
  } else {
    const float2 ir2 = make_float2(rcp_ftz(r2.x), rcp_ftz(r2.y));
    const float2 s2 = __fmul2_rn(k.c0, ir2);
    const float2 s6 = __fmul2_rn(__fmul2_rn(s2, s2), s2);
    if (WITH_E) {
      e.x = q.a1 * s6.x * (s6.x - 1.0f) - q.a4;
      e.y = q.a1 * s6.y * (s6.y - 1.0f) - q.a4;
    }
    // 24 eps s6 (2 s6 - 1) / r^2
    return __fmul2_rn(__fmul2_rn(k.c1, s6), __fmul2_rn(__ffma2_rn(k.c2, s6, k.c3), ir2));
  }
}

template <int POT, bool MULTI, int NT, int INTEG>
__global__ void __launch_bounds__(NT, FusedShape<NT>::kMinBlocks) k_fused_md(FusedArgs A) {
  // the integrator: fixed at compile time for the common single-species
  // Langevin launches (the other integrators' code is then left out), else read
  const int integ = INTEG >= 0 ? INTEG : A.integrator;
  // the block shape's table sizes (these names shadow nothing at namespace scope)
  constexpr int kFusedThreads = NT;
  constexpr int kListLen = FusedShape<NT>::kListLen;
  constexpr int kListGroups = kListLen / 4;
  constexpr int kExtMax = FusedShape<NT>::kExtMax;
  constexpr int kMaxBins = FusedShape<NT>::kMaxBins;
  constexpr size_t kSmemList = FusedSmem<NT>::kList;
  constexpr size_t kSmemExt = FusedSmem<NT>::kExt;
  constexpr size_t kSmemGhost = FusedSmem<NT>::kGhost;
  constexpr size_t kSmemSorted = FusedSmem<NT>::kSorted;
  // the last image slot holds a point far from everything: list padding entries
  // point at it and contribute nothing (outside every cutoff and FP64 band)
  constexpr int kSentinel = kExtMax - 1;
  // single-species LJ / Morse: pairs evaluated two at a time in FP32x2
  constexpr bool kPaired = !MULTI && POT != TSB_POT_SOFT;
  extern __shared__ __align__(16) unsigned char smem[];
  uint2 *s_list = (uint2 *)smem;
  float4 *s_ext = (float4 *)(smem + kSmemList);
  uint32_t *s_gshift = (uint32_t *)(smem + kSmemList + kSmemExt);
  uint16_t *s_sorted = (uint16_t *)(smem + kSmemList + kSmemExt + kSmemGhost);
  int *s_bin = (int *)(smem + kSmemList + kSmemExt + kSmemGhost + kSmemSorted);
  uint16_t *list16 = (uint16_t *)s_list;
  uint16_t *s_ebin = (uint16_t *)s_list;  // bin of each entry, during a rebuild only
  // the atoms' new FP64 wrapped positions [n, 3], from the integrator phase of
  // a step to the image refresh of the same step (the sort and bin tables of
  // the list build are free then)
  double *s_posd = (double *)s_sorted;
  __shared__ FusedGeom g;
  __shared__ PairPrm<float> prm[kFusedMaxSpecies * kFusedMaxSpecies];
  __shared__ double rc2d[kFusedMaxSpecies * kFusedMaxSpecies];
  __shared__ int s_scan[33];
  __shared__ int s_work;
  // per-step decisions (bit 1 rebuild the list, bit 2 prune it), OR-ed by the
  // warps before the refresh barrier; two slots by step parity, so that the
  // slot of the next step is cleared while this one is read
  __shared__ int s_flags[2];
  __shared__ double s_red[kFusedThreads / 32];
  __shared__ double s_red7[7][kFusedThreads / 32];

  const int tid = threadIdx.x;
  const int nsp2 = A.n_species * A.n_species;
  for (int k = tid; k < nsp2; k += blockDim.x) {
    prm[k] = make_prm<float>(POT, A.table + 5 * k, A.cutoff);
    prm_fast_extra(POT, A.table + 5 * k, prm[k]);
    rc2d[k] = pair_rc2(POT, A.table + 5 * k, A.cutoff);
  }
  __syncthreads();
  const PairPrm<float> p0 = prm[0];  // single-species parameters in registers
  const Prm2 k2 = make_prm2<POT>(p0);
  const double rc2d0 = rc2d[0];
  const uint64_t counter0 = A.counter + (A.counter_dev ? *A.counter_dev : 0ull);

  if (tid == 0) s_ext[kSentinel] = make_float4(1e18f, 1e18f, 1e18f, __int_as_float(0));
  for (;;) {
    __syncthreads();
    if (tid == 0) s_work = atomicAdd(A.queue, 1);
    __syncthreads();
    const int64_t w = s_work;
    if (w >= (A.n_work > 0 ? A.n_work : A.n_sys)) break;
    const int64_t s = A.order ? A.order[w] : w;
    if (tid == 0) {
      s_flags[0] = s_flags[1] = 0;
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
      {
        // Gram matrix of the lattice vectors and a Gershgorin lower bound of the
        // smallest eigenvalue of its unit-diagonal form (cosines off the diagonal)
        double G[3][3];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j)
            G[i][j] = C[3 * i] * C[3 * j] + C[3 * i + 1] * C[3 * j + 1] + C[3 * i + 2] * C[3 * j + 2];
        double lam = 1.0;
        for (int i = 0; i < 3; ++i) {
          double off = 0.0;
          for (int j = 0; j < 3; ++j)
            if (j != i) off += fabs(G[i][j]) / sqrt(G[i][i] * G[j][j]);
          lam = fmin(lam, 1.0 - off);
          g.alen2[i] = (float)(G[i][i] * (1.0 - 1e-6));
        }
        g.ilam = lam > 0.05 ? (float)(1.0 / lam) * 1.0001f : 1e30f;
      }
      g.skin = A.skin;
      g.dt = A.dt[s];
      g.half = g.dt / 2.0;
      g.c1 = (integ == TSB_INT_LANGEVIN) ? exp(-(A.gamma[s] * g.dt)) : 1.0;
      if (integ == TSB_INT_NOSE_HOOVER || integ == TSB_INT_VRESCALE) {
        g.nf = 3.0 * (double)g.n - 3.0;  // COM motion removed (nvt.py:287-290)
        g.kt = A.kT[s];
        g.tau = A.tau[s];
        if (integ == TSB_INT_NOSE_HOOVER) {
          g.cdt = A.cdt[s];
          g.cke = A.cke[s];
          for (int j = 0; j < A.M; ++j) {
            g.cq[j] = g.kt * (g.tau * g.tau) * (j == 0 ? g.nf : 1.0);
            g.cx[j] = A.cxi[s * A.M + j];
            g.cv[j] = A.cpxi[s * A.M + j];
          }
        }
      }
      const bool rep_ok =
          isfinite(d) && d != 0.0 && set_margins<kMaxBins>(g, A.cutoff, A.prune, rc2d, nsp2);
      int tpa = 1;
      const int lmax = A.lanes_max > 0 ? min(A.lanes_max, 32) : 32;
      while (tpa * 2 <= lmax && g.n * tpa * 2 <= kFusedThreads) tpa *= 2;
      g.tpa = tpa;
      if (g.n <= 0) {
        g.ok = 0;
        A.energy[s] = 0.0;
        if (A.stress)
          for (int k = 0; k < 9; ++k) A.stress[9 * s + k] = 0.0;
        if (A.n_rebuilds) A.n_rebuilds[s] = 0;
      } else if (g.n > (kFusedMaxAtoms < kFusedThreads ? kFusedMaxAtoms : kFusedThreads) ||
                 !rep_ok) {
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
    double *Y = A.f + 3 * g.start;  // FP64 wrapped positions of this system (see top)
    // owner state (every lane of the atom holds an identical copy)
    double x0 = 0, x1 = 0, x2 = 0, px = 0, py = 0, pz = 0, inv_m = 1.0, c2m = 0.0;
    float F0 = 0.f, F1 = 0.f, F2 = 0.f;
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
      if (integ == TSB_INT_LANGEVIN)
        c2m = sqrt(A.kT[s] * (1.0 - exp(-2.0 * (A.gamma[s] * A.dt[s])))) * sqrt(mass);
    }
    int Wx = 0, Wy = 0, Wz = 0;        // integer wrap of the owned atom at the last build
    int ncore = 0, nshell = 0, rebuilds = 0;
    int nact = 0;                      // shell entries kept by the last pruning
    int aslot16 = 0;                   // byte offset of the owned atom's table entry
    int n_ext = 0;                     // atoms + images in the table
    bool failed = false;
    float yb0 = 0.f, yb1 = 0.f, yb2 = 0.f;  // wrapped position at the build (FP32)
    float zp0 = 0.f, zp1 = 0.f, zp2 = 0.f;  // wrapped position at the last pruning (FP32)

    // ------------------------------------------------------------- rebuild
    // Wrap the owned atom and create its periodic images inside the
    // cutoff+skin margin of the cell; bin all entries (counting sort, index
    // order inside a bin); every atom scans the 5x5x5 bins around its own and
    // files each neighbour as core or shell.  If the shared-memory tables
    // overflow, the skin of this system shrinks by 10 % and the build is
    // retried (for the rest of the launch it keeps the skin that fits).
    //
    // list entries and the bin-sorted entry order hold byte offsets (entry * 16)
    // into the image table
#define EXT(OFF) (*(const float4 *)((const unsigned char *)s_ext + (OFF)))
    // file a candidate at byte offset E (position Q) as a core or shell
    // neighbour of the owned atom
#define TSB_FILE_PAIR(E, Q)                                                                  \
  {                                                                                          \
    const float dx = (Q).x - xi.x, dy = (Q).y - xi.y, dz = (Q).z - xi.z;                     \
    const float d2 = dx * dx + dy * dy + dz * dz;                                            \
    if (d2 < build2 && (E) != a16) {                                                         \
      const float cr2 = MULTI ? g.core2[sp * A.n_species + __float_as_int((Q).w)] : core0;   \
      if (ncore + nshell < kListLen) {                                                       \
        const int slot_ = d2 < cr2 ? ncore : kListLen - 1 - nshell;                          \
        list16[(((slot_ >> 2) * kFusedThreads + tid) << 2) | (slot_ & 3)] = (uint16_t)(E);   \
      }                                                                                      \
      if (d2 < cr2)                                                                          \
        ++ncore;                                                                             \
      else                                                                                   \
        ++nshell;                                                                            \
    }                                                                                        \
  }
#define TSB_REBUILD()                                                                        \
  for (;;) {                                                                                 \
    int over = 0, over_size = 0;                                                             \
    int gcount = 0;                                                                          \
    double f0 = 0, f1 = 0, f2 = 0, y0_ = 0, y1_ = 0, y2_ = 0;                                \
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
      wrapped(g, x0, x1, x2, Wx, Wy, Wz, y0_, y1_, y2_);                                     \
      yb0 = (float)y0_;                                                                      \
      yb1 = (float)y1_;                                                                      \
      yb2 = (float)y2_;                                                                      \
      if (lead) {                                                                            \
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
    const int goff = block_excl_scan_i<NT>(gcount, &total, s_scan);                              \
    n_ext = n + total;                                                                       \
    if (n_ext > kSentinel) { /* the last slot is the sentinel */                             \
      over = 1;                                                                              \
      over_size = n_ext;                                                                     \
    } else {                                                                                 \
      const int nbins = g.nbins;                                                             \
      for (int b = tid; b < nbins; b += kFusedThreads) s_bin[b] = 0;                         \
      /* the initial force reads of all lanes precede the scan's barriers */                 \
      if (lead) {                                                                            \
        s_ext[a] = make_float4(yb0, yb1, yb2, __int_as_float(sp));                           \
        Y[3 * a] = y0_;                                                                      \
        Y[3 * a + 1] = y1_;                                                                  \
        Y[3 * a + 2] = y2_;                                                                  \
        s_ebin[a] = (uint16_t)((bin_coord(g, f0, 0) * g.nb[1] + bin_coord(g, f1, 1)) *       \
                                   g.nb[2] +                                                 \
                               bin_coord(g, f2, 2));                                         \
        int gg = n + goff; /* the lead's ghost slots */                                      \
        for (int sx = -g.rep[0]; gcount && sx <= g.rep[0]; ++sx) {                           \
          if (!in_margin(g, f0 + sx, 0)) continue;                                           \
          const int bx = bin_coord(g, f0 + sx, 0);                                           \
          for (int sy = -g.rep[1]; sy <= g.rep[1]; ++sy) {                                   \
            if (!in_margin(g, f1 + sy, 1)) continue;                                         \
            const int bxy = bx * g.nb[1] + bin_coord(g, f1 + sy, 1);                         \
            for (int sz = -g.rep[2]; sz <= g.rep[2]; ++sz) {                                 \
              if (!in_margin(g, f2 + sz, 2)) continue;                                       \
              if ((sx | sy | sz) == 0) continue;                                             \
              s_ext[gg] = image_of(g, y0_, y1_, y2_, sx, sy, sz, sp);                        \
              s_gshift[gg - n] = pack_ghost(a, sx, sy, sz);                                  \
              s_ebin[gg] = (uint16_t)(bxy * g.nb[2] + bin_coord(g, f2 + sz, 2));             \
              ++gg;                                                                          \
            }                                                                                \
          }                                                                                  \
        }                                                                                    \
      }                                                                                      \
      __syncthreads();                                                                       \
      for (int e = tid; e < n_ext; e += kFusedThreads) atomicAdd(&s_bin[s_ebin[e]], 1);      \
      __syncthreads();                                                                       \
      {                                                                                      \
        const int b0 = 4 * tid;                                                              \
        int c4[4], sum = 0;                                                                  \
        for (int q = 0; q < 4; ++q) {                                                        \
          c4[q] = b0 + q < nbins ? s_bin[b0 + q] : 0;                                        \
          sum += c4[q];                                                                      \
        }                                                                                    \
        int tot_;                                                                            \
        int off = block_excl_scan_i<NT>(sum, &tot_, s_scan);                                     \
        for (int q = 0; q < 4; ++q) {                                                        \
          if (b0 + q < nbins) s_bin[b0 + q] = off;                                           \
          off += c4[q];                                                                      \
        }                                                                                    \
      }                                                                                      \
      __syncthreads();                                                                       \
      for (int e = tid; e < n_ext; e += kFusedThreads)                                       \
        s_sorted[atomicAdd(&s_bin[s_ebin[e]], 1)] = (uint16_t)(e << 4);                      \
      __syncthreads();                                                                       \
      /* s_bin[b] is now the end of bin b; order each bin by entry */                        \
      for (int b = tid; b < nbins; b += kFusedThreads) {                                     \
        const int lo_ = b ? s_bin[b - 1] : 0, hi_ = s_bin[b];                                \
        for (int i_ = lo_ + 1; i_ < hi_; ++i_) {                                             \
          const uint16_t v_ = s_sorted[i_];                                                  \
          int j_ = i_ - 1;                                                                   \
          while (j_ >= lo_ && s_sorted[j_] > v_) {                                           \
            s_sorted[j_ + 1] = s_sorted[j_];                                                 \
            --j_;                                                                            \
          }                                                                                  \
          s_sorted[j_ + 1] = v_;                                                             \
        }                                                                                    \
      }                                                                                      \
      __syncthreads();                                                                       \
      /* the table in bin order: entry p becomes generated entry s_sorted[p], its  */        \
      /* descriptor (owner, shift) beside it (atoms: shift 0); staged in the list   */       \
      /* area (free until the scan files entries), then copied back              */          \
      {                                                                                      \
        float4 *t_ext_ = (float4 *)s_list;                                                   \
        uint32_t *t_desc_ = (uint32_t *)(t_ext_ + kExtMax);                                  \
        for (int p = tid; p < n_ext; p += kFusedThreads) {                                   \
          const int e = s_sorted[p] >> 4;                                                    \
          t_ext_[p] = s_ext[e];                                                              \
          t_desc_[p] = e < n ? pack_ghost(e, 0, 0, 0) : s_gshift[e - n];                     \
        }                                                                                    \
        __syncthreads();                                                                     \
        uint16_t *aslot_ = s_sorted; /* slot of each atom's own entry */                     \
        for (int p = tid; p < n_ext; p += kFusedThreads) {                                   \
          const uint32_t d = t_desc_[p];                                                     \
          s_ext[p] = t_ext_[p];                                                              \
          s_gshift[p] = d;                                                                   \
          if ((d & 0x7FFFu) == 0) aslot_[d >> 15] = (uint16_t)p;                             \
        }                                                                                    \
        __syncthreads();                                                                     \
        aslot16 = own ? (int)aslot_[a] << 4 : 0;                                             \
      }                                                                                      \
      ncore = 0;                                                                             \
      nshell = 0;                                                                            \
      if (own) {                                                                             \
        const float4 xi = EXT(aslot16);                                                      \
        const float build2 = g.build2;                                                       \
        const float core0 = g.core2[0];                                                      \
        const int a16 = aslot16;                                                             \
        /* bins within the list radius in each fractional coordinate; per bin row */        \
        /* (cx, cy) the z range left by the row's gaps gx, gy to the atom:          */       \
        /* |d|^2 >= lambda (|a_x|^2 gx^2 + |a_y|^2 gy^2 + |a_z|^2 du_z^2)           */       \
        const float fx_ = (float)f0, fy_ = (float)f1, fz_ = (float)f2;                       \
        const float rl2_ = g.build2 * 1.00001f * g.ilam;                                     \
        const int xlo_ = max((int)floorf((fx_ - g.stw[0] + g.sh[0]) * g.siw[0]), 0);         \
        const int xhi_ = min((int)floorf((fx_ + g.stw[0] + g.sh[0]) * g.siw[0]), g.nb[0] - 1); \
        const int ylo_ = max((int)floorf((fy_ - g.stw[1] + g.sh[1]) * g.siw[1]), 0);         \
        const int yhi_ = min((int)floorf((fy_ + g.stw[1] + g.sh[1]) * g.siw[1]), g.nb[1] - 1); \
        for (int cx = xlo_; cx <= xhi_; ++cx) {                                              \
          const float bl_ = (float)cx * g.sw[0] - g.sh[0];                                   \
          const float gx_ = fmaxf(fmaxf(bl_ - fx_, fx_ - (bl_ + g.sw[0])) - 1e-5f, 0.0f);    \
          const float qx_ = rl2_ - g.alen2[0] * gx_ * gx_;                                   \
          for (int cy = ylo_; cy <= yhi_; ++cy) {                                            \
            const float cl_ = (float)cy * g.sw[1] - g.sh[1];                                 \
            const float gy_ = fmaxf(fmaxf(cl_ - fy_, fy_ - (cl_ + g.sw[1])) - 1e-5f, 0.0f);  \
            const float rem_ = qx_ - g.alen2[1] * gy_ * gy_;                                 \
            if (rem_ < 0.0f) continue;                                                       \
            const float zw_ = fminf(g.stw[2], sqrtf(rem_ / g.alen2[2]) + 1e-5f);             \
            const int zlo = max((int)floorf((fz_ - zw_ + g.sh[2]) * g.siw[2]), 0);           \
            const int zhi = min((int)floorf((fz_ + zw_ + g.sh[2]) * g.siw[2]), g.nb[2] - 1); \
            if (zlo > zhi) continue;                                                         \
            const int row = (cx * g.nb[1] + cy) * g.nb[2];                                   \
            const int plo = (row + zlo) ? s_bin[row + zlo - 1] : 0;                          \
            const int phi = s_bin[row + zhi];                                                \
            /* four candidates per iteration (independent loads), kept in order; */          \
            /* positions past the row read the far sentinel entry instead        */          \
            for (int p_ = plo + lane; p_ < phi; p_ += 4 * tpa) {                             \
              const int e0 = p_ << 4;                                                        \
              const int e1 = p_ + tpa < phi ? (p_ + tpa) << 4 : kSentinel << 4;              \
              const int e2 = p_ + 2 * tpa < phi ? (p_ + 2 * tpa) << 4 : kSentinel << 4;      \
              const int e3 = p_ + 3 * tpa < phi ? (p_ + 3 * tpa) << 4 : kSentinel << 4;      \
              const float4 q0 = EXT(e0), q1 = EXT(e1), q2 = EXT(e2), q3 = EXT(e3);           \
              TSB_FILE_PAIR(e0, q0)                                                          \
              TSB_FILE_PAIR(e1, q1)                                                          \
              TSB_FILE_PAIR(e2, q2)                                                          \
              TSB_FILE_PAIR(e3, q3)                                                          \
            }                                                                                \
          }                                                                                  \
        }                                                                                    \
      }                                                                                      \
      if (own && ncore + nshell <= kListLen) {                                               \
        /* whole groups of four: the last ncore % 4 core pairs join the shell (they  */      \
        /* pass its cutoff test anyway), and the shell is padded to a multiple of 4 */       \
        /* with the far sentinel entry, so no lane has a partial group to handle    */       \
        const int extra_ = ncore & 3;                                                        \
        for (int k_ = 0; k_ < extra_; ++k_) {                                                \
          const int from_ = ncore - 1 - k_, to_ = kListLen - 1 - nshell;                     \
          list16[(((to_ >> 2) * kFusedThreads + tid) << 2) | (to_ & 3)] =                    \
              list16[(((from_ >> 2) * kFusedThreads + tid) << 2) | (from_ & 3)];             \
          ++nshell;                                                                          \
        }                                                                                    \
        ncore -= extra_;                                                                     \
        while (nshell & 3) {                                                                 \
          const int to_ = kListLen - 1 - nshell;                                             \
          list16[(((to_ >> 2) * kFusedThreads + tid) << 2) | (to_ & 3)] =                    \
              (uint16_t)(kSentinel << 4);                                                    \
          ++nshell;                                                                          \
        }                                                                                    \
      }                                                                                      \
      if (__syncthreads_or(ncore + nshell > kListLen)) {                                     \
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
      g.skin = g.skin > 0.05 ? 0.9 * g.skin : 0.0;                                           \
      set_margins<kMaxBins>(g, A.cutoff, A.prune, rc2d, nsp2);                                                  \
    }                                                                                        \
    __syncthreads();                                                                         \
  }

    // ------------------------------------------------------------ pruning
    // Each thread reorders its own shell entries (no other thread reads them):
    // those closer than sqrt(act2) go to the front part [0, nact), which is all
    // the force loop evaluates of the shell until the next pruning.  After a
    // list build the whole shell is partitioned (FROM = 0).  Between builds only
    // the entries outside the front part are examined (FROM = nact): those now
    // within reach join it; entries of the front part that moved out stay in it
    // (they are evaluated with the cutoff test, so results do not change) until
    // the next build.  The atom's FP32 position in the table is the one the
    // next pruning test measures from.  Without pruning, the whole shell is
    // evaluated.
#define TSB_PRUNE_STEP(I, E, ACT)                                                            \
  {                                                                                          \
    const int k_ = 4 * j_ + (I);                                                             \
    if ((ACT) && k_ >= from_) {                                                              \
      if (w_ != k_) { /* the entry at w_ (outside reach) moves to k_ */                      \
        const int sw_ = kListLen - 1 - w_, sk_ = kListLen - 1 - k_;                          \
        const int iw_ = (((sw_ >> 2) * kFusedThreads + tid) << 2) | (sw_ & 3);              \
        const int ik_ = (((sk_ >> 2) * kFusedThreads + tid) << 2) | (sk_ & 3);              \
        list16[ik_] = list16[iw_];                                                           \
        list16[iw_] = (uint16_t)(E);                                                         \
      }                                                                                      \
      ++w_;                                                                                  \
    }                                                                                        \
  }
#define TSB_PRUNE(FROM)                                                                      \
  if (g.prune_on) {                                                                          \
    if (own) {                                                                               \
      const float4 xi_ = EXT(aslot16);                                                       \
      const float act2_ = g.act2;                                                            \
      const int from_ = (FROM);                                                              \
      int w_ = from_;                                                                        \
      /* groups of four shell entries (shell entry 4j + i sits in slot        */             \
      /* kListLen - 1 - 4j - i), the next group's word loaded one ahead; the  */             \
      /* group's four distances first, then its entries in order             */             \
      uint2 gn_ = s_list[max(kListGroups - 1 - (from_ >> 2), 0) * kFusedThreads + tid];    \
      for (int j_ = from_ >> 2; j_ < (nshell >> 2); ++j_) {                                  \
        const uint2 ge_ = gn_;                                                               \
        gn_ = s_list[max(kListGroups - 2 - j_, 0) * kFusedThreads + tid];                    \
        const uint32_t e0_ = ge_.y >> 16, e1_ = ge_.y & 0xFFFFu;                             \
        const uint32_t e2_ = ge_.x >> 16, e3_ = ge_.x & 0xFFFFu;                             \
        const float4 q0_ = EXT(e0_), q1_ = EXT(e1_), q2_ = EXT(e2_), q3_ = EXT(e3_);         \
        bool a0_, a1_, a2_, a3_;                                                             \
        {                                                                                    \
          float dx_ = q0_.x - xi_.x, dy_ = q0_.y - xi_.y, dz_ = q0_.z - xi_.z;               \
          a0_ = dx_ * dx_ + dy_ * dy_ + dz_ * dz_ < act2_;                                   \
          dx_ = q1_.x - xi_.x, dy_ = q1_.y - xi_.y, dz_ = q1_.z - xi_.z;                     \
          a1_ = dx_ * dx_ + dy_ * dy_ + dz_ * dz_ < act2_;                                   \
          dx_ = q2_.x - xi_.x, dy_ = q2_.y - xi_.y, dz_ = q2_.z - xi_.z;                     \
          a2_ = dx_ * dx_ + dy_ * dy_ + dz_ * dz_ < act2_;                                   \
          dx_ = q3_.x - xi_.x, dy_ = q3_.y - xi_.y, dz_ = q3_.z - xi_.z;                     \
          a3_ = dx_ * dx_ + dy_ * dy_ + dz_ * dz_ < act2_;                                   \
        }                                                                                    \
        TSB_PRUNE_STEP(0, e0_, a0_)                                                          \
        TSB_PRUNE_STEP(1, e1_, a1_)                                                          \
        TSB_PRUNE_STEP(2, e2_, a2_)                                                          \
        TSB_PRUNE_STEP(3, e3_, a3_)                                                          \
      }                                                                                      \
      nact = w_;                                                                             \
      zp0 = xi_.x;                                                                           \
      zp1 = xi_.y;                                                                           \
      zp2 = xi_.z;                                                                           \
    }                                                                                        \
  } else {                                                                                   \
    nact = nshell;                                                                           \
  }

    // ------------------------------------------------------------ pair loop
    // Four list entries per iteration, branch-free (out-of-range pairs are
    // evaluated and masked), so the loads and the math of the four pairs
    // overlap.  Core pairs need no cutoff test.
  // pair virial fr d (x) d (the same for d and -d), FP32 products summed in FP64
#define TSB_VIR1(FR, DX, DY, DZ)                                                             \
  {                                                                                          \
    const float tx_ = (FR) * (DX), ty_ = (FR) * (DY), tz_ = (FR) * (DZ);                     \
    vxx += (double)(tx_ * (DX));                                                             \
    vyy += (double)(ty_ * (DY));                                                             \
    vzz += (double)(tz_ * (DZ));                                                             \
    vyz += (double)(ty_ * (DZ));                                                             \
    vxz += (double)(tx_ * (DZ));                                                             \
    vxy += (double)(tx_ * (DY));                                                             \
  }
#define TSB_PAIR_CORE(Q, WITH_E)                                                             \
  {                                                                                          \
    const float4 q = (Q);                                                                    \
    const float rx = q.x - xi.x, ry = q.y - xi.y, rz = q.z - xi.z;                           \
    const float r2 = fmaxf(rx * rx + ry * ry + rz * rz, 1e-30f);                             \
    const PairPrm<float> &pq = MULTI ? row[__float_as_int(q.w)] : p0;                        \
    float ep, fr;                                                                            \
    pair_eval_fast<POT>(pq, r2, ep, fr);                                                     \
    fx -= fr * rx;                                                                           \
    fy -= fr * ry;                                                                           \
    fz -= fr * rz;                                                                           \
    if (WITH_E) {                                                                            \
      en += (double)ep;                                                                      \
      TSB_VIR1(fr, rx, ry, rz)                                                               \
    }                                                                                        \
  }
#define TSB_PAIR_SHELL(Q, E, WITH_E)                                                         \
  {                                                                                          \
    const float4 q = (Q);                                                                    \
    const float rx = q.x - xi.x, ry = q.y - xi.y, rz = q.z - xi.z;                           \
    const float r2 = fmaxf(rx * rx + ry * ry + rz * rz, 1e-30f);                             \
    const PairPrm<float> &pq = MULTI ? row[__float_as_int(q.w)] : p0;                        \
    float ep, fr;                                                                            \
    pair_eval_fast<POT>(pq, r2, ep, fr);                                                     \
    bool in_ = r2 < pq.a3;                                                                   \
    if (fabsf(r2 - pq.a3) < band_)                                                           \
      in_ = exact_r2(Y, s_gshift, g, a, (int)((E) >> 4)) <                                \
            (MULTI ? rc2d[sp * A.n_species + __float_as_int(q.w)] : rc2d0);                  \
    fr = in_ ? fr : 0.f;                                                                     \
    fx -= fr * rx;                                                                           \
    fy -= fr * ry;                                                                           \
    fz -= fr * rz;                                                                           \
    if (WITH_E) {                                                                            \
      en += in_ ? (double)ep : 0.0;                                                          \
      TSB_VIR1(fr, rx, ry, rz)                                                               \
    }                                                                                        \
  }
  // two list entries at once (FP32x2); displacement xi - q so that the force
  // accumulates as f += fr * d
#define TSB_PAIR2(QA, QB, EA, EB, SHELL, WITH_E)                                             \
  {                                                                                          \
    const float4 qa = (QA), qb = (QB);                                                       \
    const float2 dx = make_float2(xi.x - qa.x, xi.x - qb.x);                                 \
    const float2 dy = make_float2(xi.y - qa.y, xi.y - qb.y);                                 \
    const float2 dz = make_float2(xi.z - qa.z, xi.z - qb.z);                                 \
    float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));                  \
    /* shell entries include the far sentinel; core pairs are never at r = 0 */          \
    if (SHELL) r2 = make_float2(fmaxf(r2.x, 1e-30f), fmaxf(r2.y, 1e-30f));                   \
    float2 e2;                                                                               \
    float2 fr = pair_fr2<POT, WITH_E>(k2, p0, r2, e2);                                       \
    if (SHELL) {                                                                             \
      bool ina = r2.x < p0.a3, inb = r2.y < p0.a3;                                           \
      const bool near_a = fabsf(r2.x - p0.a3) < band_;                                       \
      const bool near_b = fabsf(r2.y - p0.a3) < band_;                                       \
      if (near_a || near_b) { /* rare: one branch for both pairs */                          \
        if (near_a) ina = exact_r2(Y, s_gshift, g, a, (int)((EA) >> 4)) < rc2d0;          \
        if (near_b) inb = exact_r2(Y, s_gshift, g, a, (int)((EB) >> 4)) < rc2d0;          \
      }                                                                                      \
      fr = make_float2(ina ? fr.x : 0.f, inb ? fr.y : 0.f);                                  \
      if (WITH_E) e2 = make_float2(ina ? e2.x : 0.f, inb ? e2.y : 0.f);                      \
    }                                                                                        \
    f2x = __ffma2_rn(fr, dx, f2x);                                                           \
    f2y = __ffma2_rn(fr, dy, f2y);                                                           \
    f2z = __ffma2_rn(fr, dz, f2z);                                                           \
    if (WITH_E) {                                                                            \
      en += (double)e2.x + (double)e2.y;                                                     \
      TSB_VIR1(fr.x, dx.x, dy.x, dz.x)                                                       \
      TSB_VIR1(fr.y, dx.y, dy.y, dz.y)                                                       \
    }                                                                                        \
  }
#define TSB_FORCES(WITH_E)                                                                   \
  {                                                                                          \
    float fx = 0.f, fy = 0.f, fz = 0.f;                                                      \
    double en = 0.0, vxx = 0.0, vyy = 0.0, vzz = 0.0, vyz = 0.0, vxz = 0.0, vxy = 0.0;        \
    if (own) {                                                                               \
      const float4 xi = EXT(aslot16);                                                        \
      const float band_ = g.band;                                                            \
      const PairPrm<float> *row = prm + sp * A.n_species;                                    \
      (void)row;                                                                             \
      const int full = ncore >> 2, rem = ncore & 3;                                          \
      /* the pruned shell in whole groups of four (a group's tail entries beyond */           \
      /* nact are shell entries outside the cutoff, or the far sentinel)         */           \
      const int sfull = (nact + 3) >> 2, srem = 0;                                           \
      if constexpr (kPaired) {                                                               \
        float2 f2x = make_float2(0.f, 0.f), f2y = f2x, f2z = f2x;                            \
        /* the next group's list word loads one iteration ahead (in-bounds index) */         \
        uint2 gn = s_list[tid];                                                              \
        for (int k4 = 0; k4 < full; ++k4) {                                                  \
          const uint2 ge = gn;                                                               \
          gn = s_list[min(k4 + 1, kListGroups - 1) * kFusedThreads + tid];                   \
          TSB_PAIR2(EXT(ge.x & 0xFFFFu), EXT(ge.x >> 16), 0, 0, false, WITH_E)           \
          TSB_PAIR2(EXT(ge.y & 0xFFFFu), EXT(ge.y >> 16), 0, 0, false, WITH_E)           \
        }                                                                                    \
        if (rem) {                                                                           \
          const uint2 ge = gn; /* group `full` */                                            \
          if (rem > 1) {                                                                     \
            TSB_PAIR2(EXT(ge.x & 0xFFFFu), EXT(ge.x >> 16), 0, 0, false, WITH_E)         \
            if (rem > 2) TSB_PAIR_CORE(EXT(ge.y & 0xFFFFu), WITH_E)                        \
          } else {                                                                           \
            TSB_PAIR_CORE(EXT(ge.x & 0xFFFFu), WITH_E)                                     \
          }                                                                                  \
        }                                                                                    \
        /* shell entry k sits in slot kListLen - 1 - k */                                    \
        uint2 gs = s_list[(kListGroups - 1) * kFusedThreads + tid];                          \
        for (int k4 = 0; k4 < sfull; ++k4) {                                                 \
          const uint2 ge = gs;                                                               \
          gs = s_list[max(kListGroups - 2 - k4, 0) * kFusedThreads + tid];                   \
          TSB_PAIR2(EXT(ge.y >> 16), EXT(ge.y & 0xFFFFu), ge.y >> 16, ge.y & 0xFFFFu,    \
                    true, WITH_E)                                                            \
          TSB_PAIR2(EXT(ge.x >> 16), EXT(ge.x & 0xFFFFu), ge.x >> 16, ge.x & 0xFFFFu,    \
                    true, WITH_E)                                                            \
        }                                                                                    \
        if (srem) {                                                                          \
          const uint2 ge = gs; /* group kListGroups - 1 - sfull */                           \
          if (srem > 1) {                                                                    \
            TSB_PAIR2(EXT(ge.y >> 16), EXT(ge.y & 0xFFFFu), ge.y >> 16, ge.y & 0xFFFFu,  \
                      true, WITH_E)                                                          \
            if (srem > 2) TSB_PAIR_SHELL(EXT(ge.x >> 16), ge.x >> 16, WITH_E)              \
          } else {                                                                           \
            TSB_PAIR_SHELL(EXT(ge.y >> 16), ge.y >> 16, WITH_E)                            \
          }                                                                                  \
        }                                                                                    \
        fx += f2x.x + f2x.y;                                                                 \
        fy += f2y.x + f2y.y;                                                                 \
        fz += f2z.x + f2z.y;                                                                 \
      } else {                                                                               \
        for (int k4 = 0; k4 < full; ++k4) {                                                  \
          const uint2 ge = s_list[k4 * kFusedThreads + tid];                                 \
          TSB_PAIR_CORE(EXT(ge.x & 0xFFFFu), WITH_E)                                       \
          TSB_PAIR_CORE(EXT(ge.x >> 16), WITH_E)                                           \
          TSB_PAIR_CORE(EXT(ge.y & 0xFFFFu), WITH_E)                                       \
          TSB_PAIR_CORE(EXT(ge.y >> 16), WITH_E)                                           \
        }                                                                                    \
        if (rem) {                                                                           \
          const uint2 ge = s_list[full * kFusedThreads + tid];                               \
          TSB_PAIR_CORE(EXT(ge.x & 0xFFFFu), WITH_E)                                       \
          if (rem > 1) TSB_PAIR_CORE(EXT(ge.x >> 16), WITH_E)                              \
          if (rem > 2) TSB_PAIR_CORE(EXT(ge.y & 0xFFFFu), WITH_E)                          \
        }                                                                                    \
        /* shell entry k sits in slot kListLen - 1 - k */                                    \
        for (int k4 = 0; k4 < sfull; ++k4) {                                                 \
          const uint2 ge = s_list[(kListGroups - 1 - k4) * kFusedThreads + tid];             \
          TSB_PAIR_SHELL(EXT(ge.y >> 16), ge.y >> 16, WITH_E)                              \
          TSB_PAIR_SHELL(EXT(ge.y & 0xFFFFu), ge.y & 0xFFFFu, WITH_E)                      \
          TSB_PAIR_SHELL(EXT(ge.x >> 16), ge.x >> 16, WITH_E)                              \
          TSB_PAIR_SHELL(EXT(ge.x & 0xFFFFu), ge.x & 0xFFFFu, WITH_E)                      \
        }                                                                                    \
        if (srem) {                                                                          \
          const uint2 ge = s_list[(kListGroups - 1 - sfull) * kFusedThreads + tid];          \
          TSB_PAIR_SHELL(EXT(ge.y >> 16), ge.y >> 16, WITH_E)                              \
          if (srem > 1) TSB_PAIR_SHELL(EXT(ge.y & 0xFFFFu), ge.y & 0xFFFFu, WITH_E)        \
          if (srem > 2) TSB_PAIR_SHELL(EXT(ge.x >> 16), ge.x >> 16, WITH_E)                \
        }                                                                                    \
      }                                                                                      \
    }                                                                                        \
    for (int o = 1; o < tpa; o <<= 1) {                                                      \
      fx += __shfl_xor_sync(0xffffffffu, fx, o);                                             \
      fy += __shfl_xor_sync(0xffffffffu, fy, o);                                             \
      fz += __shfl_xor_sync(0xffffffffu, fz, o);                                             \
      if (WITH_E) {                                                                          \
        en += __shfl_xor_sync(0xffffffffu, en, o);                                           \
        vxx += __shfl_xor_sync(0xffffffffu, vxx, o);                                         \
        vyy += __shfl_xor_sync(0xffffffffu, vyy, o);                                         \
        vzz += __shfl_xor_sync(0xffffffffu, vzz, o);                                         \
        vyz += __shfl_xor_sync(0xffffffffu, vyz, o);                                         \
        vxz += __shfl_xor_sync(0xffffffffu, vxz, o);                                         \
        vxy += __shfl_xor_sync(0xffffffffu, vxy, o);                                         \
      }                                                                                      \
    }                                                                                        \
    F0 = fx;                                                                                 \
    F1 = fy;                                                                                 \
    F2 = fz;                                                                                 \
    if (WITH_E) {                                                                            \
      /* each pair is seen from both ends: half weight; FP64 sums over the block */         \
      const double h_ = lead ? 0.5 : 0.0;                                                    \
      warp_sum_store(h_ * en, s_red7[0]);                                                    \
      warp_sum_store(h_ * vxx, s_red7[1]);                                                   \
      warp_sum_store(h_ * vyy, s_red7[2]);                                                   \
      warp_sum_store(h_ * vzz, s_red7[3]);                                                   \
      warp_sum_store(h_ * vyz, s_red7[4]);                                                   \
      warp_sum_store(h_ * vxz, s_red7[5]);                                                   \
      warp_sum_store(h_ * vxy, s_red7[6]);                                                   \
      __syncthreads();                                                                       \
      if (tid == 0) warps_sum7<NT>(s_red7, g.esum7);                                             \
      __syncthreads();                                                                       \
    }                                                                                        \
  }

    TSB_REBUILD()
    if (failed) continue;
    TSB_PRUNE(0)
    for (int64_t step = 0; step < A.n_steps; ++step) {
      const double dt = g.dt, half = g.half, c1 = g.c1;
      // thermostat before the step: V-rescale factor from the current kinetic
      // energy (nvt.py:715-741), or the first Nose-Hoover half step with the
      // kinetic energy carried from the last one (nvt.py:462-470)
      if (integ == TSB_INT_VRESCALE) {
        const double k2 = block_sum_to0<NT>(lead ? (px * px + py * py + pz * pz) * inv_m : 0.0,
                                        s_red);
        if (tid == 0)
          g.th_scale = vrescale_lambda(k2, g.nf, g.kt, dt, g.tau, nullptr, A.seed, s,
                                       counter0 + (uint64_t)step);
        __syncthreads();
        const double sc = g.th_scale;
        px *= sc;
        py *= sc;
        pz *= sc;
      } else if (integ == TSB_INT_NOSE_HOOVER) {
        if (tid == 0)
          g.th_scale = nhc_half(g.cdt, A.M, A.nc, A.nsy, g.cq, g.cx, g.cv, g.cke, g.nf, g.kt);
        __syncthreads();
        const double sc = g.th_scale;
        px *= sc;
        py *= sc;
        pz *= sc;
      }
      if (own) {
        px += F0 * half;
        py += F1 * half;
        pz += F2 * half;
        if (integ == TSB_INT_LANGEVIN) {
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
      // displacement since the build and since the last pruning, in FP64 on
      // the wrapped position; the new position goes to the staging table
      double y0 = 0.0, y1 = 0.0, y2 = 0.0;
      int flag = 0;
      if (own) {
        wrapped(g, x0, x1, x2, Wx, Wy, Wz, y0, y1, y2);
        const double d0 = y0 - yb0, d1 = y1 - yb1, d2 = y2 - yb2;
        if (d0 * d0 + d1 * d1 + d2 * d2 > g.half_skin2) flag |= 1;
        const double e0 = y0 - zp0, e1 = y1 - zp1, e2 = y2 - zp2;
        const double ee = e0 * e0 + e1 * e1 + e2 * e2;
        if (ee > g.half_prune2) flag |= 2;
        if (lead) {
          s_posd[3 * a] = y0;
          s_posd[3 * a + 1] = y1;
          s_posd[3 * a + 2] = y2;
        }
      }
      // all warps are done reading the previous positions
      __syncthreads();
      // refresh: every thread rewrites an even share of the table, each entry
      // fl32 of its FP64 value (atom, or owner + lattice shift), so that the
      // rounding errors of different entries are independent (FP32 shift
      // arithmetic would give every image of one shift the same error)
      if (lead) {
        Y[3 * a] = y0;
        Y[3 * a + 1] = y1;
        Y[3 * a + 2] = y2;
      }
      for (int e = tid; e < n_ext; e += kFusedThreads) {
        const int sp_e = MULTI ? __float_as_int(s_ext[e].w) : 0;
        int owner, sx, sy, sz;
        unpack_ghost(s_gshift[e], owner, sx, sy, sz);
        s_ext[e] = image_of(g, s_posd[3 * owner], s_posd[3 * owner + 1],
                            s_posd[3 * owner + 2], sx, sy, sz, sp_e);
      }
      {
        const int wf = __reduce_or_sync(0xffffffffu, flag);
        if ((tid & 31) == 0 && wf) atomicOr(&s_flags[step & 1], wf);
      }
      __syncthreads();
      const int fl = s_flags[step & 1];
      if (tid == 0) s_flags[(step + 1) & 1] = 0;
      if (fl & 1) {
        TSB_REBUILD()
        if (failed) break;
        TSB_PRUNE(0)
      } else if (fl & 2) {
        TSB_PRUNE(nact)
      }
      const bool report = A.rep_every > 0 && (step + 1) % A.rep_every == 0 &&
                          (step + 1) / A.rep_every <= A.n_frames;
      if (step + 1 == A.n_steps || report) {
        TSB_FORCES(true)
      } else {
        TSB_FORCES(false)
      }
      if (own) {
        px += F0 * g.half;
        py += F1 * g.half;
        pz += F2 * g.half;
      }
      if (integ == TSB_INT_NOSE_HOOVER) {
        // second half step with the kinetic energy after velocity Verlet
        const double k2 = block_sum_to0<NT>(lead ? (px * px + py * py + pz * pz) * inv_m : 0.0,
                                        s_red);
        if (tid == 0) {
          g.cke = 0.5 * k2;
          g.th_scale = nhc_half(g.cdt, A.M, A.nc, A.nsy, g.cq, g.cx, g.cv, g.cke, g.nf, g.kt);
        }
        __syncthreads();
        const double sc = g.th_scale;
        px *= sc;
        py *= sc;
        pz *= sc;
      }
      if (report) {
        // frame f: FP32 positions (as the reference's trajectories store them by
        // default) and the system's potential energy at this step
        const int64_t f = (step + 1) / A.rep_every - 1;
        if (lead) {
          float *o = A.frame_x + 3 * (f * A.n_atoms_total + gi);
          o[0] = (float)x0;
          o[1] = (float)x1;
          o[2] = (float)x2;
        }
        if (tid == 0) A.frame_e[f * A.n_sys + s] = g.esum7[0];
      }
    }
    if (failed) continue;
    if (A.n_steps == 0) TSB_FORCES(true)
#undef TSB_FORCES
#undef TSB_PAIR_CORE
#undef TSB_PAIR_SHELL
#undef TSB_PAIR2
#undef TSB_VIR1
#undef EXT
#undef TSB_REBUILD
#undef TSB_PRUNE
#undef TSB_PRUNE_STEP
#undef TSB_FILE_PAIR
    // ---- write back + FP64 energy reduction (each pair seen from both ends)
    __syncthreads();  // every lane is done reading Y before forces overwrite it
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
    if (tid == 0) {
      A.energy[s] = g.esum7[0];
      if (A.stress) {
        // stress = -W / V (torch_sim/models/pair_potential.py:200-274)
        const double *w = g.esum7 + 1;
        const double *C = g.C;
        const double vol = fabs(C[0] * (C[4] * C[8] - C[5] * C[7]) -
                                C[1] * (C[3] * C[8] - C[5] * C[6]) +
                                C[2] * (C[3] * C[7] - C[4] * C[6]));
        const double iv = -1.0 / vol;
        double *o = A.stress + 9 * s;
        o[0] = w[0] * iv;
        o[4] = w[1] * iv;
        o[8] = w[2] * iv;
        o[5] = o[7] = w[3] * iv;
        o[2] = o[6] = w[4] * iv;
        o[1] = o[3] = w[5] * iv;
      }
      if (A.n_rebuilds) A.n_rebuilds[s] = rebuilds;
      if (integ == TSB_INT_NOSE_HOOVER) {
        for (int j = 0; j < A.M; ++j) {
          A.cxi[s * A.M + j] = g.cx[j];
          A.cpxi[s * A.M + j] = g.cv[j];
          A.cQ[s * A.M + j] = g.cq[j];
        }
        A.cke[s] = g.cke;
      }
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

// Atom range [lo[s], hi[s]) of every system from the sorted system index.  An
// index outside [0, n_sys) is reported in status (code, atom, 3, index) and
// skipped, so nothing is written outside lo/hi.
__global__ void k_bounds_fused(const int64_t *sys, int64_t n, int64_t n_sys, int64_t *lo,
                               int64_t *hi, int32_t *status) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t s = sys[i];
  if (s < 0 || s >= n_sys) {
    report(status, TSB_ERR_INVALID_ARG, i, 3, (int)(s < INT32_MIN ? INT32_MIN
                                                    : s > INT32_MAX ? INT32_MAX : s));
    return;
  }
  if (i == 0 || sys[i - 1] != s) lo[s] = i;
  if (i == n - 1 || sys[i + 1] != s) hi[s] = i + 1;
}

template <int POT, bool MULTI, int NT, int INTEG = -1>
static void launch_fused(const FusedArgs &A, int64_t grid, cudaStream_t st) {
  cudaFuncSetAttribute(k_fused_md<POT, MULTI, NT, INTEG>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FusedSmem<NT>::kTotal);
  k_fused_md<POT, MULTI, NT, INTEG><<<(unsigned)grid, NT, FusedSmem<NT>::kTotal, st>>>(A);
}

template <int NT>
static void launch_shape(const FusedArgs &A, int64_t grid, cudaStream_t st) {
  const bool multi = A.n_species > 1;
  const bool lgv = A.integrator == TSB_INT_LANGEVIN;
  if (A.potential == TSB_POT_LJ) {
    if (multi) launch_fused<TSB_POT_LJ, true, NT>(A, grid, st);
    else if (lgv) launch_fused<TSB_POT_LJ, false, NT, TSB_INT_LANGEVIN>(A, grid, st);
    else launch_fused<TSB_POT_LJ, false, NT>(A, grid, st);
  } else if (A.potential == TSB_POT_MORSE) {
    if (multi) launch_fused<TSB_POT_MORSE, true, NT>(A, grid, st);
    else if (lgv) launch_fused<TSB_POT_MORSE, false, NT, TSB_INT_LANGEVIN>(A, grid, st);
    else launch_fused<TSB_POT_MORSE, false, NT>(A, grid, st);
  } else {
    multi ? launch_fused<TSB_POT_SOFT, true, NT>(A, grid, st)
          : launch_fused<TSB_POT_SOFT, false, NT>(A, grid, st);
  }
}

// A second stream per device for the narrow launch, created on first use.
constexpr int kSideDevices = 64;
static cudaStream_t g_side_stream[kSideDevices];
static std::mutex g_side_mu;

static cudaStream_t side_stream() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kSideDevices) return nullptr;
  std::lock_guard<std::mutex> lock(g_side_mu);
  if (!g_side_stream[dev] &&
      cudaStreamCreateWithFlags(&g_side_stream[dev], cudaStreamNonBlocking) != cudaSuccess)
    g_side_stream[dev] = nullptr;
  return g_side_stream[dev];
}

// One persistent launch over all systems (wide blocks), or, with an order whose
// first n_wide systems need wide blocks, a wide launch over those and a narrow
// launch (two blocks per SM) over the rest.  The narrow launch goes on a side
// stream forked from `st` after the wide one, so its blocks take the SMs the
// wide blocks leave at the end of their work (the two launches' tails overlap),
// and `st` waits for it before anything after this call.  queue[0] and
// queue[1] are the two launches' work counters (zeroed before).
static void launch_all(FusedArgs A, int64_t n_wide, int32_t *queue, cudaStream_t st) {
  int dev = 0, n_sm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  const int64_t n = A.n_sys;
  if (!A.order || n_wide < 0 || n_wide >= n) {
    A.n_work = n;
    A.queue = queue;
    launch_shape<512>(A, std::min<int64_t>(std::min<int64_t>(n_sm, kMaxGrid), n), st);
    return;
  }
  FusedArgs Nw = A;
  Nw.order = A.order + n_wide;
  Nw.n_work = n - n_wide;
  Nw.queue = queue + 1;
  const int64_t grid_n = std::min<int64_t>(std::min<int64_t>(2 * n_sm, 2 * kMaxGrid), n - n_wide);
  cudaStream_t side = n_wide > 0 ? side_stream() : nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  if (side && (cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) != cudaSuccess ||
               cudaEventCreateWithFlags(&join, cudaEventDisableTiming) != cudaSuccess))
    side = nullptr;
  if (side) cudaEventRecord(fork, st);
  if (n_wide > 0) {
    FusedArgs W = A;
    W.n_work = n_wide;
    W.queue = queue;
    launch_shape<512>(W, std::min<int64_t>(std::min<int64_t>(n_sm, kMaxGrid), n_wide), st);
  }
  if (side) {
    cudaStreamWaitEvent(side, fork, 0);
    launch_shape<256>(Nw, grid_n, side);
    cudaEventRecord(join, side);
    cudaStreamWaitEvent(st, join, 0);
  } else {
    launch_shape<256>(Nw, grid_n, st);
  }
  if (fork) cudaEventDestroy(fork);
  if (join) cudaEventDestroy(join);
}

extern "C" int tsb_fused_md(int integrator, int potential, const double *table,
                            int n_species, const int32_t *species, double *positions,
                            double *momenta, double *forces, const double *masses,
                            const double *cell_row, const int64_t *system_idx,
                            int64_t n_atoms, int64_t n_systems, const int32_t *order,
                            double cutoff, double skin, int64_t n_steps,
                            const double *dt_sys, const double *kT_sys,
                            const double *gamma_sys, uint64_t seed, uint64_t counter,
                            uint64_t *counter_dev, double *energy, double *stress,
                            int32_t *n_rebuilds, int32_t *status, void *workspace,
                            size_t workspace_bytes, void *stream) {
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
  cudaMemsetAsync(lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(hi, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(queue, 0, sizeof(int32_t) * 4, st);
  cudaMemsetAsync(status, 0, sizeof(int32_t) * 4, st);
  k_bounds_fused<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, n_systems, lo,
                                                       hi, status);
  FusedArgs A{integrator, potential, n_species, table, species, positions, momenta, forces,
              masses, cell_row, lo, hi, n_systems, order, cutoff, skin, n_steps, dt_sys,
              kT_sys, gamma_sys, seed, counter, counter_dev, energy, n_rebuilds, queue,
              status};
  A.stress = stress;
  launch_all(A, -1, queue, st);
  if (counter_dev) k_advance_counter<<<1, 32, 0, st>>>(counter_dev, n_steps);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_fused_md_nvt(int thermostat, int potential, const double *table,
                                int n_species, const int32_t *species, double *positions,
                                double *momenta, double *forces, const double *masses,
                                const double *cell_row, const int64_t *system_idx,
                                int64_t n_atoms, int64_t n_systems, const int32_t *order,
                                double cutoff, double skin, int64_t n_steps,
                                const double *dt_sys, const double *kT_sys,
                                const double *tau_sys, double *chain_xi, double *chain_pxi,
                                double *chain_Q, double *chain_ke, const double *chain_dt,
                                int chain_length, int chain_steps, int sy_steps, uint64_t seed,
                                uint64_t counter, uint64_t *counter_dev, double *energy,
                                double *stress, int32_t *n_rebuilds, int32_t *status,
                                void *workspace, size_t workspace_bytes, void *stream) {
  if (thermostat != TSB_INT_NOSE_HOOVER && thermostat != TSB_INT_VRESCALE)
    return TSB_ERR_INVALID_ARG;
  if (potential < TSB_POT_LJ || potential > TSB_POT_SOFT) return TSB_ERR_INVALID_ARG;
  if (n_species < 1 || !table || (n_species > 1 && !species)) return TSB_ERR_INVALID_ARG;
  if (n_species > kFusedMaxSpecies) return TSB_ERR_UNSUPPORTED;
  if (n_atoms < 1 || n_systems < 1 || !(cutoff > 0.0) || !(skin >= 0.0) || n_steps < 0)
    return TSB_ERR_INVALID_ARG;
  if (!positions || !momenta || !forces || !masses || !cell_row || !system_idx || !dt_sys ||
      !kT_sys || !tau_sys || !energy || !status)
    return TSB_ERR_INVALID_ARG;
  if (thermostat == TSB_INT_NOSE_HOOVER) {
    if (!chain_xi || !chain_pxi || !chain_Q || !chain_ke || !chain_dt) return TSB_ERR_INVALID_ARG;
    if (chain_length < 1 || chain_length > kMaxChain || chain_steps < 1) return TSB_ERR_INVALID_ARG;
    if (sy_steps != 1 && sy_steps != 3 && sy_steps != 5 && sy_steps != 7)
      return TSB_ERR_INVALID_ARG;
  }
  Carver c(workspace, workspace_bytes);
  int64_t *lo = c.take<int64_t>(n_systems);
  int64_t *hi = c.take<int64_t>(n_systems);
  int32_t *queue = c.take<int32_t>(4);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(hi, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(queue, 0, sizeof(int32_t) * 4, st);
  cudaMemsetAsync(status, 0, sizeof(int32_t) * 4, st);
  k_bounds_fused<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, n_systems, lo,
                                                       hi, status);
  FusedArgs A{thermostat, potential, n_species, table, species, positions, momenta, forces,
              masses, cell_row, lo, hi, n_systems, order, cutoff, skin, n_steps, dt_sys,
              kT_sys, nullptr, seed, counter, counter_dev, energy, n_rebuilds, queue,
              status, chain_xi, chain_pxi, chain_Q, chain_ke, tau_sys, chain_dt,
              chain_length, chain_steps, sy_steps};
  A.stress = stress;
  launch_all(A, -1, queue, st);
  if (counter_dev) k_advance_counter<<<1, 32, 0, st>>>(counter_dev, n_steps);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_fused_md_ex(int integrator, int potential, const double *table,
                               int n_species, const int32_t *species, double *positions,
                               double *momenta, double *forces, const double *masses,
                               const double *cell_row, const int64_t *system_idx,
                               int64_t n_atoms, int64_t n_systems, const int32_t *order,
                               double cutoff, double skin, int64_t n_steps,
                               const double *dt_sys, const double *kT_sys,
                               const double *gamma_sys, const double *tau_sys,
                               double *chain_xi, double *chain_pxi, double *chain_Q,
                               double *chain_ke, const double *chain_dt, int chain_length,
                               int chain_steps, int sy_steps, uint64_t seed, uint64_t counter,
                               uint64_t *counter_dev, float *frame_x, double *frame_e,
                               int64_t report_every, int64_t n_frames, int lanes_max,
                               int64_t n_wide, double prune_skin, double *energy,
                               double *stress, int32_t *n_rebuilds, int32_t *status,
                               void *workspace, size_t workspace_bytes, void *stream) {
  if (integrator < TSB_INT_NVE || integrator > TSB_INT_VRESCALE) return TSB_ERR_INVALID_ARG;
  if (potential < TSB_POT_LJ || potential > TSB_POT_SOFT) return TSB_ERR_INVALID_ARG;
  if (n_species < 1 || !table || (n_species > 1 && !species)) return TSB_ERR_INVALID_ARG;
  if (n_species > kFusedMaxSpecies) return TSB_ERR_UNSUPPORTED;
  if (n_atoms < 1 || n_systems < 1 || !(cutoff > 0.0) || !(skin >= 0.0) || n_steps < 0)
    return TSB_ERR_INVALID_ARG;
  if (!positions || !momenta || !forces || !masses || !cell_row || !system_idx || !dt_sys ||
      !energy || !status)
    return TSB_ERR_INVALID_ARG;
  if (integrator == TSB_INT_LANGEVIN && (!kT_sys || !gamma_sys)) return TSB_ERR_INVALID_ARG;
  if (integrator >= TSB_INT_NOSE_HOOVER && (!kT_sys || !tau_sys)) return TSB_ERR_INVALID_ARG;
  if (integrator == TSB_INT_NOSE_HOOVER) {
    if (!chain_xi || !chain_pxi || !chain_Q || !chain_ke || !chain_dt) return TSB_ERR_INVALID_ARG;
    if (chain_length < 1 || chain_length > kMaxChain || chain_steps < 1) return TSB_ERR_INVALID_ARG;
    if (sy_steps != 1 && sy_steps != 3 && sy_steps != 5 && sy_steps != 7)
      return TSB_ERR_INVALID_ARG;
  }
  if (report_every < 0 || n_frames < 0) return TSB_ERR_INVALID_ARG;
  if (lanes_max < 0 || lanes_max > 32 || (lanes_max & (lanes_max - 1))) return TSB_ERR_INVALID_ARG;
  if (n_wide >= 0 && !order) return TSB_ERR_INVALID_ARG;
  if (!(prune_skin >= 0.0) || !std::isfinite(prune_skin)) return TSB_ERR_INVALID_ARG;
  if (report_every > 0 && n_frames > 0 && (!frame_x || !frame_e)) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  int64_t *lo = c.take<int64_t>(n_systems);
  int64_t *hi = c.take<int64_t>(n_systems);
  int32_t *queue = c.take<int32_t>(4);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(hi, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(queue, 0, sizeof(int32_t) * 4, st);
  cudaMemsetAsync(status, 0, sizeof(int32_t) * 4, st);
  k_bounds_fused<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, n_systems, lo,
                                                       hi, status);
  FusedArgs A{integrator, potential, n_species, table, species, positions, momenta, forces,
              masses, cell_row, lo, hi, n_systems, order, cutoff, skin, n_steps, dt_sys,
              kT_sys, gamma_sys, seed, counter, counter_dev, energy, n_rebuilds, queue,
              status, chain_xi, chain_pxi, chain_Q, chain_ke, tau_sys, chain_dt,
              chain_length, chain_steps, sy_steps, frame_x, frame_e,
              report_every > 0 && n_frames > 0 ? report_every : 0, n_frames, n_atoms};
  A.stress = stress;
  A.lanes_max = lanes_max;
  A.prune = prune_skin;
  launch_all(A, n_wide, queue, st);
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

// The address is looked up again on every call made outside stream capture (a
// cudaDeviceReset or a reloaded module may have moved the array); during a
// capture the address cached by the last uncaptured call on this device is used.
static int fused_static_scratch(void **out, cudaStream_t st) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TSB_ERR_CUDA;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
    (void)cudaGetLastError();  // e.g. the legacy stream queried while another captures
    cs = cudaStreamCaptureStatusActive;
  }
  std::lock_guard<std::mutex> lock(g_fused_static_mu);
  if (cs == cudaStreamCaptureStatusNone) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_fused_static_scratch) != cudaSuccess || !p)
      return TSB_ERR_CUDA;
    g_fused_static_ptr[dev] = p;
  }
  if (!g_fused_static_ptr[dev]) return TSB_ERR_CUDA;  // first call made inside a capture
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
  cudaStream_t st = (cudaStream_t)stream;
  void *scratch = nullptr;
  TSB_TRY(fused_static_scratch(&scratch, st));
  char *base = (char *)scratch;
  int64_t *lo = (int64_t *)base;
  int64_t *hi = lo + kStaticMaxSystems;
  int32_t *queue = (int32_t *)(hi + kStaticMaxSystems);
  // the array keeps the previous call's contents: clear what must start at zero
  cudaMemsetAsync(lo, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(hi, 0, sizeof(int64_t) * n_systems, st);
  cudaMemsetAsync(queue, 0, sizeof(int32_t) * 4, st);
  cudaMemsetAsync(status, 0, sizeof(int32_t) * 4, st);
  k_bounds_fused<<<grid_for(n_atoms), kBlock, 0, st>>>(system_idx, n_atoms, n_systems, lo,
                                                       hi, status);
  FusedArgs A{integrator, potential, n_species, table, species, positions, momenta, forces,
              masses, cell_row, lo, hi, n_systems, order, cutoff, skin, n_steps, dt_sys,
              kT_sys, gamma_sys, seed, counter, nullptr, energy, n_rebuilds, queue, status};
  launch_all(A, -1, queue, st);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}
