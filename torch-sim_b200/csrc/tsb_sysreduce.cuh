// Per-system energy / virial sums shared by the pair-force paths.
#pragma once

#include "tsb_common.cuh"

namespace tsb {

// Per-system energy / virial sums in FP64, in a fixed order (deterministic).
// Block (s, c) sums slice c of `chunks` equal slices of system s's atoms; with
// one slice it writes the outputs, otherwise k_sys_final adds the slices in
// order (so one large system is summed by many blocks, many small ones by one
// block each).
template <class P>
__device__ inline void write_sys(const SysGeom &G, const double *t, int flags, int64_t s,
                                 P *energy, P *stress) {
  energy[s] = (P)t[0];
  if (flags & TSB_OUT_STRESS) {
    const double c = -1.0 / G.vol;  // stress = -1/V sum r (x) f (pair_potential.py:226-232)
    P *o = stress + 9 * s;
    o[0] = (P)(c * t[1]); o[1] = (P)(c * t[6]); o[2] = (P)(c * t[5]);
    o[3] = (P)(c * t[6]); o[4] = (P)(c * t[2]); o[5] = (P)(c * t[4]);
    o[6] = (P)(c * t[5]); o[7] = (P)(c * t[4]); o[8] = (P)(c * t[3]);
  }
}

template <class P>
__global__ void k_sys_reduce(const SysGeom *g, const double *e_half, const double *vir_half,
                             int flags, P *energy, P *stress, const uint8_t *sys_active,
                             int chunks, double *part) {
  __shared__ double sh[7][kBlock / 32];
  const int s = blockIdx.x, ch = blockIdx.y;
  if (sys_active && !sys_active[s]) return;
  const SysGeom &G = g[s];
  const int64_t step = (G.count + chunks - 1) / chunks;
  const int64_t lo = (int64_t)ch * step;
  const int64_t hi = lo + step < G.count ? lo + step : G.count;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int64_t a = lo + threadIdx.x; a < hi; a += blockDim.x) {
    int64_t i = G.start + a;
    acc[0] += e_half[i];
    for (int k = 0; k < 6; ++k) acc[1 + k] += vir_half[6 * i + k];
  }
  for (int k = 0; k < 7; ++k) {
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = acc[k];
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double t[7];
  for (int k = 0; k < 7; ++k) {
    t[k] = 0;
    for (int w = 0; w < kBlock / 32; ++w) t[k] += sh[k][w];
  }
  if (chunks == 1) {
    write_sys(G, t, flags, s, energy, stress);
  } else {
    for (int k = 0; k < 7; ++k) part[7 * ((int64_t)s * chunks + ch) + k] = t[k];
  }
}

template <class P>
__global__ void k_sys_final(const SysGeom *g, const double *part, int64_t ns, int chunks,
                            int flags, P *energy, P *stress, const uint8_t *sys_active) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns || (sys_active && !sys_active[s])) return;
  double t[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int c = 0; c < chunks; ++c)
    for (int k = 0; k < 7; ++k) t[k] += part[7 * (s * chunks + c) + k];
  write_sys(g[s], t, flags, s, energy, stress);
}

// slices per system for the sums above: about 8192 atoms per slice for the mean
// system size, at most 128
inline int reduce_chunks(int64_t n, int64_t ns) {
  const int64_t per = ns > 0 ? (n + ns - 1) / ns : 0;
  int64_t c = (per + 8191) / 8192;
  if (c < 1) c = 1;
  if (c > 128) c = 128;
  return (int)c;
}

}  // namespace tsb
