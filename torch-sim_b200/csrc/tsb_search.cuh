// Cell-list neighbour search over the binned, wrapped positions.
#pragma once

#include <type_traits>

#include "tsb_common.cuh"

namespace tsb {

__device__ inline void frame_coords(const SysGeom &G, double x, double y, double z,
                                    double *u) {
  u[0] = G.T[0] * x + G.T[1] * y + G.T[2] * z;
  u[1] = G.T[3] * x + G.T[4] * y + G.T[5] * z;
  u[2] = G.T[6] * x + G.T[7] * y + G.T[8] * z;
}

__device__ inline int floordiv_dev(int a, int b) {
  int q = a / b;
  return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q;
}

// Visit every image (j, S) with |w_j + S @ cell - w_i|^2 < rc2 (FP64), where w
// are the wrapped positions.  The unshifted self image is skipped unless
// `self_pairs`.  Callback: f(j, Sx, Sy, Sz, dx, dy, dz, d2) with d = w_j + S@cell - w_i,
// or f(..., d2, species_j) when it takes the species tag as a ninth argument.
template <class F>
__device__ inline void search_neighbors(const SysGeom &G, const double4 *__restrict__ spos,
                                        const int64_t *__restrict__ bin_start, int i,
                                        double wx, double wy, double wz, double rc2,
                                        bool self_pairs, F &&f) {
  double u[3];
  frame_coords(G, wx, wy, wz, u);
  int lo[3], hi[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double a = floor((u[k] - G.h[k] - G.org[k]) * G.scale[k]);
    double b = floor((u[k] + G.h[k] - G.org[k]) * G.scale[k]);
    if (!G.per[k]) {
      a = fmax(a, 0.0);
      b = fmin(b, (double)(G.nb[k] - 1));
    }
    lo[k] = (int)a;
    hi[k] = (int)b;
  }
  for (int cx = lo[0]; cx <= hi[0]; ++cx) {
    int ix = G.per[0] ? floordiv_dev(cx, G.nb[0]) : 0;
    int bx = cx - ix * G.nb[0];
    for (int cy = lo[1]; cy <= hi[1]; ++cy) {
      int iy = G.per[1] ? floordiv_dev(cy, G.nb[1]) : 0;
      int by = cy - iy * G.nb[1];
      for (int cz = lo[2]; cz <= hi[2]; ++cz) {
        int iz = G.per[2] ? floordiv_dev(cz, G.nb[2]) : 0;
        int bz = cz - iz * G.nb[2];
        const double sx = ix * G.cell[0] + iy * G.cell[3] + iz * G.cell[6];
        const double sy = ix * G.cell[1] + iy * G.cell[4] + iz * G.cell[7];
        const double sz = ix * G.cell[2] + iy * G.cell[5] + iz * G.cell[8];
        const bool zero_shift = (ix | iy | iz) == 0;
        const int bin = G.bin_base + (bx * G.nb[1] + by) * G.nb[2] + bz;
        const int64_t p1 = bin_start[bin + 1];
        for (int64_t p = bin_start[bin]; p < p1; ++p) {
          const double4 q = spos[p];
          const double dx = (q.x + sx) - wx;
          const double dy = (q.y + sy) - wy;
          const double dz = (q.z + sz) - wz;
          const double d2 = dx * dx + dy * dy + dz * dz;
          if (d2 < rc2) {
            const int j = tag_atom(q.w);
            if (j == i && zero_shift && !self_pairs) continue;
            if constexpr (std::is_invocable_v<F, int, int, int, int, double, double, double,
                                              double, int>)
              f(j, ix, iy, iz, dx, dy, dz, d2, tag_species(q.w));
            else
              f(j, ix, iy, iz, dx, dy, dz, d2);
          }
        }
      }
    }
  }
}

// Group-cooperative search_neighbors for batches too small to fill the GPU with
// one thread per atom: the G lanes of a group (G = 2..32, aligned within the
// warp) share the central atom i and walk its window row by row; the bins of one
// row and image are adjacent in bin order, so each span of candidates is
// contiguous and the lanes test G of them per step.  f(j, Sx, Sy, Sz, dx, dy, dz,
// d2, species_j) runs on every lane whose candidate lies inside rc2; each lane
// accumulates its own partial sums, which the caller reduces with group_sum<G>.
template <int G, class F>
__device__ inline void group_search_neighbors(const SysGeom &G_, const double4 *__restrict__ spos,
                                              const int64_t *__restrict__ bin_start, int i,
                                              double wx, double wy, double wz, double rc2,
                                              bool self_pairs, F &&f) {
  const SysGeom &Gm = G_;
  const int lane = threadIdx.x & (G - 1);
  double u[3];
  frame_coords(Gm, wx, wy, wz, u);
  int lo[3], hi[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double a = floor((u[k] - Gm.h[k] - Gm.org[k]) * Gm.scale[k]);
    double b = floor((u[k] + Gm.h[k] - Gm.org[k]) * Gm.scale[k]);
    if (!Gm.per[k]) {
      a = fmax(a, 0.0);
      b = fmin(b, (double)(Gm.nb[k] - 1));
    }
    lo[k] = (int)a;
    hi[k] = (int)b;
  }
  const int nb1 = Gm.nb[1], nb2 = Gm.nb[2];
  for (int cx = lo[0]; cx <= hi[0]; ++cx) {
    const int ix = Gm.per[0] ? floordiv_dev(cx, Gm.nb[0]) : 0;
    const int bx = cx - ix * Gm.nb[0];
    for (int cy = lo[1]; cy <= hi[1]; ++cy) {
      const int iy = Gm.per[1] ? floordiv_dev(cy, nb1) : 0;
      const int by = cy - iy * nb1;
      const int row = Gm.bin_base + (bx * nb1 + by) * nb2;
      for (int cz = lo[2]; cz <= hi[2];) {
        const int iz = Gm.per[2] ? floordiv_dev(cz, nb2) : 0;
        const int bz = cz - iz * nb2;
        const int bz_end = min(nb2 - 1, bz + (hi[2] - cz));  // last bin of this image
        cz += bz_end - bz + 1;
        const double sx = ix * Gm.cell[0] + iy * Gm.cell[3] + iz * Gm.cell[6];
        const double sy = ix * Gm.cell[1] + iy * Gm.cell[4] + iz * Gm.cell[7];
        const double sz = ix * Gm.cell[2] + iy * Gm.cell[5] + iz * Gm.cell[8];
        const bool zero_shift = (ix | iy | iz) == 0;
        const int64_t q1 = bin_start[row + bz_end + 1];
        for (int64_t q = bin_start[row + bz] + lane; q < q1; q += G) {
          const double4 o = spos[q];
          const double dx = (o.x + sx) - wx;
          const double dy = (o.y + sy) - wy;
          const double dz = (o.z + sz) - wz;
          const double d2 = dx * dx + dy * dy + dz * dz;
          if (d2 < rc2) {
            const int j = tag_atom(o.w);
            if (j == i && zero_shift && !self_pairs) continue;
            f(j, ix, iy, iz, dx, dy, dz, d2, tag_species(o.w));
          }
        }
      }
    }
  }
}

// sum over the G lanes of a group in a fixed butterfly order (every lane of the
// group gets the total); the whole warp must call it
template <int G, class T>
__device__ inline T group_sum(T x) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// batches of at most this many atoms take the group-per-atom kernels, with
// kSearchGroup lanes per atom
constexpr int64_t kGroupSearchMaxAtoms = 65536;
#ifndef TSB_SEARCH_GROUP
#define TSB_SEARCH_GROUP 4
#endif
constexpr int kSearchGroup = TSB_SEARCH_GROUP;

}  // namespace tsb
