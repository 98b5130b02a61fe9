// Neighbour-list construction (drop-in for torch_nl_linked_cell,
// torch_sim/neighbors/torch_nl.py:156-215).  Two passes over a cell-list
// search: count per atom -> exclusive scan -> fill, so the output is grouped by
// the central atom i in ascending order and deterministic.
#include "tsb_search.cuh"

namespace tsb {

// full_to_half_list rule (pair_potential.py:86-127): keep i < j; for i == j keep
// the copy whose first non-zero shift component is positive.
__device__ inline bool keep_half(int i, int j, int sx, int sy, int sz) {
  if (i != j) return i < j;
  int first = sx != 0 ? sx : (sy != 0 ? sy : sz);
  return first > 0;
}

__global__ void k_nl_count(BinData b, int64_t n, double rc2, int flags, int32_t *cnt) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double4 w = b.spos[p];
  const int i = tag_atom(w.w);
  const SysGeom &G = b.geom[b.sys_of[i]];
  const bool self = flags & TSB_NL_SELF_INTERACTION;
  const bool half = flags & TSB_NL_HALF;
  const int *W = b.wrap;
  int c = 0;
  search_neighbors(G, b.spos, b.bin_start, i, w.x, w.y, w.z, rc2, self,
                   [&](int j, int sx, int sy, int sz, double, double, double, double) {
                     if (half) {
                       int fx = sx + W[3 * i] - W[3 * j];
                       int fy = sy + W[3 * i + 1] - W[3 * j + 1];
                       int fz = sz + W[3 * i + 2] - W[3 * j + 2];
                       if (!keep_half(i, j, fx, fy, fz)) return;
                     }
                     ++c;
                   });
  cnt[i] = c;
}

template <class P>
__global__ void k_nl_fill(BinData b, int64_t n, double rc2, int flags, const int64_t *off,
                          int64_t cap, int64_t *mapping, int64_t stride,
                          int64_t *system_mapping, P *shifts) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double4 w = b.spos[p];
  const int i = tag_atom(w.w);
  int64_t o = off[i];
  if (o >= cap) return;
  const int s = b.sys_of[i];
  const SysGeom &G = b.geom[s];
  const bool self = flags & TSB_NL_SELF_INTERACTION;
  const bool half = flags & TSB_NL_HALF;
  const int *W = b.wrap;
  search_neighbors(G, b.spos, b.bin_start, i, w.x, w.y, w.z, rc2, self,
                   [&](int j, int sx, int sy, int sz, double, double, double, double) {
                     // shift valid for the unwrapped positions (torch_nl.py:214)
                     int fx = sx + W[3 * i] - W[3 * j];
                     int fy = sy + W[3 * i + 1] - W[3 * j + 1];
                     int fz = sz + W[3 * i + 2] - W[3 * j + 2];
                     if (half && !keep_half(i, j, fx, fy, fz)) return;
                     if (o < cap) {
                       mapping[o] = i;
                       mapping[stride + o] = j;
                       system_mapping[o] = s;
                       shifts[3 * o] = (P)fx;
                       shifts[3 * o + 1] = (P)fy;
                       shifts[3 * o + 2] = (P)fz;
                     }
                     ++o;
                   });
}

struct NlWork {
  BinData b;
  int32_t *cnt;
  int64_t *off;
};

static void carve_nl(Carver &c, NlWork &w, int64_t n, int64_t ns) {
  carve_bins(c, w.b, n, ns);
  w.cnt = c.take<int32_t>(n);
  w.off = c.take<int64_t>(n + 1);
}

template <class P>
static int nl_build(const P *pos, const P *cell, const uint8_t *pbc, const int64_t *sys,
                    int64_t n, int64_t ns, double cutoff, int flags, int64_t *mapping,
                    int64_t stride, int64_t *sysmap, P *shifts, int64_t cap,
                    int64_t *n_pairs, NlWork &w, cudaStream_t st) {
  TSB_TRY(prepare_bins<P>(pos, cell, pbc, sys, n, ns, cutoff, w.b, st));
  const double rc2 = cutoff * cutoff;
  k_nl_count<<<grid_for(n, 128), 128, 0, st>>>(w.b, n, rc2, flags, w.cnt);
  TSB_TRY(exclusive_scan(w.cnt, w.off, n, w.b.scan_tmp, st));
  cudaMemcpyAsync(n_pairs, w.off + n, sizeof(int64_t), cudaMemcpyDeviceToDevice, st);
  if (cap > 0)
    k_nl_fill<P><<<grid_for(n, 128), 128, 0, st>>>(w.b, n, rc2, flags, w.off, cap, mapping,
                                                   stride, sysmap, shifts);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

}  // namespace tsb

using namespace tsb;

extern "C" size_t tsb_nl_workspace_size(int64_t n_atoms, int64_t n_systems) {
  Carver c(nullptr, (size_t)-1);
  NlWork w;
  carve_nl(c, w, n_atoms, n_systems);
  return c.off + 256;
}

extern "C" int tsb_nl_build(const void *positions, const void *cell_row, const uint8_t *pbc,
                            const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                            int dtype, double cutoff, int flags, int64_t *mapping,
                            int64_t mapping_stride, int64_t *system_mapping, void *shifts,
                            int64_t capacity, int64_t *n_pairs, void *workspace,
                            size_t workspace_bytes, void *stream) {
  if (n_atoms < 0 || n_systems < 1 || !(cutoff > 0.0) || !n_pairs || !cell_row || !pbc)
    return TSB_ERR_INVALID_ARG;
  if (n_atoms > 0 && (!positions || !system_idx)) return TSB_ERR_INVALID_ARG;
  if (capacity > 0 && (!mapping || !system_mapping || !shifts || mapping_stride < capacity))
    return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  if (n_atoms >= (int64_t)1 << 30) return TSB_ERR_UNSUPPORTED;
  Carver c(workspace, workspace_bytes);
  NlWork w;
  carve_nl(c, w, n_atoms, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (n_atoms == 0) {
    cudaMemsetAsync(n_pairs, 0, sizeof(int64_t), st);
    TSB_CHECK_LAUNCH();
    return TSB_OK;
  }
  if (dtype == TSB_F64)
    return nl_build<double>((const double *)positions, (const double *)cell_row, pbc,
                            system_idx, n_atoms, n_systems, cutoff, flags, mapping,
                            mapping_stride, system_mapping, (double *)shifts, capacity,
                            n_pairs, w, st);
  return nl_build<float>((const float *)positions, (const float *)cell_row, pbc, system_idx,
                         n_atoms, n_systems, cutoff, flags, mapping, mapping_stride,
                         system_mapping, (float *)shifts, capacity, n_pairs, w, st);
}
