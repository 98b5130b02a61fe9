// Scan, per-system geometry and cell binning (counting sort) shared by the
// neighbour-list and fused pair kernels.
//
// Binning frame (one per system):
//   * periodic systems with an invertible cell: fractional coordinates
//     u = inv(cell_row^T) r, wrapped to [0,1) on periodic axes exactly as
//     torch_sim/transforms.py:160-210 does (integer wrap W = floor(u));
//   * otherwise Cartesian coordinates over the system's bounding box.
// A sphere of radius rc spans u_k +- rc*|row k of T| (the reciprocal-vector
// norm of transforms.py:435-467), so the search visits every "unbounded" bin
// index c_k in [floor((u_k-h_k)*scale_k), floor((u_k+h_k)*scale_k)], mapping
// c_k -> (bin c_k mod nb_k, image floor(c_k / nb_k)) on periodic axes.  That
// covers all images the reference replicates (get_cell_shift_idx,
// transforms.py:470-497) for any cell, including cells smaller than rc.
#include "tsb_common.cuh"

namespace tsb {

// ---------------------------------------------------------------- scan
__device__ inline int64_t warp_incl_scan(int64_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int64_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.
__device__ inline int64_t block_excl_scan(int64_t v, int64_t *total) {
  __shared__ int64_t warp_sums[kBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t inc = warp_incl_scan(v);
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int64_t w = lane < kBlock / 32 ? warp_sums[lane] : 0;
    int64_t wi = warp_incl_scan(w);
    if (lane < kBlock / 32) warp_sums[lane] = wi - w;
    if (lane == kBlock / 32 - 1) *total = wi;
  }
  __syncthreads();
  int64_t r = inc - v + warp_sums[warp];
  __syncthreads();
  return r;
}

__global__ void k_scan_tiles(const int32_t *in, int64_t *out, int64_t n, int64_t *sums,
                             int64_t *total) {
  __shared__ int64_t tot;
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t v[kScanItems];
  int64_t local = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < n) ? (int64_t)in[base + k] : 0;
    local += v[k];
  }
  int64_t pre = block_excl_scan(local, &tot);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = pre;
    pre += v[k];
  }
  if (threadIdx.x == 0) {
    sums[blockIdx.x] = tot;
    if (total) *total = tot;  // single tile: the scan is complete
  }
}

__global__ void k_scan_sums(int64_t *sums, int64_t nb, int64_t *out_total) {
  __shared__ int64_t tot;
  int64_t carry = 0;
  for (int64_t b0 = 0; b0 < nb; b0 += kBlock) {
    int64_t i = b0 + threadIdx.x;
    int64_t v = i < nb ? sums[i] : 0;
    int64_t pre = block_excl_scan(v, &tot);
    if (i < nb) sums[i] = pre + carry;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *out_total = carry;
}

__global__ void k_scan_add(int64_t *out, int64_t n, const int64_t *sums) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += sums[i / kScanTile];
}

size_t scan_tmp_elems(int64_t n) { return (size_t)((n + kScanTile - 1) / kScanTile + 1); }

int exclusive_scan(const int32_t *in, int64_t *out, int64_t n, int64_t *tmp,
                   cudaStream_t st) {
  int64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles < 1) tiles = 1;
  if (tiles == 1) {
    k_scan_tiles<<<1, kBlock, 0, st>>>(in, out, n, tmp, out + n);
  } else {
    k_scan_tiles<<<(unsigned)tiles, kBlock, 0, st>>>(in, out, n, tmp, nullptr);
    k_scan_sums<<<1, kBlock, 0, st>>>(tmp, tiles, out + n);
    k_scan_add<<<grid_for(n), kBlock, 0, st>>>(out, n, tmp);
  }
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

// ---------------------------------------------------------------- geometry
__global__ void k_sys_bounds(const int64_t *sys, int64_t n, int64_t *lo, int64_t *hi,
                             int32_t *sys_of) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t s = sys[i];
  sys_of[i] = (int32_t)s;
  if (i == 0 || sys[i - 1] != s) lo[s] = i;
  if (i == n - 1 || sys[i + 1] != s) hi[s] = i + 1;
}

__device__ inline double det3(const double *a) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
         a[2] * (a[3] * a[7] - a[4] * a[6]);
}

// inverse of a row-major 3x3 matrix
__device__ inline void inv3(const double *a, double *r) {
  double d = det3(a);
  double id = 1.0 / d;
  r[0] = (a[4] * a[8] - a[5] * a[7]) * id;
  r[1] = (a[2] * a[7] - a[1] * a[8]) * id;
  r[2] = (a[1] * a[5] - a[2] * a[4]) * id;
  r[3] = (a[5] * a[6] - a[3] * a[8]) * id;
  r[4] = (a[0] * a[8] - a[2] * a[6]) * id;
  r[5] = (a[2] * a[3] - a[0] * a[5]) * id;
  r[6] = (a[3] * a[7] - a[4] * a[6]) * id;
  r[7] = (a[1] * a[6] - a[0] * a[7]) * id;
  r[8] = (a[0] * a[4] - a[1] * a[3]) * id;
}

template <class P>
__device__ SysGeom geom_setup_one(const P *cell_row, const uint8_t *pbc, int64_t s,
                                  double cutoff, const int64_t *lo, const int64_t *hi) {
  SysGeom G;
  for (int k = 0; k < 9; ++k) G.cell[k] = (double)cell_row[s * 9 + k];
  double d = det3(G.cell);
  bool anyp = pbc[s * 3] || pbc[s * 3 + 1] || pbc[s * 3 + 2];
  bool inv_ok = isfinite(d) && fabs(d) > 1e-12;
  G.active = anyp && inv_ok;
  G.vol = fabs(d);
  if (G.active) {
    // T = inv(cell_row^T) = inv(cell_row)^T
    double ic[9];
    inv3(G.cell, ic);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) G.T[r * 3 + c] = ic[c * 3 + r];
  } else {
    for (int k = 0; k < 9; ++k) G.T[k] = (k % 4 == 0) ? 1.0 : 0.0;
  }
  for (int k = 0; k < 3; ++k) {
    double nrm = sqrt(G.T[3 * k] * G.T[3 * k] + G.T[3 * k + 1] * G.T[3 * k + 1] +
                      G.T[3 * k + 2] * G.T[3 * k + 2]);
    // small relative margin so rounding in u never drops a bin at the edge
    G.h[k] = cutoff * nrm * (1.0 + 1e-9) + 1e-12;
    G.per[k] = G.active && pbc[s * 3 + k];
    G.org[k] = 0.0;
    G.scale[k] = 1.0;
    G.nb[k] = 1;
  }
  G.start = lo[s];
  G.count = (int32_t)(hi[s] - lo[s]);
  G.bin_base = 0;
  G.nbins = 1;
  return G;
}

template <class P>
__global__ void k_geom_setup(const P *cell_row, const uint8_t *pbc, int64_t ns,
                             double cutoff, const int64_t *lo, const int64_t *hi,
                             SysGeom *g) {
  int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  g[s] = geom_setup_one<P>(cell_row, pbc, s, cutoff, lo, hi);
}

__device__ inline void frame_u(const SysGeom &G, double x, double y, double z, double *u) {
  u[0] = G.T[0] * x + G.T[1] * y + G.T[2] * z;
  u[1] = G.T[3] * x + G.T[4] * y + G.T[5] * z;
  u[2] = G.T[6] * x + G.T[7] * y + G.T[8] * z;
}

// Extents of non-periodic axes, then the bin grid of one system; called by
// every thread of a block, thread 0 writes the grid into G.
template <class P>
__device__ void geom_bins_block(const P *pos, SysGeom &G) {
  __shared__ double smin[3][kBlock / 32], smax[3][kBlock / 32];
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  bool need = !(G.per[0] && G.per[1] && G.per[2]);
  if (need) {
    for (int a = threadIdx.x; a < G.count; a += blockDim.x) {
      int64_t i = G.start + a;
      double u[3];
      frame_u(G, (double)pos[3 * i], (double)pos[3 * i + 1], (double)pos[3 * i + 2], u);
      for (int k = 0; k < 3; ++k) {
        mn[k] = fmin(mn[k], u[k]);
        mx[k] = fmax(mx[k], u[k]);
      }
    }
    for (int k = 0; k < 3; ++k) {
      for (int o = 16; o > 0; o >>= 1) {
        mn[k] = fmin(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
        mx[k] = fmax(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
      }
      if ((threadIdx.x & 31) == 0) {
        smin[k][threadIdx.x >> 5] = mn[k];
        smax[k][threadIdx.x >> 5] = mx[k];
      }
    }
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double len[3];
  double nbd[3];
  for (int k = 0; k < 3; ++k) {
    if (G.per[k]) {
      G.org[k] = 0.0;
      len[k] = 1.0;
    } else {
      double a = INFINITY, b = -INFINITY;
      for (int w = 0; w < kBlock / 32; ++w) {
        a = fmin(a, smin[k][w]);
        b = fmax(b, smax[k][w]);
      }
      if (!(a <= b)) { a = 0.0; b = 0.0; }
      G.org[k] = a;
      len[k] = fmax(b - a, 1e-9);
    }
    // bins at least half the search half-width wide: the search window spans at
    // most 5 bins per axis and tests ~3.7x the sphere's volume instead of the
    // ~6.4x (27 bins of one cutoff) that cutoff-wide bins give
    double q = floor(2.0 * len[k] / G.h[k]);
    nbd[k] = fmin(fmax(q, 1.0), 1048576.0);
  }
  double cap = fmax(1.0, 2.0 * (double)G.count);
  while (nbd[0] * nbd[1] * nbd[2] > cap) {
    int k = (nbd[0] >= nbd[1] && nbd[0] >= nbd[2]) ? 0 : (nbd[1] >= nbd[2] ? 1 : 2);
    nbd[k] = ceil(nbd[k] * 0.5);
  }
  for (int k = 0; k < 3; ++k) {
    G.nb[k] = (int32_t)nbd[k];
    G.scale[k] = nbd[k] / len[k];
  }
  G.nbins = G.nb[0] * G.nb[1] * G.nb[2];
}


// One block per system: extents of non-periodic axes, then the bin grid.
template <class P>
__global__ void k_geom_bins(const P *pos, SysGeom *g, int32_t *sys_nbins) {
  const int s = blockIdx.x;
  geom_bins_block<P>(pos, g[s]);
  if (threadIdx.x == 0) sys_nbins[s] = g[s].nbins;
}

__global__ void k_set_binbase(SysGeom *g, const int64_t *off, int64_t ns) {
  int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < ns) g[s].bin_base = (int32_t)off[s];
}

// bin of one atom: integer wrap W on periodic axes, wrapped position w, bin
// coordinates c (clamped into the grid)
__device__ inline void bin_atom(const SysGeom &G, const double *r, int *W, int *c, double *w) {
  double u[3];
  frame_u(G, r[0], r[1], r[2], u);
  for (int k = 0; k < 3; ++k) {
    double uk = u[k];
    W[k] = 0;
    if (G.per[k]) {
      double f = floor(uk);
      f = isfinite(f) ? fmin(fmax(f, -1e9), 1e9) : 0.0;
      W[k] = (int)f;
      uk -= f;
    }
    double cc = floor((uk - G.org[k]) * G.scale[k]);
    cc = isfinite(cc) ? cc : 0.0;
    cc = fmin(fmax(cc, 0.0), (double)(G.nb[k] - 1));
    c[k] = (int)cc;
  }
  // wrapped position w = r - W @ cell
  for (int m = 0; m < 3; ++m)
    w[m] = r[m] - (W[0] * G.cell[m] + W[1] * G.cell[3 + m] + W[2] * G.cell[6 + m]);
}

template <class P>
__global__ void k_bin_assign(const P *pos, const SysGeom *g, const int32_t *sys_of,
                             int64_t n, int32_t *wrap, int32_t *bin_of,
                             int32_t *bin_count, double4 *wpos) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SysGeom &G = g[sys_of[i]];
  double r[3] = {(double)pos[3 * i], (double)pos[3 * i + 1], (double)pos[3 * i + 2]};
  int W[3], c[3];
  double w[3];
  bin_atom(G, r, W, c, w);
  int b = G.bin_base + (c[0] * G.nb[1] + c[1]) * G.nb[2] + c[2];
  wrap[3 * i] = W[0];
  wrap[3 * i + 1] = W[1];
  wrap[3 * i + 2] = W[2];
  bin_of[i] = b;
  wpos[i] = make_double4(w[0], w[1], w[2], 0.0);
  atomicAdd(&bin_count[b], 1);
}

__global__ void k_bin_scatter(const int32_t *bin_of, const int64_t *bin_start,
                              int32_t *bin_fill, int64_t n, int32_t *sidx) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = bin_of[i];
  int64_t slot = bin_start[b] + atomicAdd(&bin_fill[b], 1);
  sidx[slot] = (int32_t)i;
}

// Deterministic order inside each bin (ascending atom index), then gather the
// wrapped positions into bin order.
__global__ void k_bin_sort(const int64_t *bin_start, int64_t nbins_total, int32_t *sidx,
                           const double4 *wpos, const int32_t *species, double4 *spos) {
  int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbins_total) return;
  int64_t s0 = bin_start[b], s1 = bin_start[b + 1];
  for (int64_t p = s0 + 1; p < s1; ++p) {
    int32_t v = sidx[p];
    int64_t q = p - 1;
    while (q >= s0 && sidx[q] > v) {
      sidx[q + 1] = sidx[q];
      --q;
    }
    sidx[q + 1] = v;
  }
  for (int64_t p = s0; p < s1; ++p) {
    int32_t j = sidx[p];
    double4 w = wpos[j];
    const unsigned long long hi = species ? (unsigned long long)(uint32_t)species[j] : 0ull;
    w.w = __longlong_as_double((long long)((hi << 32) | (uint32_t)j));
    spos[p] = w;
  }
}

// Per-system binning for batches of small systems: one block per selected
// system does the geometry, the bin assignment, the counting sort and the
// gather into bin order, so one launch replaces the batch-wide passes and
// systems not selected keep their bins untouched.  Bin regions are static
// (system s owns bins [2 lo_s + s, 2 (lo_s + count_s) + s], room for the
// 2 count_s + 1 bins and the sentinel its grid may use), so no scan over the
// batch is needed.  Order inside a bin is ascending atom index, as k_bin_sort
// gives: atoms are placed a block-sized chunk at a time, one warp after
// another, each lane taking its slot after the lower lanes with the same bin.
// Systems of at most kSysBinMaxAtoms atoms keep the histogram and the atoms'
// bins in shared memory; a larger one uses its regions of bin_count / bin_of
// (correct, but one block does all of its work).
template <class P>
__global__ void __launch_bounds__(kBlock)
    k_bins_sys(const P *pos, const P *cell_row, const uint8_t *pbc, double cutoff,
               const int32_t *only, const int32_t *species, BinData b) {
  __shared__ int32_t cur_s[2 * kSysBinMaxAtoms + 2];
  __shared__ int16_t lbin_s[kSysBinMaxAtoms];
  __shared__ int64_t chunk_tot;
  const int64_t s = blockIdx.x;
  if (only && !only[s]) return;
  SysGeom &G = b.geom[s];
  if (threadIdx.x == 0) G = geom_setup_one<P>(cell_row, pbc, s, cutoff, b.sys_lo, b.sys_hi);
  __syncthreads();
  const int count = G.count;
  if (count == 0) return;
  geom_bins_block<P>(pos, G);
  __syncthreads();
  const int64_t start = G.start;
  const int nbins = G.nbins;  // <= 2 count
  const int64_t base = 2 * start + s;
  const bool small = count <= kSysBinMaxAtoms;
  int32_t *cur = small ? cur_s : b.bin_count + base;
  int32_t *lbin_g = b.bin_of + start;
  if (threadIdx.x == 0) G.bin_base = (int32_t)base;
  for (int k = threadIdx.x; k <= nbins; k += blockDim.x) cur[k] = 0;
  __syncthreads();
  for (int a = threadIdx.x; a < count; a += blockDim.x) {
    const int64_t i = start + a;
    const double r[3] = {(double)pos[3 * i], (double)pos[3 * i + 1], (double)pos[3 * i + 2]};
    int W[3], c[3];
    double w[3];
    bin_atom(G, r, W, c, w);
    const int lb = (c[0] * G.nb[1] + c[1]) * G.nb[2] + c[2];
    b.wrap[3 * i] = W[0];
    b.wrap[3 * i + 1] = W[1];
    b.wrap[3 * i + 2] = W[2];
    b.wpos[i] = make_double4(w[0], w[1], w[2], 0.0);
    if (small)
      lbin_s[a] = (int16_t)lb;
    else
      lbin_g[a] = lb;
    atomicAdd(&cur[lb], 1);
  }
  __syncthreads();
  // exclusive scan of cur[0..nbins] (cur[nbins] = 0 becomes the total), each
  // thread a contiguous run of entries
  const int per = (nbins + 1 + blockDim.x - 1) / blockDim.x;
  const int k0 = min((int)threadIdx.x * per, nbins + 1), k1 = min(k0 + per, nbins + 1);
  int64_t run = 0;
  for (int k = k0; k < k1; ++k) run += cur[k];
  int64_t pre = block_excl_scan(run, &chunk_tot);
  for (int k = k0; k < k1; ++k) {
    const int v = cur[k];
    cur[k] = (int32_t)pre;
    b.bin_start[base + k] = start + pre;
    pre += v;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  for (int c0 = 0; c0 < count; c0 += blockDim.x) {
    const int a = c0 + threadIdx.x;
    const int lb = a < count ? (small ? (int)lbin_s[a] : lbin_g[a]) : -1;
    // the atom's tagged position is loaded before the warp-by-warp slot
    // assignment, so the serialised part touches shared memory only
    const int64_t i = start + a;
    double4 wv4 = make_double4(0.0, 0.0, 0.0, 0.0);
    if (lb >= 0) {
      wv4 = b.wpos[i];
      const unsigned long long hi = species ? (unsigned long long)(uint32_t)species[i] : 0ull;
      wv4.w = __longlong_as_double((long long)((hi << 32) | (uint32_t)i));
    }
    int at = 0, rank = 0;
    for (int wv = 0; wv < (int)(blockDim.x >> 5); ++wv) {
      if (warp == wv) {
        const unsigned peers = __match_any_sync(0xffffffffu, lb);
        rank = __popc(peers & lt);
        at = lb >= 0 ? cur[lb] : 0;
        __syncwarp();
        if (lb >= 0 && rank == 0) cur[lb] = at + __popc(peers);
      }
      __syncthreads();
    }
    if (lb >= 0) {
      const int64_t slot = start + at + rank;
      b.spos[slot] = wv4;
      b.sidx[slot] = (int32_t)i;
    }
  }
}

template <class P>
int prepare_bins_sys(const P *positions, const P *cell_row, const uint8_t *pbc,
                     const int64_t *system_idx, int64_t n, int64_t ns, double cutoff,
                     BinData &b, cudaStream_t st, const int32_t *species, const int32_t *only) {
  cudaMemsetAsync(b.sys_lo, 0, sizeof(int64_t) * ns, st);
  cudaMemsetAsync(b.sys_hi, 0, sizeof(int64_t) * ns, st);
  if (n > 0) k_sys_bounds<<<grid_for(n), kBlock, 0, st>>>(system_idx, n, b.sys_lo, b.sys_hi,
                                                         b.sys_of);
  k_bins_sys<P><<<(unsigned)ns, kBlock, 0, st>>>(positions, cell_row, pbc, cutoff, only, species,
                                                 b);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

template <class P>
int prepare_bins_any(const P *positions, const P *cell_row, const uint8_t *pbc,
                     const int64_t *system_idx, int64_t n, int64_t ns, double cutoff,
                     BinData &b, cudaStream_t st, const int32_t *species,
                     int64_t max_system_atoms) {
  if (max_system_atoms > 0 && max_system_atoms <= kSysBinMaxAtoms)
    return prepare_bins_sys<P>(positions, cell_row, pbc, system_idx, n, ns, cutoff, b, st,
                               species, nullptr);
  return prepare_bins<P>(positions, cell_row, pbc, system_idx, n, ns, cutoff, b, st, species);
}

#define TSB_BINS_INST(P)                                                                       \
  template int prepare_bins_sys<P>(const P *, const P *, const uint8_t *, const int64_t *,     \
                                   int64_t, int64_t, double, BinData &, cudaStream_t,          \
                                   const int32_t *, const int32_t *);                          \
  template int prepare_bins_any<P>(const P *, const P *, const uint8_t *, const int64_t *,     \
                                   int64_t, int64_t, double, BinData &, cudaStream_t,          \
                                   const int32_t *, int64_t);
TSB_BINS_INST(float)
TSB_BINS_INST(double)
#undef TSB_BINS_INST

int64_t bin_capacity(int64_t n_atoms, int64_t n_systems) {
  return 2 * n_atoms + n_systems + 1;
}

void carve_bins(Carver &c, BinData &b, int64_t n, int64_t ns) {
  b.bcap = bin_capacity(n, ns);
  b.geom = c.take<SysGeom>(ns);
  b.sys_of = c.take<int32_t>(n);
  b.bin_of = c.take<int32_t>(n);
  b.wrap = c.take<int32_t>(3 * n);
  b.spos = c.take<double4>(n);
  b.wpos = c.take<double4>(n);
  b.sidx = c.take<int32_t>(n);
  b.bin_count = c.take<int32_t>(b.bcap);
  b.bin_start = c.take<int64_t>(b.bcap + 1);
  b.bin_fill = c.take<int32_t>(b.bcap);
  b.sys_nbins = c.take<int32_t>(ns);
  b.sys_binoff = c.take<int64_t>(ns + 1);
  b.sys_lo = c.take<int64_t>(ns);
  b.sys_hi = c.take<int64_t>(ns);
  int64_t m = b.bcap > n ? b.bcap : n;
  b.scan_tmp = c.take<int64_t>((int64_t)scan_tmp_elems(m > ns ? m : ns));
}

template <class P>
int prepare_bins(const P *positions, const P *cell_row, const uint8_t *pbc,
                 const int64_t *system_idx, int64_t n, int64_t ns, double cutoff,
                 BinData &b, cudaStream_t st, const int32_t *species) {
  cudaMemsetAsync(b.sys_lo, 0, sizeof(int64_t) * ns, st);
  cudaMemsetAsync(b.sys_hi, 0, sizeof(int64_t) * ns, st);
  cudaMemsetAsync(b.bin_count, 0, sizeof(int32_t) * b.bcap, st);
  cudaMemsetAsync(b.bin_fill, 0, sizeof(int32_t) * b.bcap, st);
  if (n > 0) k_sys_bounds<<<grid_for(n), kBlock, 0, st>>>(system_idx, n, b.sys_lo, b.sys_hi,
                                                         b.sys_of);
  k_geom_setup<P><<<grid_for(ns), kBlock, 0, st>>>(cell_row, pbc, ns, cutoff, b.sys_lo,
                                                   b.sys_hi, b.geom);
  k_geom_bins<P><<<(unsigned)ns, kBlock, 0, st>>>(positions, b.geom, b.sys_nbins);
  TSB_TRY(exclusive_scan(b.sys_nbins, b.sys_binoff, ns, b.scan_tmp, st));
  k_set_binbase<<<grid_for(ns), kBlock, 0, st>>>(b.geom, b.sys_binoff, ns);
  if (n > 0) {
    k_bin_assign<P><<<grid_for(n), kBlock, 0, st>>>(positions, b.geom, b.sys_of, n, b.wrap,
                                                    b.bin_of, b.bin_count, b.wpos);
    TSB_TRY(exclusive_scan(b.bin_count, b.bin_start, b.bcap, b.scan_tmp, st));
    k_bin_scatter<<<grid_for(n), kBlock, 0, st>>>(b.bin_of, b.bin_start, b.bin_fill, n,
                                                  b.sidx);
    k_bin_sort<<<grid_for(b.bcap), kBlock, 0, st>>>(b.bin_start, b.bcap, b.sidx, b.wpos,
                                                    species, b.spos);
  }
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

template int prepare_bins<float>(const float *, const float *, const uint8_t *,
                                 const int64_t *, int64_t, int64_t, double, BinData &,
                                 cudaStream_t, const int32_t *);
template int prepare_bins<double>(const double *, const double *, const uint8_t *,
                                  const int64_t *, int64_t, int64_t, double, BinData &,
                                  cudaStream_t, const int32_t *);

}  // namespace tsb
