// Common device/host helpers for the tsb CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/tsb.h"

#define TSB_CHECK_LAUNCH()                              \
  do {                                                  \
    cudaError_t e_ = cudaGetLastError();                \
    if (e_ != cudaSuccess) return TSB_ERR_CUDA;         \
  } while (0)

#define TSB_TRY(x)                 \
  do {                             \
    int s_ = (x);                  \
    if (s_ != TSB_OK) return s_;   \
  } while (0)

namespace tsb {

constexpr int kBlock = 256;

inline unsigned grid_for(int64_t n, int block = kBlock) {
  int64_t g = (n + block - 1) / block;
  return (unsigned)(g < 1 ? 1 : g);
}

// Bump allocator over the caller's workspace; every carve is 256-byte aligned.
struct Carver {
  char *base;
  size_t off = 0;
  size_t cap;
  bool ok = true;
  Carver(void *b, size_t c) : base((char *)b), cap(c) {}
  template <class T>
  T *take(int64_t n) {
    off = (off + 255) & ~(size_t)255;
    T *p = base ? (T *)(base + off) : nullptr;
    off += (size_t)(n > 0 ? n : 1) * sizeof(T);
    if (off > cap) ok = false;
    return p;
  }
};

// Per-system geometry of the binning frame.
//   u = T r  (T = inv(cell_row^T) -> fractional coordinates, or T = I -> Cartesian)
//   bin coordinate c_k = floor((u_k - org_k) * scale_k), scale_k = nb_k / len_k
//   search half-width in u-space: h_k = cutoff * |row k of T|
struct SysGeom {
  double cell[9];   // row-vector cell, cell[3*k + m] = component m of lattice vector k
  double T[9];      // frame matrix (row-major)
  double org[3];    // frame origin per axis (0 on periodic axes)
  double scale[3];  // nb_k / len_k
  double h[3];      // search half-width (u units)
  double vol;       // |det cell|
  int64_t start;    // first atom
  int32_t count;    // atoms in system
  int32_t nb[3];    // bins per axis
  int32_t per[3];   // periodic axis (wrap + images) flags
  int32_t active;   // fractional frame (pbc.any and invertible cell)
  int32_t bin_base; // first global bin
  int32_t nbins;
};

// A bin-ordered position's .w carries the atom index in its low 32 bits and
// the atom's species (0 when the caller gave none) in its high 32 bits.
__device__ inline int tag_atom(double w) {
  return (int)(uint32_t)(unsigned long long)__double_as_longlong(w);
}
__device__ inline int tag_species(double w) { return (int)(__double_as_longlong(w) >> 32); }

struct Vec3 {
  double x, y, z;
};

__host__ __device__ inline int floordiv_i(int a, int b) {
  int q = a / b;
  return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q;
}

// ---------------------------------------------------------------------------
// Exclusive scan of int32 counts into int64 offsets (out has n+1 entries,
// out[n] = total).  Three phases: per-block scan, scan of block sums, add.
// ---------------------------------------------------------------------------
constexpr int kScanItems = 4;
constexpr int kScanTile = kBlock * kScanItems;

size_t scan_tmp_elems(int64_t n);
int exclusive_scan(const int32_t *in, int64_t *out, int64_t n, int64_t *tmp,
                   cudaStream_t st);

// ---------------------------------------------------------------------------
// Shared preparation for the neighbour search (neighbour list and fused pair
// kernels): system offsets, geometry, binning by counting sort.
// ---------------------------------------------------------------------------
struct BinData {
  SysGeom *geom;        // [S]
  int32_t *sys_of;      // [N] system of atom
  int32_t *bin_of;      // [N] global bin of atom
  int32_t *wrap;        // [N*3] integer wrap shift W_i (r_i = w_i + W_i @ cell)
  double4 *spos;        // [N] wrapped position in bin order; .w = atom index bits
  double4 *wpos;        // [N] wrapped position in atom order (scratch)
  int32_t *sidx;        // [N] atom index in bin order
  int32_t *bin_count;   // [Bcap]
  int64_t *bin_start;   // [Bcap+1]
  int32_t *bin_fill;    // [Bcap]
  int32_t *sys_nbins;   // [S]
  int64_t *sys_binoff;  // [S+1]
  int64_t *sys_lo;      // [S] first atom of system
  int64_t *sys_hi;      // [S] one past last atom
  int64_t *scan_tmp;
  int64_t bcap;
};

int64_t bin_capacity(int64_t n_atoms, int64_t n_systems);
void carve_bins(Carver &c, BinData &b, int64_t n_atoms, int64_t n_systems);

// dtype-generic preparation.  `search_cutoff` sets the bin size; `species`
// (optional) is tagged into the bin-ordered positions.
template <class P>
int prepare_bins(const P *positions, const P *cell_row, const uint8_t *pbc,
                 const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                 double search_cutoff, BinData &b, cudaStream_t st,
                 const int32_t *species = nullptr);

// Systems up to this size are binned with shared-memory tables by the
// per-system binning.
constexpr int kSysBinMaxAtoms = 4096;

// Per-system binning of the systems with only[s] != 0 (all when only is null),
// one block each, into the same BinData layout (static bin regions: bin_base =
// 2 sys_lo + s).  Fast for systems of at most kSysBinMaxAtoms atoms; larger ones
// are binned correctly but slowly.
template <class P>
int prepare_bins_sys(const P *positions, const P *cell_row, const uint8_t *pbc,
                     const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                     double search_cutoff, BinData &b, cudaStream_t st, const int32_t *species,
                     const int32_t *only);

// prepare_bins_sys over every system when the caller's max_system_atoms (the
// largest system's atom count, 0 = unknown) is at most kSysBinMaxAtoms, else the
// batch-wide prepare_bins.
template <class P>
int prepare_bins_any(const P *positions, const P *cell_row, const uint8_t *pbc,
                     const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                     double search_cutoff, BinData &b, cudaStream_t st, const int32_t *species,
                     int64_t max_system_atoms);

}  // namespace tsb
