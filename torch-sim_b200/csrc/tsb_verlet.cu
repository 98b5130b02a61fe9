// Verlet-list force path for large periodic systems (one or a few systems of
// up to millions of atoms): the list (cutoff + skin) is built once with the
// cell-list search and reused until an atom moved more than skin/2.
//
// The reference rebuilds its neighbour list inside every model call
// (torch_sim/models/pair_potential.py:168-174); pairs and forces are the same
// as PairPotentialModel.forward (pair_potential.py:351-464) because every pair
// within the cutoff is in the list and the cutoff is applied at evaluation.
//
// Layout: ELL table list[k * N + i] (uint32: j << 5 | image code), code =
// (sx+1)*9 + (sy+1)*3 + (sz+1) for lattice shifts in {-1,0,1}^3 relative to the
// positions wrapped at build time (requires every periodic cell width >= cutoff +
// skin; the build kernel flags wider shifts).  At evaluation the current
// positions are mapped with the build-time integer wraps into FP64 "build-frame"
// coordinates, so displacements across the periodic boundary are exact.
#include "tsb_pair.cuh"
#include "tsb_search.cuh"

namespace tsb {

constexpr int kVerletBlock = 256;  // threads per block of the force kernel

struct VerletWork {
  BinData b;
  double4 *wpos;  // [N] current positions in the build frame (FP64), .w = species bits
  uint8_t *pbc;   // [3] all periodic
  double *cell0;  // [9] cell of the last build (a changed cell expires the list)
  int64_t *sys;   // [N] single system
  double *part;   // [7 * blocks] per-block energy / virial sums of the force kernel
};

static void carve_verlet(Carver &c, VerletWork &w, int64_t n) {
  carve_bins(c, w.b, n, 1);
  w.wpos = c.take<double4>(n);
  w.pbc = c.take<uint8_t>(16);
  w.cell0 = c.take<double>(9);
  w.sys = c.take<int64_t>(n);
  w.part = c.take<double>(7 * ((n + kVerletBlock - 1) / kVerletBlock));
}

// build: thread per atom (bin order), ELL write, overflow flag
__global__ void k_verlet_build(BinData b, int64_t n, double rcs2, uint32_t *list,
                               int32_t *cnt, int max_nb, int32_t *status, int32_t *wrap_out) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double4 w = b.spos[p];
  const int i = tag_atom(w.w);
  const SysGeom &G = b.geom[0];
  int c = 0;
  search_neighbors(G, b.spos, b.bin_start, i, w.x, w.y, w.z, rcs2, false,
                   [&](int j, int sx, int sy, int sz, double, double, double, double) {
                     if (sx < -1 || sx > 1 || sy < -1 || sy > 1 || sz < -1 || sz > 1) {
                       atomicMax(status, 1 << 30);  // cell narrower than rc + skin
                       return;
                     }
                     if (c < max_nb)
                       list[(size_t)c * n + i] =
                           ((uint32_t)j << 5) | (uint32_t)((sx + 1) * 9 + (sy + 1) * 3 + (sz + 1));
                     ++c;
                   });
  cnt[i] = c < max_nb ? c : max_nb;
  if (c > max_nb) atomicMax(status, c);
  wrap_out[3 * i] = b.wrap[3 * i];
  wrap_out[3 * i + 1] = b.wrap[3 * i + 1];
  wrap_out[3 * i + 2] = b.wrap[3 * i + 2];
}

// current positions -> build frame (FP64) and the displacement since the build
template <class P>
__global__ void k_verlet_frame(const P *pos, const double *ref, const int32_t *wrap,
                               const double *cell, const int32_t *species, int64_t n,
                               double half_skin2, const double *cell0, double4 *wpos,
                               int32_t *expired) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x0 = (double)pos[3 * i], x1 = (double)pos[3 * i + 1], x2 = (double)pos[3 * i + 2];
  const int W0 = wrap[3 * i], W1 = wrap[3 * i + 1], W2 = wrap[3 * i + 2];
  double4 w;
  w.x = x0 - (W0 * cell[0] + W1 * cell[3] + W2 * cell[6]);
  w.y = x1 - (W0 * cell[1] + W1 * cell[4] + W2 * cell[7]);
  w.z = x2 - (W0 * cell[2] + W1 * cell[5] + W2 * cell[8]);
  w.w = __longlong_as_double((long long)(species ? species[i] : 0));
  wpos[i] = w;
  const double d0 = x0 - ref[3 * i], d1 = x1 - ref[3 * i + 1], d2 = x2 - ref[3 * i + 2];
  if (d0 * d0 + d1 * d1 + d2 * d2 > half_skin2) atomicOr(expired, 1);
  // the list's images belong to the build cell: any change of the cell expires it
  if (i == 0)
    for (int k = 0; k < 9; ++k)
      if (cell[k] != cell0[k]) atomicOr(expired, 1);
}

template <int POT, class P>
__global__ void __launch_bounds__(256, 3)
    k_verlet_forces(const double4 *__restrict__ wpos, const uint32_t *__restrict__ list,
                    const int32_t *__restrict__ cnt, int64_t n, const double *__restrict__ cell,
                    const double *__restrict__ table, int ns_species, double cutoff,
                    int flags, P *forces, double *e_atom, double *vir_atom, double *part) {
  __shared__ PairPrm<float> prm[kMaxSpecies * kMaxSpecies];
  __shared__ double prc2[kMaxSpecies * kMaxSpecies];
  __shared__ double sv[27 * 3];
  for (int k = threadIdx.x; k < ns_species * ns_species; k += blockDim.x) {
    prm[k] = make_prm<float>(POT, table + 5 * k, cutoff);
    prm_fast_extra(POT, table + 5 * k, prm[k]);
    prc2[k] = pair_rc2(POT, table + 5 * k, cutoff);
  }
  for (int k = threadIdx.x; k < 27; k += blockDim.x) {
    const int sx = k / 9 - 1, sy = (k / 3) % 3 - 1, sz = k % 3 - 1;
    for (int m = 0; m < 3; ++m) sv[3 * k + m] = sx * cell[m] + sy * cell[3 + m] + sz * cell[6 + m];
  }
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double ei = 0.0, vxx = 0, vyy = 0, vzz = 0, vyz = 0, vxz = 0, vxy = 0;
  const bool want_vir = flags & TSB_OUT_STRESS;
  if (i < n) {
    const double4 wi = wpos[i];
    const int si = (int)__double_as_longlong(wi.w);
    const PairPrm<float> *row = prm + si * ns_species;
    const int c = cnt[i];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    // one pair (entry E, neighbour position WJ): FP64 displacement, cutoff test,
    // force and virial accumulation; FP32 pair function of r^2, evaluated for
    // every entry and masked beyond the cutoff (no divergent branch)
#define TSB_VPAIR(E, WJ)                                                                     \
  {                                                                                          \
    const int code = (int)((E) & 31u);                                                       \
    const double dx = (WJ).x - wi.x + sv[3 * code];                                          \
    const double dy = (WJ).y - wi.y + sv[3 * code + 1];                                      \
    const double dz = (WJ).z - wi.z + sv[3 * code + 2];                                      \
    const int sj = (int)__double_as_longlong((WJ).w);                                        \
    const double d2 = dx * dx + dy * dy + dz * dz;                                           \
    {                                                                                        \
      const bool in_ = d2 < prc2[si * ns_species + sj];                                      \
      float ep, fr;                                                                          \
      pair_eval_fast<POT>(row[sj], (float)d2, ep, fr);                                       \
      fr = in_ ? fr : 0.f;                                                                   \
      ep = in_ ? ep : 0.f;                                                                   \
      const double gr = (double)fr;                                                          \
      const double gx = gr * dx, gy = gr * dy, gz = gr * dz;                                 \
      fx -= gx;                                                                              \
      fy -= gy;                                                                              \
      fz -= gz;                                                                              \
      ei += (double)ep;                                                                      \
      if (want_vir) {                                                                        \
        vxx += dx * gx;                                                                      \
        vyy += dy * gy;                                                                      \
        vzz += dz * gz;                                                                      \
        vyz += dy * gz;                                                                      \
        vxz += dx * gz;                                                                      \
        vxy += dx * gy;                                                                      \
      }                                                                                      \
    }                                                                                        \
  }
    // four entries per iteration; the next four list words are loaded one
    // iteration ahead so their DRAM latency overlaps the current gathers and math
    int k = 0;
    const uint32_t *lp = list + i;
    uint32_t e0 = 0, e1 = 0, e2 = 0, e3 = 0;
    if (c >= 4) {
      e0 = lp[0];
      e1 = lp[(size_t)n];
      e2 = lp[(size_t)2 * n];
      e3 = lp[(size_t)3 * n];
    }
    for (; k + 4 <= c; k += 4) {
      uint32_t f0 = 0, f1 = 0, f2 = 0, f3 = 0;
      if (k + 8 <= c) {
        const uint32_t *q = lp + (size_t)(k + 4) * n;
        f0 = q[0];
        f1 = q[(size_t)n];
        f2 = q[(size_t)2 * n];
        f3 = q[(size_t)3 * n];
      }
      const double4 w0 = wpos[e0 >> 5], w1 = wpos[e1 >> 5];
      const double4 w2 = wpos[e2 >> 5], w3 = wpos[e3 >> 5];
      TSB_VPAIR(e0, w0)
      TSB_VPAIR(e1, w1)
      TSB_VPAIR(e2, w2)
      TSB_VPAIR(e3, w3)
      e0 = f0;
      e1 = f1;
      e2 = f2;
      e3 = f3;
    }
    for (; k < c; ++k) {
      const uint32_t e = lp[(size_t)k * n];
      const double4 wj = wpos[e >> 5];
      TSB_VPAIR(e, wj)
    }
#undef TSB_VPAIR
    forces[3 * i] = (P)fx;
    forces[3 * i + 1] = (P)fy;
    forces[3 * i + 2] = (P)fz;
    e_atom[i] = 0.5 * ei;
    if (want_vir) {
      double *v = vir_atom + 6 * i;
      v[0] = 0.5 * vxx;
      v[1] = 0.5 * vyy;
      v[2] = 0.5 * vzz;
      v[3] = 0.5 * vyz;
      v[4] = 0.5 * vxz;
      v[5] = 0.5 * vxy;
    }
  }
  // per-block sums of the half pair energies / virials in a fixed order (FP64):
  // shuffles inside each warp, then the warps in order; the last kernel adds blocks
  __shared__ double sh[7][kVerletBlock / 32];
  double acc[7] = {0.5 * ei, 0.5 * vxx, 0.5 * vyy, 0.5 * vzz, 0.5 * vyz, 0.5 * vxz, 0.5 * vxy};
  for (int k = 0; k < 7; ++k) {
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = acc[k];
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    double t = 0.0;
    for (int w = 0; w < kVerletBlock / 32; ++w) t += sh[threadIdx.x][w];
    part[7 * blockIdx.x + threadIdx.x] = t;
  }
}

// sum of the force kernel's block partials in a fixed order (FP64)
template <class P>
__global__ void k_verlet_final(const double *part, int64_t n_blocks, int flags,
                               const double *cell, P *energy, P *stress) {
  __shared__ double sh[7][32];
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int64_t b = threadIdx.x; b < n_blocks; b += blockDim.x)
    for (int k = 0; k < 7; ++k) acc[k] += part[7 * b + k];
  for (int k = 0; k < 7; ++k) {
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = acc[k];
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double t[7];
  for (int k = 0; k < 7; ++k) {
    t[k] = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t[k] += sh[k][w];
  }
  energy[0] = (P)t[0];
  if (flags & TSB_OUT_STRESS) {
    const double *a = cell;
    const double vol = fabs(a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                            a[2] * (a[3] * a[7] - a[4] * a[6]));
    const double c = -1.0 / vol;
    stress[0] = (P)(c * t[1]); stress[1] = (P)(c * t[6]); stress[2] = (P)(c * t[5]);
    stress[3] = (P)(c * t[6]); stress[4] = (P)(c * t[2]); stress[5] = (P)(c * t[4]);
    stress[6] = (P)(c * t[5]); stress[7] = (P)(c * t[4]); stress[8] = (P)(c * t[3]);
  }
}

template <class P>
__global__ void k_copy_ref(const P *pos, double *ref, int64_t n, const P *cell, double *cell0) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 3 * n) ref[i] = (double)pos[i];
  if (i < 9) cell0[i] = (double)cell[i];
}

}  // namespace tsb

using namespace tsb;

extern "C" size_t tsb_verlet_workspace_size(int64_t n_atoms) {
  Carver c(nullptr, (size_t)-1);
  VerletWork w;
  carve_verlet(c, w, n_atoms);
  return c.off + 256;
}

extern "C" int tsb_verlet_build(const void *positions, const void *cell_row, int64_t n_atoms,
                                int dtype, double cutoff, double skin, uint32_t *list,
                                int32_t *counts, int max_neighbors, double *ref_positions,
                                int32_t *wraps, int32_t *status, void *workspace,
                                size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || !positions || !cell_row || !list || !counts || !ref_positions ||
      !wraps || !status || max_neighbors < 1 || !(cutoff > 0.0) || !(skin >= 0.0))
    return TSB_ERR_INVALID_ARG;
  if (n_atoms >= ((int64_t)1 << 27)) return TSB_ERR_UNSUPPORTED;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  VerletWork w;
  carve_verlet(c, w, n_atoms);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  uint8_t *pbc = w.pbc;
  int64_t *sys = w.sys;
  cudaMemsetAsync(pbc, 1, 3, st);
  cudaMemsetAsync(sys, 0, sizeof(int64_t) * n_atoms, st);
  cudaMemsetAsync(status, 0, sizeof(int32_t), st);
  const double rcs = cutoff + skin;
  if (dtype == TSB_F64) {
    TSB_TRY(prepare_bins<double>((const double *)positions, (const double *)cell_row, pbc, sys,
                                 n_atoms, 1, rcs, w.b, st));
    k_copy_ref<double><<<grid_for(3 * n_atoms), kBlock, 0, st>>>((const double *)positions,
                                                                 ref_positions, n_atoms,
                                                                 (const double *)cell_row,
                                                                 w.cell0);
  } else {
    TSB_TRY(prepare_bins<float>((const float *)positions, (const float *)cell_row, pbc, sys,
                                n_atoms, 1, rcs, w.b, st));
    k_copy_ref<float><<<grid_for(3 * n_atoms), kBlock, 0, st>>>((const float *)positions,
                                                                ref_positions, n_atoms,
                                                                (const float *)cell_row,
                                                                w.cell0);
  }
  k_verlet_build<<<grid_for(n_atoms, 128), 128, 0, st>>>(w.b, n_atoms, rcs * rcs, list, counts,
                                                         max_neighbors, status, wraps);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_verlet_check(const void *positions, const double *ref_positions,
                                const int32_t *wraps, const double *cell_row,
                                const int32_t *species, int64_t n_atoms, int dtype,
                                double skin, int32_t *expired, void *workspace,
                                size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || !positions || !ref_positions || !wraps || !cell_row || !expired)
    return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  VerletWork w;
  carve_verlet(c, w, n_atoms);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(expired, 0, sizeof(int32_t), st);
  const double hs2 = 0.25 * skin * skin;
  if (dtype == TSB_F64)
    k_verlet_frame<double><<<grid_for(n_atoms), kBlock, 0, st>>>(
        (const double *)positions, ref_positions, wraps, cell_row, species, n_atoms, hs2,
        w.cell0, w.wpos, expired);
  else if (dtype == TSB_F32)
    k_verlet_frame<float><<<grid_for(n_atoms), kBlock, 0, st>>>(
        (const float *)positions, ref_positions, wraps, cell_row, species, n_atoms, hs2,
        w.cell0, w.wpos, expired);
  else
    return TSB_ERR_INVALID_ARG;
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_verlet_forces(int potential, const double *table, int n_species,
                                 const uint32_t *list, const int32_t *counts, int64_t n_atoms,
                                 const double *cell_row, int dtype, double cutoff,
                                 int out_flags, void *energy, void *forces, void *stress,
                                 double *e_atom, double *vir_atom, void *workspace,
                                 size_t workspace_bytes, void *stream) {
  if (potential < TSB_POT_LJ || potential > TSB_POT_SOFT || n_species < 1 ||
      n_species > kMaxSpecies || !table || n_atoms < 1 || !list || !counts || !cell_row ||
      !energy || !forces || !e_atom)
    return TSB_ERR_INVALID_ARG;
  if ((out_flags & TSB_OUT_STRESS) && (!stress || !vir_atom)) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  VerletWork w;
  carve_verlet(c, w, n_atoms);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
#define TSB_VF(POT, P)                                                                      \
  k_verlet_forces<POT, P><<<grid_for(n_atoms, kVerletBlock), kVerletBlock, 0, st>>>(      \
      w.wpos, list, counts, n_atoms, cell_row, table, n_species, cutoff, out_flags,       \
      (P *)forces, e_atom, vir_atom, w.part);                                              \
  k_verlet_final<P><<<1, 256, 0, st>>>(w.part, grid_for(n_atoms, kVerletBlock), out_flags, \
                                       cell_row, (P *)energy, (P *)stress);
  if (dtype == TSB_F64) {
    if (potential == TSB_POT_LJ) { TSB_VF(TSB_POT_LJ, double) }
    else if (potential == TSB_POT_MORSE) { TSB_VF(TSB_POT_MORSE, double) }
    else { TSB_VF(TSB_POT_SOFT, double) }
  } else if (dtype == TSB_F32) {
    if (potential == TSB_POT_LJ) { TSB_VF(TSB_POT_LJ, float) }
    else if (potential == TSB_POT_MORSE) { TSB_VF(TSB_POT_MORSE, float) }
    else { TSB_VF(TSB_POT_SOFT, float) }
  } else {
    return TSB_ERR_INVALID_ARG;
  }
#undef TSB_VF
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}
