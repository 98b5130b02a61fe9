// Fused neighbour search + pair energy/force/virial (drop-in for
// PairPotentialModel.forward, torch_sim/models/pair_potential.py:351-464).
//
// One thread per atom i (launched in bin order so neighbouring threads share
// candidate bins in L1/L2) walks the full neighbour set of i, so forces need no
// atomics and the summation order is fixed (deterministic results).  Each
// unordered pair is evaluated from both ends; per-atom energies/virials take
// half of each visit, matching the half-list weights of pair_potential.py:402-441.
// Displacements are formed in FP64 from the wrapped FP64 positions; the pair
// function runs in R (float by default, double with TSB_MATH_FP64).
#include "tsb_pair.cuh"
#include "tsb_search.cuh"
#include "tsb_sysreduce.cuh"

namespace tsb {

// LANES > 1: LANES lanes per atom (small batches; lanes split the candidates and the
// partial sums are reduced in a fixed order), LANES = 1: one thread per atom.
template <int POT, class R, class P, int LANES>
__global__ void __launch_bounds__(128)
    k_pair_forces(BinData b, int64_t n, const double *__restrict__ table, int ns_species,
                  const int32_t *__restrict__ species, double cutoff, int flags, P *forces,
                  P *energies, P *stresses, double *e_half, double *vir_half,
                  const uint8_t *__restrict__ sys_active) {
  __shared__ PairPrm<R> prm[kMaxSpecies * kMaxSpecies];
  __shared__ double prc2[kMaxSpecies * kMaxSpecies];
  for (int k = threadIdx.x; k < ns_species * ns_species; k += blockDim.x) {
    prm[k] = make_prm<R>(POT, table + 5 * k, cutoff);
    prc2[k] = pair_rc2(POT, table + 5 * k, cutoff);
  }
  __syncthreads();
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t p = t / LANES;
  if (p >= n) return;
  const double4 w = b.spos[p];
  const int i = tag_atom(w.w);
  const int s = b.sys_of[i];
  if (sys_active && !sys_active[s]) return;
  const SysGeom &G = b.geom[s];
  const int si = min(max(tag_species(w.w), 0), ns_species - 1);
  const PairPrm<R> *row = prm + si * ns_species;
  // forces accumulate in R; energy and virial in FP64 (per-system sums in FP64)
  R fx = 0, fy = 0, fz = 0;
  double ei = 0, vxx = 0, vyy = 0, vzz = 0, vyz = 0, vxz = 0, vxy = 0;
  auto pair = [&](int, int, int, int, double dx, double dy, double dz, double d2,
                       int sp) {
                     const int sj = min(max(sp, 0), ns_species - 1);
                     if (!(d2 < prc2[si * ns_species + sj])) return;  // FP64 decision
                     const PairPrm<R> &q = row[sj];
                     const R rx = (R)dx, ry = (R)dy, rz = (R)dz;
                     const R r2 = rx * rx + ry * ry + rz * rz;
                     R e, fr;
                     pair_eval<POT, R>(q, r2, e, fr);
                     // force-defined pairs: i's thread sees both directed pairs
                     // (i, j) and (j, i) of the reference's full list, so the force
                     // adds f_ij and f_ji and the virial takes half of it
                     // (pair_potential.py:567-600, stress scale 1/2 for a full list)
                     double vw = 1.0;
                     if constexpr (POT == TSB_POT_PLIFE) {
                       R e2, fr2;
                       pair_eval<POT, R>(prm[sj * ns_species + si], r2, e2, fr2);
                       fr += fr2;
                       vw = 0.5;
                     }
                     const R gx = fr * rx, gy = fr * ry, gz = fr * rz;  // force on j
                     fx -= gx;
                     fy -= gy;
                     fz -= gz;
                     ei += (double)e;
                     vxx += vw * (double)(rx * gx);
                     vyy += vw * (double)(ry * gy);
                     vzz += vw * (double)(rz * gz);
                     vyz += vw * (double)(ry * gz);
                     vxz += vw * (double)(rx * gz);
                     vxy += vw * (double)(rx * gy);
                   };
  if constexpr (LANES > 1) {
    group_search_neighbors<LANES>(G, b.spos, b.bin_start, i, w.x, w.y, w.z, cutoff * cutoff, false,
                          pair);
    fx = group_sum<LANES>(fx);
    fy = group_sum<LANES>(fy);
    fz = group_sum<LANES>(fz);
    ei = group_sum<LANES>(ei);
    vxx = group_sum<LANES>(vxx);
    vyy = group_sum<LANES>(vyy);
    vzz = group_sum<LANES>(vzz);
    vyz = group_sum<LANES>(vyz);
    vxz = group_sum<LANES>(vxz);
    vxy = group_sum<LANES>(vxy);
    if ((threadIdx.x & (LANES - 1)) != 0) return;
  } else {
    search_neighbors(G, b.spos, b.bin_start, i, w.x, w.y, w.z, cutoff * cutoff, false, pair);
  }
  if (flags & TSB_OUT_FORCES) {
    forces[3 * i] = (P)fx;
    forces[3 * i + 1] = (P)fy;
    forces[3 * i + 2] = (P)fz;
  }
  // reference per-atom energies: each endpoint receives the full pair energy
  // (pair_potential.py:411-417 with weight 1 on both mapping rows)
  if (flags & TSB_OUT_ENERGIES) energies[i] = (P)ei;
  if (flags & TSB_OUT_STRESSES) {
    // per-atom stress: -1/2 sum_j r_ij (x) f_ij / V (pair_potential.py:262-272)
    const double c = -0.5 / G.vol;
    P *o = stresses + 9 * i;
    o[0] = (P)(c * vxx); o[1] = (P)(c * vxy); o[2] = (P)(c * vxz);
    o[3] = (P)(c * vxy); o[4] = (P)(c * vyy); o[5] = (P)(c * vyz);
    o[6] = (P)(c * vxz); o[7] = (P)(c * vyz); o[8] = (P)(c * vzz);
  }
  e_half[i] = 0.5 * ei;
  double *v = vir_half + 6 * i;
  v[0] = 0.5 * vxx;
  v[1] = 0.5 * vyy;
  v[2] = 0.5 * vzz;
  v[3] = 0.5 * vyz;
  v[4] = 0.5 * vxz;
  v[5] = 0.5 * vxy;
}

struct PairWork {
  BinData b;
  double *e_half;
  double *vir_half;
  double *part;  // [7 * ns * chunks] slice sums (chunks > 1 only)
  int chunks;
};

static void carve_pair(Carver &c, PairWork &w, int64_t n, int64_t ns) {
  carve_bins(c, w.b, n, ns);
  w.e_half = c.take<double>(n);
  w.vir_half = c.take<double>(6 * n);
  w.chunks = reduce_chunks(n, ns);
  w.part = w.chunks > 1 ? c.take<double>(7 * ns * w.chunks) : nullptr;
}

template <int POT, class R, class P>
static void launch_forces(PairWork &w, int64_t n, const double *table, int nsp,
                          const int32_t *species, double cutoff, int flags, P *forces,
                          P *energies, P *stresses, const uint8_t *active, cudaStream_t st) {
  if (n <= kGroupSearchMaxAtoms)
    k_pair_forces<POT, R, P, kSearchGroup><<<grid_for(kSearchGroup * n, 128), 128, 0, st>>>(
        w.b, n, table, nsp, species, cutoff, flags, forces, energies, stresses, w.e_half,
        w.vir_half, active);
  else
    k_pair_forces<POT, R, P, 1><<<grid_for(n, 128), 128, 0, st>>>(
        w.b, n, table, nsp, species, cutoff, flags, forces, energies, stresses, w.e_half,
        w.vir_half, active);
}

template <class P>
static int pair_forward(int pot, const double *table, int nsp, const int32_t *species,
                        const P *pos, const P *cell, const uint8_t *pbc, const int64_t *sys,
                        int64_t n, int64_t ns, double cutoff, int flags, P *energy,
                        P *forces, P *stress, P *energies, P *stresses,
                        const uint8_t *active, int64_t max_sys, PairWork &w,
                        cudaStream_t st) {
  TSB_TRY(prepare_bins_any<P>(pos, cell, pbc, sys, n, ns, cutoff, w.b, st, species, max_sys));
  const bool f64 = flags & TSB_MATH_FP64;
  if (n > 0) {
#define TSB_LAUNCH(POT)                                                                    \
  if (f64)                                                                                 \
    launch_forces<POT, double, P>(w, n, table, nsp, species, cutoff, flags, forces,       \
                                  energies, stresses, active, st);                         \
  else                                                                                     \
    launch_forces<POT, float, P>(w, n, table, nsp, species, cutoff, flags, forces,        \
                                 energies, stresses, active, st);
    if (pot == TSB_POT_LJ) {
      TSB_LAUNCH(TSB_POT_LJ)
    } else if (pot == TSB_POT_MORSE) {
      TSB_LAUNCH(TSB_POT_MORSE)
    } else if (pot == TSB_POT_SOFT) {
      TSB_LAUNCH(TSB_POT_SOFT)
    } else {
      TSB_LAUNCH(TSB_POT_PLIFE)
    }
#undef TSB_LAUNCH
  }
  k_sys_reduce<P><<<dim3((unsigned)ns, (unsigned)w.chunks), kBlock, 0, st>>>(
      w.b.geom, w.e_half, w.vir_half, flags, energy, stress, active, w.chunks, w.part);
  if (w.chunks > 1)
    k_sys_final<P><<<grid_for(ns), kBlock, 0, st>>>(w.b.geom, w.part, ns, w.chunks, flags,
                                                     energy, stress, active);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

}  // namespace tsb

using namespace tsb;

extern "C" size_t tsb_pair_workspace_size(int64_t n_atoms, int64_t n_systems) {
  Carver c(nullptr, (size_t)-1);
  PairWork w;
  carve_pair(c, w, n_atoms, n_systems);
  return c.off + 256;
}

extern "C" int tsb_pair_forward(int potential, const double *table, int n_species,
                                const int32_t *species, const void *positions,
                                const void *cell_row, const uint8_t *pbc,
                                const int64_t *system_idx, int64_t n_atoms,
                                int64_t n_systems, int dtype, double cutoff, int out_flags,
                                void *energy, void *forces, void *stress, void *energies,
                                void *stresses, const uint8_t *sys_active,
                                int64_t max_system_atoms, void *workspace,
                                size_t workspace_bytes, void *stream) {
  if (potential < TSB_POT_LJ || potential > TSB_POT_PLIFE) return TSB_ERR_INVALID_ARG;
  if (n_species < 1 || n_species > kMaxSpecies || !table) return TSB_ERR_INVALID_ARG;
  if (n_species > 1 && !species) return TSB_ERR_INVALID_ARG;
  if (n_atoms < 0 || n_systems < 1 || !(cutoff > 0.0) || !cell_row || !pbc || !energy)
    return TSB_ERR_INVALID_ARG;
  if (n_atoms > 0 && (!positions || !system_idx)) return TSB_ERR_INVALID_ARG;
  if ((out_flags & TSB_OUT_FORCES) && !forces) return TSB_ERR_INVALID_ARG;
  if ((out_flags & TSB_OUT_STRESS) && !stress) return TSB_ERR_INVALID_ARG;
  if ((out_flags & TSB_OUT_ENERGIES) && !energies) return TSB_ERR_INVALID_ARG;
  if ((out_flags & TSB_OUT_STRESSES) && !stresses) return TSB_ERR_INVALID_ARG;
  if (dtype != TSB_F32 && dtype != TSB_F64) return TSB_ERR_INVALID_ARG;
  if (n_atoms >= (int64_t)1 << 30) return TSB_ERR_UNSUPPORTED;
  Carver c(workspace, workspace_bytes);
  PairWork w;
  carve_pair(c, w, n_atoms, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == TSB_F64)
    return pair_forward<double>(potential, table, n_species, species,
                                (const double *)positions, (const double *)cell_row, pbc,
                                system_idx, n_atoms, n_systems, cutoff, out_flags,
                                (double *)energy, (double *)forces, (double *)stress,
                                (double *)energies, (double *)stresses, sys_active,
                                max_system_atoms, w, st);
  return pair_forward<float>(potential, table, n_species, species, (const float *)positions,
                             (const float *)cell_row, pbc, system_idx, n_atoms, n_systems,
                             cutoff, out_flags, (float *)energy, (float *)forces,
                             (float *)stress, (float *)energies, (float *)stresses, sys_active,
                             max_system_atoms, w, st);
}
