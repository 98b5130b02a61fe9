// Kernels for the hand-written adjoint of NVE (velocity Verlet) trajectories
// with species-matrix Lennard-Jones forces, in FP64 throughout.
//
// The reference differentiates trajectories with torch.autograd through
// PairPotentialModel (pair_potential.py:420-425, create_graph=False), which
// drops the force-Jacobian terms; here the discrete adjoint is exact:
//   lam_p += (dt/m) lam_q ;  lam_q += c * J_F(q)^T lam_p ;  g_theta += c * dF/dtheta^T lam_p
// with J_F = -Hessian(E).  For a pair (i, j) with d = r_j - r_i, r = |d|,
// u = d / r, the Hessian block is K = V'' u u^T + (V'/r)(I - u u^T) and
// (H v)_i = sum_j K (v_i - v_j); the force is F_i = sum_j V'(r) u, so
// dF_i/dtheta = sum_j (dV'/dtheta) u.
//
// Also: the Gaussian-smeared pair-distance histogram of each system and its
// gradient with respect to positions (the trajectory loss).
#include "tsb_ljhvp.cuh"
#include "tsb_search.cuh"

namespace tsb {

struct AdjWork {
  BinData b;
  double *part;  // per-atom partials (parameter gradients or histogram bins)
};

static void carve_adj(Carver &c, AdjWork &w, int64_t n, int64_t ns, int64_t per_atom) {
  carve_bins(c, w.b, n, ns);
  w.part = c.take<double>(n * per_atom);
}

// LANES > 1: LANES lanes per atom (small batches; fixed-order reduction of the lanes'
// partial sums), LANES = 1: one thread per atom.  Pair arithmetic: lj_hvp_pair.
template <int LANES>
__global__ void __launch_bounds__(128)
    k_lj_hvp(BinData b, int64_t n, const double *__restrict__ table, int nsp,
             const int32_t *__restrict__ species, double cutoff, const double *__restrict__ v,
             double coef, double *__restrict__ lam_q, double *__restrict__ gpart) {
  __shared__ LjHvpTable T;
  lj_hvp_table(T, table, nsp, cutoff);
  __syncthreads();
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t p = t / LANES;
  if (p >= n) return;
  const double4 w = b.spos[p];
  const int i = tag_atom(w.w);
  const SysGeom &G = b.geom[b.sys_of[i]];
  const int si = species ? min(max(species[i], 0), nsp - 1) : 0;
  const double vi0 = v[3 * i], vi1 = v[3 * i + 1], vi2 = v[3 * i + 2];
  double hx = 0, hy = 0, hz = 0;
  // parameter gradients of the pairs (si, t) by neighbour species t, in registers
  // (a static select keeps them out of local memory)
  double gs[kAdjMaxSpecies], ge[kAdjMaxSpecies];
#pragma unroll
  for (int t2 = 0; t2 < kAdjMaxSpecies; ++t2) gs[t2] = ge[t2] = 0.0;
  auto pair = [&](int j, int, int, int, double dx, double dy, double dz, double d2, int sp) {
    const int sj = min(max(sp, 0), nsp - 1);
    lj_hvp_pair(T, si * nsp + sj, sj, dx, dy, dz, d2, vi0, vi1, vi2, v[3 * j], v[3 * j + 1],
                v[3 * j + 2], hx, hy, hz, gs, ge);
  };
  if constexpr (LANES > 1) {
    group_search_neighbors<LANES>(G, b.spos, b.bin_start, i, w.x, w.y, w.z, cutoff * cutoff, false,
                          pair);
    hx = group_sum<LANES>(hx);
    hy = group_sum<LANES>(hy);
    hz = group_sum<LANES>(hz);
#pragma unroll
    for (int t2 = 0; t2 < kAdjMaxSpecies; ++t2) {
      gs[t2] = group_sum<LANES>(gs[t2]);
      ge[t2] = group_sum<LANES>(ge[t2]);
    }
    if ((threadIdx.x & (LANES - 1)) != 0) return;
  } else {
    search_neighbors(G, b.spos, b.bin_start, i, w.x, w.y, w.z, cutoff * cutoff, false, pair);
  }
  // J_F^T v = -H v
  lam_q[3 * i] -= coef * hx;
  lam_q[3 * i + 1] -= coef * hy;
  lam_q[3 * i + 2] -= coef * hz;
  double *g = gpart + (size_t)i * (2 * nsp * nsp);
  for (int k = 0; k < nsp * nsp; ++k) {
    g[2 * k] = 0.0;
    g[2 * k + 1] = 0.0;
  }
#pragma unroll
  for (int t2 = 0; t2 < kAdjMaxSpecies; ++t2)
    if (t2 < nsp) {
      g[2 * (si * nsp + t2)] = coef * gs[t2];
      g[2 * (si * nsp + t2) + 1] = coef * ge[t2];
    }
}

// Gaussian-smeared histogram of pair distances r < r_max (each unordered pair
// once): h_b = sum_pairs exp(-(r - c_b)^2 / (2 w^2)), c_b = (b + 1/2) r_max / B.
// A pair adds to the bins with |r - c_b| <= kRdfWindow w only: a term beyond is
// below exp(-72) ~ 5e-32 of a pair's peak term, under FP64 rounding of any bin
// the pair reaches.
constexpr double kRdfWindow = 12.0;

__device__ inline void rdf_window(double r, double bw, double width, int nb, int &k0, int &k1) {
  const double reach = kRdfWindow * width;
  k0 = max(0, (int)ceil((r - reach) / bw - 0.5));
  k1 = min(nb - 1, (int)floor((r + reach) / bw - 0.5));
}

__global__ void __launch_bounds__(128)
    k_rdf_part(BinData b, int64_t n, double r_max, int nb, double width, double *part) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double4 w = b.spos[p];
  const int i = tag_atom(w.w);
  const SysGeom &G = b.geom[b.sys_of[i]];
  double *h = part + (size_t)i * nb;
  for (int k = 0; k < nb; ++k) h[k] = 0.0;
  const double bw = r_max / nb, inv2w2 = 1.0 / (2.0 * width * width);
  search_neighbors(G, b.spos, b.bin_start, i, w.x, w.y, w.z, r_max * r_max, false,
                   [&](int, int, int, int, double, double, double, double d2) {
                     const double r = sqrt(d2);
                     int k0, k1;
                     rdf_window(r, bw, width, nb, k0, k1);
                     for (int k = k0; k <= k1; ++k) {
                       const double x = r - (k + 0.5) * bw;
                       h[k] += 0.5 * exp(-x * x * inv2w2);  // each pair is visited twice
                     }
                   });
}

// dL/dq_i = sum_j dL/dr_ij * (-u_ij), dL/dr = sum_b dL/dh_b * dg/dr
__global__ void __launch_bounds__(128)
    k_rdf_grad(BinData b, int64_t n, double r_max, int nb, double width,
               const double *__restrict__ dl_dh, double *__restrict__ grad) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double4 w = b.spos[p];
  const int i = tag_atom(w.w);
  const int s = b.sys_of[i];
  const SysGeom &G = b.geom[s];
  const double *dh = dl_dh + (size_t)s * nb;
  const double bw = r_max / nb, inv2w2 = 1.0 / (2.0 * width * width), iw2 = 1.0 / (width * width);
  double gx = 0, gy = 0, gz = 0;
  search_neighbors(G, b.spos, b.bin_start, i, w.x, w.y, w.z, r_max * r_max, false,
                   [&](int, int, int, int, double dx, double dy, double dz, double d2) {
                     const double r = sqrt(d2);
                     double dlr = 0.0;
                     int k0, k1;
                     rdf_window(r, bw, width, nb, k0, k1);
                     for (int k = k0; k <= k1; ++k) {
                       const double x = r - (k + 0.5) * bw;
                       dlr += dh[k] * (-x * iw2) * exp(-x * x * inv2w2);
                     }
                     const double ir = 1.0 / r;
                     gx -= dlr * dx * ir;
                     gy -= dlr * dy * ir;
                     gz -= dlr * dz * ir;
                   });
  grad[3 * i] = gx;
  grad[3 * i + 1] = gy;
  grad[3 * i + 2] = gz;
}

// out[s, k] = sum over atoms of system s of part[i, k]  (fixed order)
__global__ void k_sum_parts(const SysGeom *g, const double *part, int width, double *out,
                            int accumulate) {
  const int s = blockIdx.x;
  const SysGeom &G = g[s];
  for (int k = threadIdx.x; k < width; k += blockDim.x) {
    double t = 0.0;
    for (int a = 0; a < G.count; ++a) t += part[(size_t)(G.start + a) * width + k];
    out[(size_t)s * width + k] = accumulate ? out[(size_t)s * width + k] + t : t;
  }
}

// Velocity-Verlet updates of the trajectory and its adjoint, one launch each,
// with the rounding of the element-wise tensor expressions they replace
// (nve.py:118-130 written as p + f * (dt / 2); q + (p * inv_m) * dt): every
// product and sum is rounded on its own (no fused multiply-add), so the results
// are bitwise those of the tensor expressions.
__global__ void k_vv_kick_drift(const double *q, const double *p, const double *f,
                                const double *inv_m, double half_dt, double dt, double *q_out,
                                double *p_out, int64_t n3) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n3) return;
  const double ph = __dadd_rn(p[k], __dmul_rn(f[k], half_dt));
  p_out[k] = ph;
  q_out[k] = __dadd_rn(q[k], __dmul_rn(__dmul_rn(ph, inv_m[k / 3]), dt));
}

__global__ void k_vv_kick(const double *p, const double *f, double half_dt, double *p_out,
                          int64_t n3) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n3) p_out[k] = __dadd_rn(p[k], __dmul_rn(f[k], half_dt));
}

// lam_p += lam_q * (dt * inv_m)
__global__ void k_adj_kick(double *lam_p, const double *lam_q, const double *inv_m, double dt,
                           int64_t n3) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n3) lam_p[k] = __dadd_rn(lam_p[k], __dmul_rn(lam_q[k], __dmul_rn(dt, inv_m[k / 3])));
}

}  // namespace tsb

using namespace tsb;

extern "C" int tsb_vv_kick_drift(const double *q, const double *p, const double *f,
                                 const double *inv_m, double half_dt, double dt, double *q_out,
                                 double *p_out, int64_t n_atoms, void *stream) {
  if (n_atoms < 0 || (n_atoms > 0 && (!q || !p || !f || !inv_m || !q_out || !p_out)))
    return TSB_ERR_INVALID_ARG;
  if (n_atoms == 0) return TSB_OK;
  k_vv_kick_drift<<<grid_for(3 * n_atoms), kBlock, 0, (cudaStream_t)stream>>>(
      q, p, f, inv_m, half_dt, dt, q_out, p_out, 3 * n_atoms);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_vv_kick(const double *p, const double *f, double half_dt, double *p_out,
                           int64_t n_atoms, void *stream) {
  if (n_atoms < 0 || (n_atoms > 0 && (!p || !f || !p_out))) return TSB_ERR_INVALID_ARG;
  if (n_atoms == 0) return TSB_OK;
  k_vv_kick<<<grid_for(3 * n_atoms), kBlock, 0, (cudaStream_t)stream>>>(p, f, half_dt, p_out,
                                                                        3 * n_atoms);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_adj_kick(double *lam_p, const double *lam_q, const double *inv_m, double dt,
                            int64_t n_atoms, void *stream) {
  if (n_atoms < 0 || (n_atoms > 0 && (!lam_p || !lam_q || !inv_m))) return TSB_ERR_INVALID_ARG;
  if (n_atoms == 0) return TSB_OK;
  k_adj_kick<<<grid_for(3 * n_atoms), kBlock, 0, (cudaStream_t)stream>>>(lam_p, lam_q, inv_m, dt,
                                                                         3 * n_atoms);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" size_t tsb_adjoint_workspace_size(int64_t n_atoms, int64_t n_systems,
                                             int64_t per_atom) {
  Carver c(nullptr, (size_t)-1);
  AdjWork w;
  carve_adj(c, w, n_atoms, n_systems, per_atom);
  return c.off + 256;
}

extern "C" int tsb_lj_hvp(const double *table, int n_species, const int32_t *species,
                          const double *positions, const double *cell_row, const uint8_t *pbc,
                          const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                          double cutoff, const double *v, double coef, double *lam_q,
                          double *grad_params, int64_t max_system_atoms, void *workspace,
                          size_t workspace_bytes, void *stream) {
  if (n_species < 1 || n_species > kAdjMaxSpecies || !table || (n_species > 1 && !species) ||
      n_atoms < 1 || n_systems < 1 || !positions || !cell_row || !pbc || !system_idx || !v ||
      !lam_q || !grad_params || !(cutoff > 0.0))
    return TSB_ERR_INVALID_ARG;
  const int per_atom = 2 * n_species * n_species;
  Carver c(workspace, workspace_bytes);
  AdjWork w;
  carve_adj(c, w, n_atoms, n_systems, per_atom);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  TSB_TRY(prepare_bins_any<double>(positions, cell_row, pbc, system_idx, n_atoms, n_systems,
                                   cutoff, w.b, st, species, max_system_atoms));
  if (n_atoms <= kGroupSearchMaxAtoms)
    k_lj_hvp<kSearchGroup><<<grid_for(kSearchGroup * n_atoms, 128), 128, 0, st>>>(
        w.b, n_atoms, table, n_species, species, cutoff, v, coef, lam_q, w.part);
  else
    k_lj_hvp<1><<<grid_for(n_atoms, 128), 128, 0, st>>>(
        w.b, n_atoms, table, n_species, species, cutoff, v, coef, lam_q, w.part);
  // per-system parameter gradients, accumulated into grad_params [S, ns, ns, 2]
  k_sum_parts<<<(unsigned)n_systems, 64, 0, st>>>(w.b.geom, w.part, per_atom, grad_params, 1);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_rdf_hist(const double *positions, const double *cell_row, const uint8_t *pbc,
                            const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                            double r_max, int n_bins, double width, double *hist,
                            int64_t max_system_atoms, void *workspace, size_t workspace_bytes,
                            void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !positions || !cell_row || !pbc || !system_idx || !hist ||
      n_bins < 1 || !(r_max > 0.0) || !(width > 0.0))
    return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  AdjWork w;
  carve_adj(c, w, n_atoms, n_systems, n_bins);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  TSB_TRY(prepare_bins_any<double>(positions, cell_row, pbc, system_idx, n_atoms, n_systems,
                                   r_max, w.b, st, nullptr, max_system_atoms));
  k_rdf_part<<<grid_for(n_atoms, 128), 128, 0, st>>>(w.b, n_atoms, r_max, n_bins, width, w.part);
  k_sum_parts<<<(unsigned)n_systems, 64, 0, st>>>(w.b.geom, w.part, n_bins, hist, 0);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_rdf_hist_grad(const double *positions, const double *cell_row,
                                 const uint8_t *pbc, const int64_t *system_idx, int64_t n_atoms,
                                 int64_t n_systems, double r_max, int n_bins, double width,
                                 const double *dl_dhist, double *grad_positions,
                                 int64_t max_system_atoms, void *workspace,
                                 size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !positions || !cell_row || !pbc || !system_idx ||
      !dl_dhist || !grad_positions || n_bins < 1 || !(r_max > 0.0) || !(width > 0.0))
    return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  AdjWork w;
  carve_adj(c, w, n_atoms, n_systems, n_bins);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  TSB_TRY(prepare_bins_any<double>(positions, cell_row, pbc, system_idx, n_atoms, n_systems,
                                   r_max, w.b, st, nullptr, max_system_atoms));
  k_rdf_grad<<<grid_for(n_atoms, 128), 128, 0, st>>>(w.b, n_atoms, r_max, n_bins, width,
                                                     dl_dhist, grad_positions);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}
