/*
 * tsb.h -- C ABI of the B200-native TorchSim classical-potential hot path.
 *
 * Every entry point takes raw device pointers, element counts, a caller-owned
 * device workspace and a CUDA stream (passed as void*), launches asynchronously
 * on that stream and returns an int status (TSB_OK on a successful launch).
 * No function allocates or frees device memory, synchronises the device or the
 * stream, or throws across the ABI.  Buffers are owned by the caller.
 *
 * Conventions (TorchSim metal units: Angstrom, eV, amu):
 *   positions  [n_atoms,3]   dtype TSB_F32 or TSB_F64, unwrapped Cartesian
 *   cell_row   [n_systems,3,3] row-vector cell (rows are lattice vectors) --
 *              the neighbour-list/pair-model convention of the reference
 *              (torch_sim/models/pair_potential.py:154,170)
 *   pbc        [n_systems,3] uint8 (0/1)
 *   system_idx [n_atoms] int64, contiguous and non-decreasing (state.py:223-254)
 *   table      [n_species,n_species,5] float64 rows (p0,p1,p2,rc,eshift):
 *              LJ:    p0=sigma p1=epsilon
 *              MORSE: p0=sigma p1=epsilon p2=alpha
 *              SOFT:  p0=sigma p1=epsilon p2=alpha
 *              PLIFE: p0=sigma p1=A p2=beta (particle life; the row of species pair
 *                     (a, b) is the force of a's neighbour b on a, so tables may be
 *                     asymmetric; no energy)
 *              rc = per-pair truncation radius, eshift subtracted inside rc.
 *   species    [n_atoms] int32 species index (NULL = all species 0)
 */
#ifndef TSB_H_
#define TSB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define TSB_OK 0
#define TSB_ERR_INVALID_ARG 1
#define TSB_ERR_CAPACITY 2     /* output/scratch capacity too small: regrow + retry */
#define TSB_ERR_NONFINITE 3    /* non-finite input detected on the device          */
#define TSB_ERR_TIMEOUT 4      /* a bounded device wait gave up                     */
#define TSB_ERR_CUDA 5         /* a CUDA launch failed                              */
#define TSB_ERR_UNSUPPORTED 6  /* configuration outside what the kernels handle     */
#define TSB_ERR_WORKSPACE 7    /* workspace smaller than *_workspace_size()         */

/* ---- dtypes / potentials / flags --------------------------------------- */
#define TSB_F32 0
#define TSB_F64 1

#define TSB_POT_LJ 0
#define TSB_POT_MORSE 1
#define TSB_POT_SOFT 2
#define TSB_POT_PLIFE 3 /* particle life (force-defined): tsb_pair_forward only */

#define TSB_NL_SELF_INTERACTION 1 /* also emit (i, i, 0) pairs                     */
#define TSB_NL_HALF 2             /* emit each unordered pair once (half list)      */

#define TSB_OUT_FORCES 1
#define TSB_OUT_STRESS 2
#define TSB_OUT_ENERGIES 4   /* per-atom energies                                */
#define TSB_OUT_STRESSES 8   /* per-atom stresses                                */
#define TSB_MATH_FP64 16     /* FP64 pair arithmetic (default: FP32 pair math,
                                FP64 displacements and FP64 per-system sums)    */

#define TSB_INT_NVE 0
#define TSB_INT_LANGEVIN 1
#define TSB_INT_NOSE_HOOVER 2 /* tsb_fused_md_nvt only */
#define TSB_INT_VRESCALE 3    /* tsb_fused_md_nvt only */

const char *tsb_version(void);
const char *tsb_status_string(int status);

/* ---- neighbour list ------------------------------------------------------
 * Replaces torch_sim/neighbors/torch_nl.py:156-215 (torch_nl_linked_cell, the
 * default backend behind torch_sim/neighbors/__init__.py:46-98 torchsim_nl).
 * Pair set: every (i, j, S) with |r_j - r_i + S @ cell_row| < cutoff, S integer
 * and zero on non-periodic axes, excluding (i, i, 0) unless
 * TSB_NL_SELF_INTERACTION; with TSB_NL_HALF only the copy full_to_half_list
 * keeps (torch_sim/models/pair_potential.py:86-127).
 * Outputs: mapping rows at mapping[0..cap) and mapping[mapping_stride..), the
 * system of each pair, integer shifts (as dtype) valid for the unwrapped
 * positions, grouped by i in ascending order.  *n_pairs (device int64) gets
 * the total; when it exceeds `capacity` nothing past capacity is written and
 * the caller regrows and calls again. */
size_t tsb_nl_workspace_size(int64_t n_atoms, int64_t n_systems);
int tsb_nl_build(const void *positions, const void *cell_row, const uint8_t *pbc,
                 const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                 int dtype, double cutoff, int flags, int64_t *mapping,
                 int64_t mapping_stride, int64_t *system_mapping, void *shifts,
                 int64_t capacity, int64_t *n_pairs, void *workspace,
                 size_t workspace_bytes, void *stream);

/* ---- pair potential energy / forces / virial -----------------------------
 * Replaces PairPotentialModel.forward (torch_sim/models/pair_potential.py:351-464)
 * for the pair functions of lennard_jones.py:23-47, morse.py:23-47,
 * soft_sphere.py:35-59 and the species-matrix lookup of soft_sphere.py:90-167.
 * The neighbour search is fused with the force evaluation (no pair list is
 * stored).  energy [S], stress [S,3,3], forces [N,3], energies [N],
 * stresses [N,3,3] are written in `dtype`; outputs not requested by
 * `out_flags` may be NULL.  `sys_active` [S] uint8 (optional): systems with 0
 * are skipped and their outputs left untouched (converged systems of a batched
 * relaxation).  `max_system_atoms`: the largest system's atom count (0 =
 * unknown); at most 4096 bins each system in one block (one launch), larger or
 * unknown bins the whole batch in passes; either is correct. */
size_t tsb_pair_workspace_size(int64_t n_atoms, int64_t n_systems);
int tsb_pair_forward(int potential, const double *table, int n_species,
                     const int32_t *species, const void *positions,
                     const void *cell_row, const uint8_t *pbc,
                     const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                     int dtype, double cutoff, int out_flags, void *energy,
                     void *forces, void *stress, void *energies, void *stresses,
                     const uint8_t *sys_active, int64_t max_system_atoms, void *workspace,
                     size_t workspace_bytes, void *stream);

/* ---- integrator steps (elementwise, per-system parameters) ---------------
 * dt_sys, kT_sys, gamma_sys are device float64 arrays of length n_systems.
 * tsb_md_kick:    p += F * (scale * dt)          (md.py:169-187, momentum_step)
 * tsb_md_drift:   q += p / m * (scale * dt)      (md.py:190-208, position_step)
 * tsb_md_baoab_boa: the B(dt/2) A(dt/2) O(dt) A(dt/2) part of nvt_langevin_step
 *   (torch_sim/integrators/nvt.py:144-240, _ou_step :27-86).  The O-step noise
 *   is read from `noise` [N,3] when non-NULL, else drawn from a counter-based
 *   Philox4x32-10 stream keyed by (seed, atom, counter + *counter_dev); when
 *   counter_dev is not NULL the call also advances *counter_dev by one on the
 *   stream, so a captured CUDA graph draws fresh noise on every replay. */
int tsb_md_kick(void *momenta, const void *forces, const int64_t *system_idx,
                const double *dt_sys, double scale, int64_t n_atoms, int dtype,
                void *stream);
int tsb_md_drift(void *positions, const void *momenta, const void *masses,
                 const int64_t *system_idx, const double *dt_sys, double scale,
                 int64_t n_atoms, int dtype, void *stream);
int tsb_md_baoab_boa(void *positions, void *momenta, const void *forces,
                     const void *masses, const int64_t *system_idx,
                     const double *dt_sys, const double *kT_sys,
                     const double *gamma_sys, const void *noise, uint64_t seed,
                     uint64_t counter, uint64_t *counter_dev, int64_t n_atoms, int dtype,
                     void *stream);

/* ---- Verlet-list forces for large periodic systems ----------------------
 * One fully periodic system whose cell widths are all >= cutoff + skin
 * (e.g. 500,000 atoms).  The reference rebuilds its list in every model call
 * (torch_sim/models/pair_potential.py:168-174); here the list holds all pairs
 * within cutoff + skin and is reused until an atom moved more than skin/2,
 * giving the same pairs and forces as PairPotentialModel.forward (:351-464).
 * tsb_verlet_build: cell-list search, ELL list[k * N + i] = j << 5 | image code,
 *   counts [N], reference positions [N,3] f64, integer wraps [N,3] i32;
 *   *status > 0 if an atom had more than max_neighbors (regrow and rebuild);
 *   cell_row in `dtype`.
 * tsb_verlet_check: maps the current positions into the build frame (kept in
 *   the workspace for tsb_verlet_forces) and sets *expired when any atom moved
 *   more than skin/2 or the cell differs from the build's (then rebuild and check
 *   again).  cell_row float64.
 * tsb_verlet_forces: energy [1], forces [N,3] (dtype), stress [1,3,3] with
 *   TSB_OUT_STRESS; e_atom [N] and vir_atom [N,6] are float64 scratch.  Uses the
 *   workspace filled by tsb_verlet_check.  cell_row float64. */
size_t tsb_verlet_workspace_size(int64_t n_atoms);
int tsb_verlet_build(const void *positions, const void *cell_row, int64_t n_atoms, int dtype,
                     double cutoff, double skin, uint32_t *list, int32_t *counts,
                     int max_neighbors, double *ref_positions, int32_t *wraps,
                     int32_t *status, void *workspace, size_t workspace_bytes,
                     void *stream);
int tsb_verlet_check(const void *positions, const double *ref_positions,
                     const int32_t *wraps, const double *cell_row, const int32_t *species,
                     int64_t n_atoms, int dtype, double skin, int32_t *expired,
                     void *workspace, size_t workspace_bytes, void *stream);
int tsb_verlet_forces(int potential, const double *table, int n_species,
                      const uint32_t *list, const int32_t *counts, int64_t n_atoms,
                      const double *cell_row, int dtype, double cutoff, int out_flags,
                      void *energy, void *forces, void *stress, double *e_atom,
                      double *vir_atom, void *workspace, size_t workspace_bytes,
                      void *stream);

/* ---- anisotropic NPT Langevin (per-axis strains) ---------------------------
 * npt_langevin_anisotropic_step (torch_sim/integrators/npt.py:513-650): strains
 * eps [S,3], cell row k = exp(eps_k) * row k of reference_cell [S,9] (float64),
 * strain forces F_k = V (-stress_kk + N kT / V - p_ext_k) with V = det(cell),
 * GJF strain and particle steps as the isotropic pair; p_ext [S,3]; f_eps [S,3];
 * cell noise [S,3] (or NULL: Philox) shared by both halves, particle noise [N,3]
 * likewise.  Workspace: tsb_npt_workspace_size. */
int tsb_npt_langevin_aniso_pre(void *positions, const void *momenta, const void *forces,
                               const void *masses, const int64_t *system_idx, int64_t n_atoms,
                               int64_t n_systems, int dtype, const void *stress,
                               const double *reference_cell, void *cell, double *eps,
                               const double *eps_dot, double *cell_masses, double *f_eps,
                               const double *alpha, const double *cell_alpha,
                               const double *b_tau, const double *kT, const double *p_ext,
                               const double *dt, const double *cell_noise,
                               const double *particle_noise, uint64_t seed, uint64_t counter,
                               void *workspace, size_t workspace_bytes, void *stream);
int tsb_npt_langevin_aniso_post(void *momenta, const void *masses, const void *forces_old,
                                const void *forces, const int64_t *system_idx, int64_t n_atoms,
                                int64_t n_systems, int dtype, const void *stress,
                                const void *cell, double *eps_dot, const double *cell_masses,
                                const double *f_eps, const double *alpha,
                                const double *cell_alpha, const double *kT, const double *p_ext,
                                const double *dt, const double *cell_noise,
                                const double *particle_noise, uint64_t seed, uint64_t counter,
                                void *workspace, size_t workspace_bytes, void *stream);

/* ---- isotropic NPT Nose-Hoover (MTK) inner step -------------------------------
 * The part of npt_nose_hoover_isotropic_step (torch_sim/integrators/npt.py:
 * 1532-1639, 1812-1963) between the chain half steps (those run on
 * tsb_nhc_half_step).  eps [S] = ln(V/V0)/3, p_eps [S] cell momentum, cell_mass
 * [S] W, reference_cell [S,9] float64, v_eps [S] out (pre) / in (post).
 * pre: p_eps += F dt/2 with F = alpha 2 KE - tr(stress) V - 3 P V, alpha =
 *   1 + 3/(3N - 3); v = p_eps/W; momenta by exp(iL2), eps += v dt, cell =
 *   (V/V0)^(1/3) ref, positions by exp(iL1).
 * post (after the force call): momenta by exp(iL2) with the new forces, p_eps +=
 *   F(new stress, new volume) dt/2.  Workspace: tsb_npt_workspace_size. */
int tsb_npt_nh_iso_pre(void *positions, void *momenta, const void *forces, const void *masses,
                       const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                       int dtype, const void *stress, const double *reference_cell, void *cell,
                       double *eps, double *p_eps, const double *cell_mass,
                       const double *p_ext, const double *dt, double *v_eps, void *workspace,
                       size_t workspace_bytes, void *stream);
int tsb_npt_nh_iso_post(void *momenta, const void *forces, const void *masses,
                        const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                        int dtype, const void *stress, const double *reference_cell,
                        const double *eps, double *p_eps, const double *p_ext,
                        const double *dt, const double *v_eps, void *workspace,
                        size_t workspace_bytes, void *stream);

/* ---- isotropic C-rescale barostat -----------------------------------------
 * The barostat step of npt_crescale_isotropic_step (torch_sim/integrators/
 * npt.py:2455-2492, 2797-2901; Bernetti & Bussi 2020): per system, the trace of
 * the instantaneous pressure (quantities.py:156-198), the stochastic update of
 * sqrt(V), mu = (V'/V)^(1/3), cell *= mu; per atom r <- mu r + (mu + 1/mu) p dt /
 * (2 m), p <- p / mu.  cell is the state's [S,3,3] cell (either convention: only
 * its determinant and a scale enter).  Per-system parameters are float64 [S];
 * noise [S] (standard normal) or NULL for the counter-based Philox draw (seed,
 * system, counter).  Workspace: tsb_npt_workspace_size. */
int tsb_npt_crescale_iso(void *positions, void *momenta, const void *masses,
                         const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                         int dtype, const void *stress, void *cell,
                         const double *compressibility, const double *tau_p, const double *kT,
                         const double *p_ext, const double *dt, const double *noise,
                         uint64_t seed, uint64_t counter, void *workspace,
                         size_t workspace_bytes, void *stream);

/* tsb_npt_crescale_aniso: the anisotropic barostat step of
 * npt_crescale_anisotropic_step (npt.py:2282-2343, 2645-2720): two half steps of
 * sqrt(V) around a traceless random per-axis deformation, per-axis factors mu_k,
 * cell row k *= mu_k (rows of the state's column-convention cell), r_k <- mu_k r_k
 * + (mu_k + 1/mu_k) p_k dt / (2 m), p_k <- p_k / mu_k.  noise [S, 5] = (volume
 * normal, z_x, z_y, z_z, volume normal) or NULL for Philox draws.  Workspace:
 * tsb_npt_workspace_size. */
int tsb_npt_crescale_aniso(void *positions, void *momenta, const void *masses,
                           const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                           int dtype, const void *stress, void *cell,
                           const double *compressibility, const double *tau_p, const double *kT,
                           const double *p_ext, const double *dt, const double *noise,
                           uint64_t seed, uint64_t counter, void *workspace,
                           size_t workspace_bytes, void *stream);

/* tsb_npt_crescale_tri: the triclinic barostat step of npt_crescale_triclinic_step
 * (npt.py:2186-2280, 2517-2644) or, with average != 0, of
 * npt_crescale_triclinic_average_step (:2376-2452, 2721-2796; average kinetic
 * pressure (3N - 3)/3 kT / V, momenta unscaled).  Per system: the pressure tensor,
 * for a tensor external pressure p_ext_tensor [S, 9] (NULL: scalar p_ext [S]) the
 * deviatoric correction through initial_cell_inv [S, 9] and initial_volume [S],
 * two half steps of sqrt(V), R = GramSchmidt(expm(a~ dt + c Z~)) (V''/V)^(1/3),
 * cell <- cell R^T; per atom r <- R r + (M + R) p dt / (2 m), p <- M p with
 * M = inv(R)^T (I for the average variant).  noise [S, 11] = (volume normal, 3x3
 * normals row-major, volume normal) or NULL for Philox draws.  Workspace:
 * tsb_npt_workspace_size. */
int tsb_npt_crescale_tri(void *positions, void *momenta, const void *masses,
                         const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                         int dtype, const void *stress, void *cell,
                         const double *compressibility, const double *tau_p, const double *kT,
                         const double *p_ext, const double *p_ext_tensor,
                         const double *initial_cell_inv, const double *initial_volume,
                         const double *dt, int average, const double *noise, uint64_t seed,
                         uint64_t counter, void *workspace, size_t workspace_bytes,
                         void *stream);

/* ---- batched Verlet lists (many systems, moving atoms and cells) ----------
 * Replaces the per-call neighbour search inside PairPotentialModel.forward
 * (torch_sim/models/pair_potential.py:168-174, 351-464) for a batch whose atoms
 * and cells change between calls (FIRE with a cell filter, NPT, MD).  Each
 * system's list holds every pair within cutoff + skin (image shifts in
 * {-1,0,1}^3 of the cell at its build) and is rebuilt, per system, when
 * 2 max|u| + (cutoff + skin) |F - I| > skin (F = C0^-1 C the cell deformation
 * since the build, u_i = w_i - w0_i F an atom's non-affine drift in the build
 * frame).  The pairs inside the cutoff, hence energy, forces and stresses, equal
 * the per-call path.
 * The workspace (tsb_vlist_workspace_size) holds the list frame and must be kept
 * by the caller between calls; tsb_vlist_reset marks every system unbuilt.
 * tsb_vlist_check: flags[0] = 1 when any active system must be rebuilt.
 *   prune_skin (0 <= prune_skin; 0 or >= skin: off) also marks the systems whose
 *   pruned lists must be formed again: 2 max|u'| + (cutoff + prune_skin)
 *   |F' - I| > prune_skin, with F' and u' measured since the system's last
 *   pruning (and every system rebuilt since it).
 * tsb_vlist_build: rebins and rebuilds the expired systems' lists
 *   (list[k * N + slot] = slot of j << 5 | image code, counts [N] by slot).
 *   max_system_atoms = the largest system's atom count (0: unknown); when it is
 *   at most 4096 only the expired systems are rebinned, one block each, else the
 *   whole batch is (the hint selects the faster way; either is correct).
 *   flags[1] = 1 << 30 when a periodic cell is narrower than cutoff + skin, else
 *   the largest neighbour count when it exceeded max_neighbors (regrow, reset and
 *   build again), else 0.
 * tsb_vlist_forces: energy [S], forces [N,3], stress [S,3,3], per-atom energies
 *   [N] and stresses [N,3,3] per out_flags (TSB_MATH_FP64: FP64 pair function),
 *   for the systems with sys_active != 0 (NULL: all).  LJ, Morse, soft sphere.
 *   prune_skin > 0 (the value given to the preceding tsb_vlist_check, which must
 *   run before every call): the marked systems' lists are first reordered in
 *   place so that the entries within their pair cutoff + prune_skin form a front
 *   part, and only front parts are evaluated.  The pairs are those of the whole
 *   lists; results equal theirs to FP64 rounding (another summation order). */
size_t tsb_vlist_workspace_size(int64_t n_atoms, int64_t n_systems);
int tsb_vlist_reset(int64_t n_atoms, int64_t n_systems, void *workspace,
                    size_t workspace_bytes, void *stream);
int tsb_vlist_check(const void *positions, const void *cell_row, const int64_t *system_idx,
                    const uint8_t *sys_active, int64_t n_atoms, int64_t n_systems, int dtype,
                    double cutoff, double skin, double prune_skin, int32_t *flags,
                    void *workspace, size_t workspace_bytes, void *stream);
int tsb_vlist_build(const void *positions, const void *cell_row, const uint8_t *pbc,
                    const int64_t *system_idx, const int32_t *species, int64_t n_atoms,
                    int64_t n_systems, int dtype, double cutoff, double skin, uint32_t *list,
                    int32_t *counts, int max_neighbors, int64_t max_system_atoms,
                    int32_t *flags, void *workspace, size_t workspace_bytes, void *stream);
/* tsb_vlist_lj_hvp: the adjoint's LJ Hessian-vector product (as tsb_lj_hvp:
 *   lam_q += coef * J_F(q)^T v, grad_params [S, ns, ns, 2] += coef *
 *   dF/d(sigma, epsilon)^T v) over lists built for `positions` (FP64; rows of
 *   `table` as for tsb_lj_hvp); scratch of tsb_vlist_hvp_scratch_size bytes. */
size_t tsb_vlist_hvp_scratch_size(int64_t n_atoms, int n_species);
int tsb_vlist_lj_hvp(const double *table, int n_species, const int32_t *species,
                     const uint32_t *list, const int32_t *counts, const double *positions,
                     const double *cell_row, const int64_t *system_idx, int64_t n_atoms,
                     int64_t n_systems, double cutoff, const double *v, double coef,
                     double *lam_q, double *grad_params, void *scratch, size_t scratch_bytes,
                     void *workspace, size_t workspace_bytes, void *stream);
int tsb_vlist_forces(int potential, const double *table, int n_species, const int32_t *species,
                     uint32_t *list, const int32_t *counts, const void *positions,
                     const void *cell_row, const int64_t *system_idx, const uint8_t *sys_active,
                     int64_t n_atoms, int64_t n_systems, int dtype, double cutoff,
                     double prune_skin, int out_flags, void *energy, void *forces, void *stress,
                     void *energies, void *stresses, void *workspace, size_t workspace_bytes,
                     void *stream);

/* ---- adjoint of NVE trajectories (species-matrix LJ, FP64) ---------------
 * No kernel of the reference corresponds: it differentiates trajectories with
 * torch.autograd through PairPotentialModel (pair_potential.py:420-425), which
 * omits the force-Jacobian terms.  These are the pieces of the exact discrete
 * adjoint of velocity Verlet (nve.py:74-130):
 * tsb_lj_hvp: lam_q += coef * J_F(q)^T v (J_F = -Hessian of the LJ energy) and
 *   grad_params [S, ns, ns, 2] += coef * dF/d(sigma_ab, epsilon_ab)^T v per system.
 * tsb_rdf_hist: hist [S, n_bins] = sum over pairs r < r_max of
 *   exp(-(r - c_b)^2 / (2 width^2)), c_b = (b + 1/2) r_max / n_bins.
 * tsb_rdf_hist_grad: grad_positions [N,3] = d(sum_sb dl_dhist_sb hist_sb)/dq.
 * per_atom for tsb_adjoint_workspace_size: 2*ns*ns (hvp) or n_bins (rdf).
 * max_system_atoms: as for tsb_pair_forward. */
size_t tsb_adjoint_workspace_size(int64_t n_atoms, int64_t n_systems, int64_t per_atom);
/* Velocity-Verlet pieces of the trajectory and its adjoint (FP64, [N,3] arrays,
 * inv_m [N]); each product and sum rounded on its own, as the tensor expressions
 * of nve.py:118-130 round them:
 * tsb_vv_kick_drift: p_out = p + f * half_dt;  q_out = q + (p_out * inv_m) * dt
 * tsb_vv_kick:       p_out = p + f * half_dt
 * tsb_adj_kick:      lam_p += lam_q * (dt * inv_m) */
int tsb_vv_kick_drift(const double *q, const double *p, const double *f, const double *inv_m,
                      double half_dt, double dt, double *q_out, double *p_out, int64_t n_atoms,
                      void *stream);
int tsb_vv_kick(const double *p, const double *f, double half_dt, double *p_out,
                int64_t n_atoms, void *stream);
int tsb_adj_kick(double *lam_p, const double *lam_q, const double *inv_m, double dt,
                 int64_t n_atoms, void *stream);
int tsb_lj_hvp(const double *table, int n_species, const int32_t *species,
               const double *positions, const double *cell_row, const uint8_t *pbc,
               const int64_t *system_idx, int64_t n_atoms, int64_t n_systems, double cutoff,
               const double *v, double coef, double *lam_q, double *grad_params,
               int64_t max_system_atoms, void *workspace, size_t workspace_bytes,
               void *stream);
int tsb_rdf_hist(const double *positions, const double *cell_row, const uint8_t *pbc,
                 const int64_t *system_idx, int64_t n_atoms, int64_t n_systems, double r_max,
                 int n_bins, double width, double *hist, int64_t max_system_atoms,
                 void *workspace, size_t workspace_bytes, void *stream);
int tsb_rdf_hist_grad(const double *positions, const double *cell_row, const uint8_t *pbc,
                      const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                      double r_max, int n_bins, double width, const double *dl_dhist,
                      double *grad_positions, int64_t max_system_atoms, void *workspace,
                      size_t workspace_bytes, void *stream);

/* ---- FIRE + Frechet cell filter -----------------------------------------
 * Per-system state arrays (dtype): dt [S], alpha [S], n_pos [S] int32; cell,
 * reference_cell, cell_positions, cell_velocities, cell_forces [S,3,3] in the
 * COLUMN-vector convention of SimState.cell (state.py:138-142); cell_factor
 * [S]; cell_masses [S] (sum of atomic masses, cell_filters.py:97-101).
 * cell_filter 0 = positions only, 1 = Frechet filter.  Systems whose `active`
 * entry is 0 are skipped.  eps is 1e-8 (float32) / 1e-16 (float64) as in
 * fire.py:154.
 * tsb_fire_ase_pre: fire.py:288-485 (_ase_fire_step up to the model call).
 * tsb_fire_vv_pre / tsb_fire_vv_post: fire.py:179-285 around the model call.
 * tsb_frechet_cell_forces: cell_filters.py:353-391 (init=1: the initial cell
 *   forces of frechet_cell_filter_init, cell_filters.py:230-284).
 * tsb_fire_converged: max|F_i| < fmax (and cell-force row norms < fmax when
 *   cell_forces is given) per system, runners.py:501-538; converged systems
 *   get active = 0, *n_active (device int32) counts the rest. */
size_t tsb_fire_workspace_size(int64_t n_systems);
#define TSB_FIRE_ARGS_DECL                                                       \
  int cell_filter, void *positions, void *velocities, const void *forces,       \
      const void *masses, const int64_t *system_idx, int64_t n_atoms,           \
      int64_t n_systems, void *dt, void *alpha, int32_t *n_pos, void *cell,     \
      const void *reference_cell, const void *cell_factor,                      \
      void *cell_positions, void *cell_velocities, const void *cell_forces,     \
      const void *cell_masses, const uint8_t *active, double dt_max,            \
      int n_min, double f_inc, double f_dec, double alpha_start,                \
      double f_alpha, double max_step, double eps, int dtype, void *workspace,  \
      size_t workspace_bytes, void *stream
int tsb_fire_ase_pre(TSB_FIRE_ARGS_DECL);
int tsb_fire_vv_pre(TSB_FIRE_ARGS_DECL);
int tsb_fire_vv_post(TSB_FIRE_ARGS_DECL);
int tsb_frechet_cell_forces(void *cell_forces, const void *stress, const void *cell,
                            const void *reference_cell, const void *pressure,
                            const void *cell_factor, int64_t n_systems, int init,
                            const uint8_t *active, int dtype, void *stream);
int tsb_fire_converged(const void *forces, const int64_t *system_idx, int64_t n_atoms,
                       int64_t n_systems, const void *cell_forces, double fmax,
                       uint8_t *active, int32_t *n_active, int dtype, void *workspace,
                       size_t workspace_bytes, void *stream);

/* ---- NVT thermostats: Nose-Hoover chains and V-rescale (CSVR) -------------
 * One block per system; per-system arrays are float64 [S] (chain arrays [S,M]).
 * tsb_kinetic_energy: ke[s] = 1/2 sum p^2/m over system s (quantities.py:104-139).
 * tsb_nhc_half_step: the chain half step of nvt_nose_hoover_step
 *   (torch_sim/integrators/md.py:388-514, nvt.py:381-488): chain_steps x sy_steps
 *   Suzuki-Yoshida sub-steps (sy_steps 1, 3, 5 or 7) of the chain positions xi and
 *   momenta p_xi (in/out), chain masses Q (out) recomputed from kT, tau and dof
 *   (Q_j = kT tau^2, Q_1 = dof kT tau^2, md.py:534-559), momenta rescaled in place.
 *   ke (in/out) is the kinetic energy the chain sees: with recompute_ke it is
 *   first summed from the momenta, else the value carried from the last call is
 *   used (as the reference carries chain.kinetic_energy).  dt is the chain's
 *   time step (the one the chain was constructed with, md.py:495-508).
 *   chain_length 1..16.
 * tsb_vrescale: momenta *= lambda per system, lambda^2 = c1 + c2 (r1^2 + 2 g) +
 *   2 r1 sqrt(c1 c2), c1 = exp(-dt/tau), c2 = (1 - c1) (dof kT / 2) / KE / dof
 *   (nvt.py:594-654).  noise [S,2] = (r1, g) with g ~ Gamma((dof-1)/2, 1) when
 *   non-NULL; else both are drawn on the device from Philox4x32-10 keyed by
 *   (seed, system, counter).  lam [S] (optional) receives lambda. */
size_t tsb_thermostat_workspace_size(int64_t n_systems);
int tsb_kinetic_energy(const void *momenta, const void *masses, const int64_t *system_idx,
                       int64_t n_atoms, int64_t n_systems, int dtype, double *ke,
                       void *workspace, size_t workspace_bytes, void *stream);
int tsb_nhc_half_step(void *momenta, const void *masses, const int64_t *system_idx,
                      int64_t n_atoms, int64_t n_systems, int dtype, double *xi,
                      double *p_xi, double *Q, double *ke, const double *dof,
                      const double *kT, const double *tau, const double *dt,
                      int chain_length, int chain_steps, int sy_steps, int recompute_ke,
                      void *workspace, size_t workspace_bytes, void *stream);
int tsb_vrescale(void *momenta, const void *masses, const int64_t *system_idx,
                 int64_t n_atoms, int64_t n_systems, int dtype, const double *dof,
                 const double *kT, const double *tau, const double *dt, const double *noise,
                 uint64_t seed, uint64_t counter, double *lam, void *workspace,
                 size_t workspace_bytes, void *stream);

/* ---- isotropic NPT Langevin (strain-based GJF) ----------------------------
 * npt_langevin_isotropic_step (torch_sim/integrators/npt.py:988-1107), split
 * around the force/stress call.  Atom arrays (positions, momenta, forces,
 * masses) and stress [S,3,3] / cell [S,3,3] have dtype `dtype`; per-system
 * scalars are float64 [S]: eps (strain, in/out), eps_dot (strain velocity),
 * cell_masses (Q = (N + 1) kT b_tau^2, written by _pre), f_eps (strain force
 * before the step, written by _pre, read by _post), alpha / cell_alpha (particle /
 * cell friction), b_tau, kT, p_ext, dt.  reference_cell [S,3,3] float64; _pre
 * writes cell = exp(eps) reference_cell.  Noise: cell_noise [S] and
 * particle_noise [N,3] standard normals, or NULL to draw them from Philox4x32-10
 * keyed by (seed, system/atom, counter); _pre and _post must see the same noise
 * (same arrays or the same seed and counter). */
size_t tsb_npt_workspace_size(int64_t n_systems);
int tsb_npt_langevin_iso_pre(void *positions, const void *momenta, const void *forces,
                             const void *masses, const int64_t *system_idx, int64_t n_atoms,
                             int64_t n_systems, int dtype, const void *stress,
                             const double *reference_cell, void *cell, double *eps,
                             const double *eps_dot, double *cell_masses, double *f_eps,
                             const double *alpha, const double *cell_alpha,
                             const double *b_tau, const double *kT, const double *p_ext,
                             const double *dt, const double *cell_noise,
                             const double *particle_noise, uint64_t seed, uint64_t counter,
                             void *workspace, size_t workspace_bytes, void *stream);
int tsb_npt_langevin_iso_post(void *momenta, const void *masses, const void *forces_old,
                              const void *forces, const int64_t *system_idx, int64_t n_atoms,
                              int64_t n_systems, int dtype, const void *stress,
                              const double *reference_cell, const double *eps,
                              double *eps_dot, const double *cell_masses,
                              const double *f_eps, const double *alpha,
                              const double *cell_alpha, const double *kT,
                              const double *p_ext, const double *dt, const double *cell_noise,
                              const double *particle_noise, uint64_t seed, uint64_t counter,
                              void *workspace, size_t workspace_bytes, void *stream);

/* ---- fused persistent batched MD ----------------------------------------
 * Advances every system by n_steps of velocity Verlet (TSB_INT_NVE,
 * nve.py:74-130) or BAOAB Langevin (TSB_INT_LANGEVIN, nvt.py:144-240) in one
 * persistent launch: one CTA owns one system at a time, keeps its atoms and a
 * Verlet list (cutoff + skin, rebuilt on the device when an atom moved more
 * than skin/2) in shared memory, and steps it without leaving the kernel.
 * positions/momenta/forces are float64 [N,3] in/out; energy [S] float64 out
 * (potential energy after the last step); stress [S,3,3] float64 out
 * (optional, NULL skips it): the stress after the last step, -W/V with the
 * virial W = sum over pairs of r (x) f (pair_potential.py:200-274); per-atom
 * energy and virial terms are summed in FP64 in a fixed order;
 * n_rebuilds [S] int32 out (optional).
 * `order` [S] int32 (optional) is the order in which CTAs pick systems
 * (largest first balances the tail).  A system whose images or neighbours do
 * not fit the shared-memory tables at the requested skin is rebuilt with a
 * smaller skin (results are unchanged; only the rebuild rate grows).
 * `status` [4] int32 device out: status[0] is TSB_OK, or TSB_ERR_CAPACITY /
 * TSB_ERR_UNSUPPORTED for a system that does not fit even with zero skin
 * (its positions and momenta are left unchanged, its forces are not);
 * status[1] its index, status[2] which table (1 images, 2 neighbour slots),
 * status[3] the size that did not fit; or TSB_ERR_INVALID_ARG with status[1]
 * an atom whose system index lies outside [0, n_systems), status[2] = 3 and
 * status[3] that index (the atom is left out of every system).  While a system runs, its rows of
 * `forces` hold FP64 positions (the kernel decides whether a pair is inside
 * the cutoff on them when FP32 rounding could flip the decision); the final
 * forces are written over them.
 * The Langevin noise of MD step t (0-based within the launch) is drawn with
 * Philox counter `counter + t` (+ *counter_dev when counter_dev is not NULL; the
 * call then advances *counter_dev by n_steps on the stream, so a captured CUDA
 * graph draws fresh noise on every replay).
 * Requirements: pbc all true, n_atoms per system <= tsb_fused_max_atoms(). */
int tsb_fused_max_atoms(void);
size_t tsb_fused_workspace_size(int64_t n_atoms, int64_t n_systems);
int tsb_fused_md(int integrator, int potential, const double *table, int n_species,
                 const int32_t *species, double *positions, double *momenta,
                 double *forces, const double *masses, const double *cell_row,
                 const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                 const int32_t *order, double cutoff, double skin, int64_t n_steps,
                 const double *dt_sys, const double *kT_sys, const double *gamma_sys,
                 uint64_t seed, uint64_t counter, uint64_t *counter_dev, double *energy,
                 double *stress, int32_t *n_rebuilds, int32_t *status, void *workspace,
                 size_t workspace_bytes, void *stream);

/* ---- fused persistent batched MD with a Nose-Hoover chain or V-rescale ----
 * tsb_fused_md with thermostat TSB_INT_NOSE_HOOVER (nvt_nose_hoover_step,
 * torch_sim/integrators/nvt.py:381-488: chain half step, velocity Verlet, chain
 * half step, per system) or TSB_INT_VRESCALE (nvt_vrescale_step, nvt.py:715-741:
 * CSVR rescale, then velocity Verlet).  The thermostat arithmetic is that of
 * tsb_nhc_half_step / tsb_vrescale (shared code), degrees of freedom 3N - 3.
 * tau_sys [S]: thermostat time constant.  Nose-Hoover: chain_xi, chain_pxi,
 * chain_Q [S, chain_length] and chain_ke [S] in/out (the state's chain; Q is
 * recomputed from kT, tau, dof), chain_dt [S] the chain's time step.
 * V-rescale draws (r1, Gamma) from the Philox stream (seed, system,
 * counter + step), the same stream tsb_vrescale uses with that counter. */
int tsb_fused_md_nvt(int thermostat, int potential, const double *table, int n_species,
                     const int32_t *species, double *positions, double *momenta,
                     double *forces, const double *masses, const double *cell_row,
                     const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                     const int32_t *order, double cutoff, double skin, int64_t n_steps,
                     const double *dt_sys, const double *kT_sys, const double *tau_sys,
                     double *chain_xi, double *chain_pxi, double *chain_Q, double *chain_ke,
                     const double *chain_dt, int chain_length, int chain_steps, int sy_steps,
                     uint64_t seed, uint64_t counter, uint64_t *counter_dev, double *energy,
                     double *stress, int32_t *n_rebuilds, int32_t *status, void *workspace,
                     size_t workspace_bytes, void *stream);

/* ---- fused persistent batched MD, every integrator, with trajectory frames ----
 * Superset of tsb_fused_md and tsb_fused_md_nvt (integrator TSB_INT_NVE ..
 * TSB_INT_VRESCALE; arguments a thermostat does not use may be NULL).  With
 * report_every > 0, after every report_every-th step the kernel writes frame
 * f = step / report_every - 1 (f < n_frames): positions as float32 into
 * frame_x [n_frames, N, 3] and each system's potential energy into
 * frame_e [n_frames, S] -- the device side of the reference's
 * TrajectoryReporter (torch_sim/trajectory.py:267-340, coerce_to_float32).
 * lanes_max (0 or a power of two <= 32; 0 means 32) caps the threads that share
 * one atom's neighbour list in small systems (a launch shape the autotuner
 * picks; results do not depend on it).  n_wide >= 0 (with `order`) splits the
 * systems over two block shapes: order[0 .. n_wide) run in 512-thread blocks,
 * one per SM, and order[n_wide .. S) in 256-thread blocks, two per SM -- those
 * systems must have at most 256 atoms and fit the narrow blocks' image table of
 * 1968 entries at the given skin (else their skin shrinks until it fits, or
 * TSB_ERR_CAPACITY is reported); n_wide < 0 runs every system in 512-thread
 * blocks.  prune_skin (0 <= prune_skin; 0 or >= skin: off) prunes the list
 * between builds: only the pairs of the list's shell that lie within
 * cutoff + prune_skin are evaluated, and the shell is pruned again whenever an
 * atom moved more than prune_skin / 2 since the last pruning.  Results do not
 * depend on it beyond FP32 summation order. */
int tsb_fused_md_ex(int integrator, int potential, const double *table, int n_species,
                    const int32_t *species, double *positions, double *momenta,
                    double *forces, const double *masses, const double *cell_row,
                    const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                    const int32_t *order, double cutoff, double skin, int64_t n_steps,
                    const double *dt_sys, const double *kT_sys, const double *gamma_sys,
                    const double *tau_sys, double *chain_xi, double *chain_pxi,
                    double *chain_Q, double *chain_ke, const double *chain_dt,
                    int chain_length, int chain_steps, int sy_steps, uint64_t seed,
                    uint64_t counter, uint64_t *counter_dev, float *frame_x, double *frame_e,
                    int64_t report_every, int64_t n_frames, int lanes_max, int64_t n_wide,
                    double prune_skin, double *energy, double *stress, int32_t *n_rebuilds,
                    int32_t *status, void *workspace, size_t workspace_bytes, void *stream);

/* ---- allocation-free fused MD -------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory -- hosts that own all device memory through their own pool and bar
 * libraries from cudaMalloc, code that must not trigger the implicit
 * device-wide synchronisation of cudaMalloc/cudaFree while other streams run,
 * or runs with a fixed memory budget that cannot risk a failed allocation.
 * Same arguments and results as tsb_fused_md, minus the workspace: the scratch
 * (per-system atom ranges and the work counter, about 256 KB) is a fixed array
 * inside the library that every GPU loading the library keeps until exit.
 * At most TSB_FUSED_STATIC_MAX_SYSTEMS systems per call; more returns
 * TSB_ERR_CAPACITY without launching anything.  The first call on each device
 * looks up the array's device address (make that first call before any stream
 * capture).  All calls share the one array: calls that overlap on the GPU
 * (from different streams or host threads) race and must be serialised.
 * Nothing here calls cudaMalloc, cudaFree or any allocating routine. */
#define TSB_FUSED_STATIC_MAX_SYSTEMS 16384
int tsb_fused_md_static(int integrator, int potential, const double *table,
                        int n_species, const int32_t *species, double *positions,
                        double *momenta, double *forces, const double *masses,
                        const double *cell_row, const int64_t *system_idx,
                        int64_t n_atoms, int64_t n_systems, const int32_t *order,
                        double cutoff, double skin, int64_t n_steps,
                        const double *dt_sys, const double *kT_sys,
                        const double *gamma_sys, uint64_t seed, uint64_t counter,
                        double *energy, int32_t *n_rebuilds, int32_t *status,
                        void *stream);

#ifdef __cplusplus
}
#endif
#endif /* TSB_H_ */
