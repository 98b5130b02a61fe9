// Batched Verlet lists: many systems, moving atoms and changing cells (FIRE with
// a cell filter, NPT, plain MD on a batch).  Drop-in for the neighbour search
// inside PairPotentialModel.forward (torch_sim/models/pair_potential.py:351-464),
// which rebuilds its list in every call (pair_potential.py:168-174).  Here each
// system's list holds every pair within cutoff + skin, is kept between calls and
// is rebuilt, per system, only when the bound below allows a pair to have moved
// from beyond cutoff + skin to inside the cutoff.  The pairs inside the cutoff,
// and so energies, forces and stresses, are those of the per-call search.
//
// Validity.  A system's list is built at cell C0 (rows = lattice vectors) from
// positions wrapped into it, w0_i = x0_i - W_i C0 (W_i integer, zero on open
// axes), with entries (i, j, S), S in {-1,0,1}^3 (code (Sx+1)*9 + (Sy+1)*3 +
// (Sz+1)); the search covers every image, and the build fails when a pair with
// |S|_inf >= 2 lies within cutoff + skin, so every pair left out of the list was
// at least cutoff + skin apart.  At a later call with positions x and cell C the
// frame positions are w_i = x_i - W_i C.  With the deformation F = C0^-1 C (the
// identity for a system without a fractional frame) and the non-affine drift
// u_i = w_i - w0_i F, any pair's vector is exactly r = r0 F + u_j - u_i (the
// image term S C - S C0 F vanishes), so |r| >= |r0| (1 - |F - I|) - 2 max|u|.
// A system's list therefore stays valid while 2 max|u| + (cutoff + skin) e <=
// skin, e = |F - I|_Frobenius (< 1): each call sets dmax = (skin - (cutoff +
// skin) e) / 2 per system and expires the system when an atom's |u_i| exceeds it.
// A uniform strain costs (cutoff + skin) e, not the atoms' affine displacement.
//
// Layout by slot: a system's atoms occupy the slots of its atom range, ordered
// by the bins of its last build (perm[slot] = atom), so neighbouring threads and
// their neighbours sit close in memory.  ELL list[k * N + slot] (uint32: slot of
// j << 5 | image code), counts per slot, frame positions per slot as double4 with
// the species in the high word of .w (and as float4 for the FP32 path).  Force
// kernel: one thread per slot over its list, pair function in R, FP64
// accumulation, per-system sums in a fixed order (deterministic).  The FP64 path
// forms displacements and the cutoff test in FP64.  The FP32 path gathers float4
// positions and decides in FP32 outside a band around each cutoff that bounds
// the FP32 rounding of r^2: with |coordinates|, |shifts| <= B, the FP32 r^2 of a
// pair near the cutoff r_c is within 2^-24 (17.3 B r_c + 6.5 r_c^2) of the FP64
// one; pairs inside twice that band are re-decided (and evaluated) from the FP64
// positions, so the pair set is the FP64 one.  B = sum of the cell rows' norms +
// skin/2 for a fully periodic system (frame positions stay within the cell plus
// the allowed drift); systems with an open axis always take the FP64 test.
//
// Pruning (prune_skin p, 0 < p < skin).  Each slot's list is partitioned in
// place: the entries within r_c(ab) + p of the slot at the pruning (FP64 test)
// form a front part, in their list order, and the force kernel evaluates only
// that part.  The same bound with p for the skin and the pruning's cell and
// positions for the build's keeps a pair left out of the front part outside its
// cutoff: a system is pruned again, before the next force evaluation, when
// 2 max|u'| + (cutoff + p) e' > p (u', e' the drift and deformation since the
// pruning), and after every rebuild.  The pairs inside the cutoff are those of
// the whole list; the order in which they are summed changes (the partition
// keeps the front part's order, but a re-pruning partitions the list as the
// last one left it), so results equal the whole list's to FP64 rounding.
#include "tsb_ljhvp.cuh"
#include "tsb_pair.cuh"
#include "tsb_search.cuh"
#include "tsb_sysreduce.cuh"

namespace tsb {

constexpr int kVlBlock = 256;
constexpr int kVlSmemSys = 16;  // systems of a force block whose shifts sit in shared memory

struct VlWork {
  BinData b;           // bins of the last rebuild (sys_of / sys_lo / sys_hi persist)
  double4 *ref;        // [N] w0 at the atom's last build
  int32_t *rwrap;      // [3N] W at the last build
  double *rinv;        // [9S] C0^-1 (rows), or the identity without a fractional frame
  int32_t *rframe;     // [S] the build had a fractional frame
  double *rslack;      // [S] skin / 2 when every axis is periodic (bound on the drift
                       // of a frame position from its affine image), else -1
  double *fdef;        // [9S] F = C0^-1 C of this call
  double *dmax;        // [S] allowed non-affine drift for this call
  int32_t *sys_exp;    // [S] rebuild this system
  int32_t *sys_built;  // [S]
  int32_t *perm;       // [N] atom of each slot (identity until a system is built)
  int32_t *ecount;     // [S] atoms to rebuild per system
  int64_t *eoff;       // [S+1] their exclusive prefix (work list of the build)
  double4 *wpos;       // [N] current frame positions by slot, species in the high word
  float4 *wpos32;      // [N] the same in FP32, species bits in .w
  float *svf;          // [81 S] FP32 shift vectors
  float *band;         // [S] FP32 decision band of r^2 (+inf: always FP64)
  double *sv;          // [81 S] S C per image code
  SysGeom *cur;        // [S] start / count / vol of the current cells
  double *e_half;      // [N]
  double *vir_half;    // [6N]
  double *part;        // [7 S chunks]
  int chunks;
  // pruning (see the top of this file)
  double *pinv;        // [9S] inverse of the cell at the last pruning (rows), or identity
  double *pfdef;       // [9S] F' = pinv C of this call
  double *pdmax;       // [S] allowed drift since the pruning for this call
  int32_t *pexp;       // [S] prune this system before the next force evaluation
  double4 *pref;       // [N] frame position of each atom at the last pruning
  int32_t *pcnt;       // [N] entries in the front part of each slot's list
};

static void carve_vl(Carver &c, VlWork &w, int64_t n, int64_t ns) {
  w.sys_built = c.take<int32_t>(ns);
  w.sys_exp = c.take<int32_t>(ns);
  carve_bins(c, w.b, n, ns);
  w.ref = c.take<double4>(n);
  w.rwrap = c.take<int32_t>(3 * n);
  w.rinv = c.take<double>(9 * ns);
  w.rframe = c.take<int32_t>(ns);
  w.rslack = c.take<double>(ns);
  w.fdef = c.take<double>(9 * ns);
  w.dmax = c.take<double>(ns);
  w.perm = c.take<int32_t>(n);
  w.ecount = c.take<int32_t>(ns);
  w.eoff = c.take<int64_t>(ns + 1);
  w.wpos = c.take<double4>(n);
  w.wpos32 = c.take<float4>(n);
  w.svf = c.take<float>(81 * ns);
  w.band = c.take<float>(ns);
  w.sv = c.take<double>(81 * ns);
  w.cur = c.take<SysGeom>(ns);
  w.e_half = c.take<double>(n);
  w.vir_half = c.take<double>(6 * n);
  w.chunks = reduce_chunks(n, ns);
  w.part = w.chunks > 1 ? c.take<double>(7 * ns * w.chunks) : nullptr;
  w.pinv = c.take<double>(9 * ns);
  w.pfdef = c.take<double>(9 * ns);
  w.pdmax = c.take<double>(ns);
  w.pexp = c.take<int32_t>(ns);
  w.pref = c.take<double4>(n);
  w.pcnt = c.take<int32_t>(n);
}

// per system: deformation F = C0^-1 C since the build -> allowed drift (or expiry)
// (and, with pruning, F' = C_p^-1 C since the pruning -> allowed drift, or a
// pending pruning; a pending pruning is cleared only by the pruning itself)
template <class P>
__global__ void k_vl_sys_check(const P *cell_row, const uint8_t *active, int64_t ns,
                               double cutoff, double skin, const double *rinv,
                               const int32_t *rframe, const int32_t *built, double *fdef,
                               double *dmax, int32_t *sys_exp, int32_t *flags, double prune,
                               const double *pinv, double *pfdef, double *pdmax,
                               int32_t *pexp) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  if (active && !active[s]) {
    dmax[s] = INFINITY;
    sys_exp[s] = 0;
    pdmax[s] = INFINITY;
    return;
  }
  if (!built[s]) {
    dmax[s] = -1.0;
    sys_exp[s] = 1;
    flags[0] = 1;
    pdmax[s] = -1.0;
    return;
  }
  if (prune > 0.0) {
    double ep2 = 0.0;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        double f = r == c ? 1.0 : 0.0;
        if (rframe[s]) {
          f = 0.0;
          for (int k = 0; k < 3; ++k)
            f += pinv[9 * s + 3 * r + k] * (double)cell_row[9 * s + 3 * k + c];
        }
        pfdef[9 * s + 3 * r + c] = f;
        const double d = f - (r == c ? 1.0 : 0.0);
        ep2 += d * d;
      }
    const double ep = sqrt(ep2);
    const double pd = ep < 1.0 ? 0.5 * (prune - (cutoff + prune) * ep) : -1.0;
    pdmax[s] = pd;
    if (!(pd >= 0.0)) pexp[s] = 1;
  }
  double F[9];
  double e2 = 0.0;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double f = r == c ? 1.0 : 0.0;
      if (rframe[s]) {
        f = 0.0;
        for (int k = 0; k < 3; ++k) f += rinv[9 * s + 3 * r + k] * (double)cell_row[9 * s + 3 * k + c];
      }
      F[3 * r + c] = f;
      const double d = f - (r == c ? 1.0 : 0.0);
      e2 += d * d;
    }
  for (int k = 0; k < 9; ++k) fdef[9 * s + k] = F[k];
  const double e = sqrt(e2);
  const double d = e < 1.0 ? 0.5 * (skin - (cutoff + skin) * e) : -1.0;
  dmax[s] = d;
  sys_exp[s] = d < 0.0;
  if (d < 0.0) flags[0] = 1;
}

// per atom: non-affine drift u_i = w_i - w0_i F against the system's allowance
// (and, with pruning, u'_i = w_i - w_p,i F' against the pruning's allowance)
template <class P>
__global__ void k_vl_atom_check(const P *pos, const P *cell_row, const int64_t *sys,
                                int64_t n, const int32_t *rwrap, const double4 *ref,
                                const double *fdef, const double *dmax, int32_t *sys_exp,
                                int32_t *flags, double prune, const double4 *pref,
                                const double *pfdef, const double *pdmax, int32_t *pexp) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = sys[i];
  const double dm = dmax[s];
  if (!(dm >= 0.0) || isinf(dm)) return;  // expired already, or inactive
  const P *C = cell_row + 9 * s;
  const double *F = fdef + 9 * s;
  const int W0 = rwrap[3 * i], W1 = rwrap[3 * i + 1], W2 = rwrap[3 * i + 2];
  const double4 r = ref[i];
  double w[3];
  double d2 = 0.0;
  for (int m = 0; m < 3; ++m) {
    w[m] = (double)pos[3 * i + m] -
           (W0 * (double)C[m] + W1 * (double)C[3 + m] + W2 * (double)C[6 + m]);
    const double d = w[m] - (r.x * F[m] + r.y * F[3 + m] + r.z * F[6 + m]);
    d2 += d * d;
  }
  if (d2 > dm * dm) {
    sys_exp[s] = 1;
    flags[0] = 1;
  }
  if (prune > 0.0) {
    const double pd = pdmax[s];
    if (!(pd >= 0.0) || isinf(pd)) return;  // pending already, or inactive
    const double *G = pfdef + 9 * s;
    const double4 q = pref[i];
    double e2 = 0.0;
    for (int m = 0; m < 3; ++m) {
      const double d = w[m] - (q.x * G[m] + q.y * G[3 + m] + q.z * G[6 + m]);
      e2 += d * d;
    }
    if (e2 > pd * pd) pexp[s] = 1;
  }
}

__global__ void k_vl_iota(int32_t *perm, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) perm[i] = (int32_t)i;
}

// atoms of expired systems, for the work list of the build
__global__ void k_vl_exp_counts(const int32_t *sys_exp, const int64_t *lo, const int64_t *hi,
                                int64_t ns, int32_t *ecount) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < ns) ecount[s] = sys_exp[s] ? (int32_t)(hi[s] - lo[s]) : 0;
}

// List search for the atoms of expired systems over fresh bins (cutoff + skin),
// one warp per atom.  Work item t (< eoff[ns]) is atom t - eoff[s] of system s,
// the last system with eoff[s] <= t (bisection; empty systems are skipped); a
// fixed grid of warps strides over the items.  The atom's search window is cut
// into spans: a row of bins (fixed x and y bin) within one periodic image along
// z is a contiguous run of candidates in bin order.  Each lane takes one span
// (32 at a time) and the warp steps through candidate t of every span together,
// two steps per iteration, so the loads of all spans are in flight at once
// instead of one span after another.  Hits are compacted with a ballot, so the
// list order (step, span) is fixed and the writes of a step are coalesced.  A
// rebuilt system's slots are its fresh bin order, so a candidate's bin-order
// index is its slot.
__global__ void __launch_bounds__(256, 4)
    k_vl_build(BinData b, int64_t n, int64_t ns, double rcs2, const int64_t *eoff,
               uint32_t *list, int32_t *cnt, int max_nb, int32_t *flags, int32_t *perm,
               double4 *ref, int32_t *rwrap) {
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  const int64_t n_work = eoff[ns];
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < n_work;
       t += warps) {
    int64_t a = 0, z = ns - 1;
    while (a < z) {
      const int64_t m = (a + z + 1) >> 1;
      if (eoff[m] <= t) a = m; else z = m - 1;
    }
    const int64_t s = a;
    const int64_t p = b.sys_lo[s] + (t - eoff[s]);
    const double4 w = b.spos[p];
    const int i = tag_atom(w.w);
    const SysGeom &G = b.geom[s];
    double u[3];
    frame_coords(G, w.x, w.y, w.z, u);
    int lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
      double f0 = floor((u[k] - G.h[k] - G.org[k]) * G.scale[k]);
      double f1 = floor((u[k] + G.h[k] - G.org[k]) * G.scale[k]);
      if (!G.per[k]) {
        f0 = fmax(f0, 0.0);
        f1 = fmin(f1, (double)(G.nb[k] - 1));
      }
      lo[k] = (int)f0;
      hi[k] = (int)f1;
    }
    const int nb0 = G.nb[0], nb1 = G.nb[1], nb2 = G.nb[2];
    const int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1;
    const int iz_lo = G.per[2] ? floordiv_dev(lo[2], nb2) : 0;
    const int nzs = G.per[2] ? floordiv_dev(hi[2], nb2) - iz_lo + 1 : (hi[2] >= lo[2]);
    const int n_spans = nx > 0 && ny > 0 ? nx * ny * nzs : 0;
    int c = 0;
    for (int base = 0; base < n_spans; base += 32) {
      // this lane's span: candidates q0..q1-1 with image shift (sx, sy, sz)
      const int k = base + lane;
      int64_t q0 = 0, q1 = 0;
      double sx = 0.0, sy = 0.0, sz = 0.0;
      uint32_t code = 0;
      bool in_range = true, zero_shift = false;
      if (k < n_spans) {
        const int zs = k % nzs, r = k / nzs;
        const int cx = lo[0] + r / ny, cy = lo[1] + r % ny;
        const int ix = G.per[0] ? floordiv_dev(cx, nb0) : 0;
        const int iy = G.per[1] ? floordiv_dev(cy, nb1) : 0;
        const int iz = iz_lo + zs;
        const int bx = cx - ix * nb0, by = cy - iy * nb1;
        const int bz0 = max(lo[2], iz * nb2) - iz * nb2;
        const int bz1 = min(hi[2], iz * nb2 + nb2 - 1) - iz * nb2;
        const int row = G.bin_base + (bx * nb1 + by) * nb2;
        q0 = b.bin_start[row + bz0];
        q1 = b.bin_start[row + bz1 + 1];
        sx = ix * G.cell[0] + iy * G.cell[3] + iz * G.cell[6];
        sy = ix * G.cell[1] + iy * G.cell[4] + iz * G.cell[7];
        sz = ix * G.cell[2] + iy * G.cell[5] + iz * G.cell[8];
        zero_shift = (ix | iy | iz) == 0;
        in_range = ix >= -1 && ix <= 1 && iy >= -1 && iy <= 1 && iz >= -1 && iz <= 1;
        code = (uint32_t)((ix + 1) * 9 + (iy + 1) * 3 + (iz + 1));
      }
      const int len = __reduce_max_sync(0xffffffffu, (unsigned)(q1 - q0));
      // test candidate q: a hit beyond the first images means a cell narrower
      // than cutoff + skin (the build fails)
#define TSB_VL_TEST(Q, O)                                                                    \
  {                                                                                          \
    bool hit = false;                                                                        \
    if ((Q) < q1) {                                                                          \
      const double dx = ((O).x + sx) - w.x;                                                  \
      const double dy = ((O).y + sy) - w.y;                                                  \
      const double dz = ((O).z + sz) - w.z;                                                  \
      hit = dx * dx + dy * dy + dz * dz < rcs2 && !((Q) == p && zero_shift);                 \
    }                                                                                        \
    if (__any_sync(0xffffffffu, hit && !in_range) && lane == 0)                              \
      atomicMax(&flags[1], 1 << 30);                                                         \
    hit = hit && in_range;                                                                   \
    const unsigned m = __ballot_sync(0xffffffffu, hit);                                      \
    if (hit) {                                                                               \
      const int kk = c + __popc(m & lt_mask);                                                \
      if (kk < max_nb) list[(size_t)kk * n + p] = ((uint32_t)(Q) << 5) | code;               \
    }                                                                                        \
    c += __popc(m);                                                                          \
  }
      for (int st = 0; st < len; st += 2) {
        const int64_t qa = q0 + st, qb = qa + 1;
        double4 oa = make_double4(0.0, 0.0, 0.0, 0.0), ob = oa;
        if (qa < q1) oa = b.spos[qa];
        if (qb < q1) ob = b.spos[qb];
        TSB_VL_TEST(qa, oa)
        TSB_VL_TEST(qb, ob)
      }
#undef TSB_VL_TEST
    }
    if (lane == 0) {
      cnt[p] = c < max_nb ? c : max_nb;
      if (c > max_nb) atomicMax(&flags[1], c);
      perm[p] = i;
      const double4 w0 = b.wpos[i];
      ref[i] = make_double4(w0.x, w0.y, w0.z, 0.0);
      rwrap[3 * i] = b.wrap[3 * i];
      rwrap[3 * i + 1] = b.wrap[3 * i + 1];
      rwrap[3 * i + 2] = b.wrap[3 * i + 2];
    }
  }
}

// per rebuilt system: record C0^-1 (the transpose of the frame matrix T)
__global__ void k_vl_sys_built(const SysGeom *g, int64_t ns, int32_t *sys_exp, int32_t *built,
                               double skin, double *rinv, int32_t *rframe, double *rslack,
                               int32_t *pexp) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns || !sys_exp[s]) return;
  const SysGeom &G = g[s];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) rinv[9 * s + 3 * r + c] = G.active ? G.T[3 * c + r] : (r == c);
  rframe[s] = G.active;
  rslack[s] = G.active && G.per[0] && G.per[1] && G.per[2] ? 0.5 * skin : -1.0;
  built[s] = 1;
  sys_exp[s] = 0;
  pexp[s] = 1;  // a new list: its front part is formed before the next forces
}

// per system for the force call: shift vectors (one thread per system and image
// code), and from the code-0 thread the FP32 band, start / count and volume
template <class P>
__global__ void k_vl_sys_geom(const P *cell_row, int64_t ns, const int64_t *lo,
                              const int64_t *hi, const double *rslack, double cutoff,
                              double *sv, float *svf, float *band, SysGeom *cur) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 27 * ns) return;
  const int64_t s = t / 27;
  const int code = (int)(t - 27 * s);
  double C[9];
  for (int k = 0; k < 9; ++k) C[k] = (double)cell_row[9 * s + k];
  const int sx = code / 9 - 1, sy = (code / 3) % 3 - 1, sz = code % 3 - 1;
  for (int m = 0; m < 3; ++m) {
    const double v = sx * C[m] + sy * C[3 + m] + sz * C[6 + m];
    sv[81 * s + 3 * code + m] = v;
    svf[81 * s + 3 * code + m] = (float)v;
  }
  if (code) return;
  double bsum = 0.0;
  for (int k = 0; k < 3; ++k)
    bsum += sqrt(C[3 * k] * C[3 * k] + C[3 * k + 1] * C[3 * k + 1] + C[3 * k + 2] * C[3 * k + 2]);
  // |frame position| <= sum of row norms + drift, |shift| <= sum of row norms:
  // FP32 rounding of the inputs, the difference, the shift sum and the square
  // sum puts r^2 within 2^-24 (17.3 B r + 6.5 r^2) of the FP64 value near
  // r = r_c, plus 2^-24 r_c^2 for the rounding of r_c^2; the band is twice it
  const double B = bsum + rslack[s];
  band[s] = rslack[s] >= 0.0
                ? (float)(2.0 * ldexp(1.0, -24) * (17.4 * B * cutoff + 7.6 * cutoff * cutoff))
                : INFINITY;
  SysGeom &G = cur[s];
  G.start = lo[s];
  G.count = (int32_t)(hi[s] - lo[s]);
  G.vol = fabs(C[0] * (C[4] * C[8] - C[5] * C[7]) - C[1] * (C[3] * C[8] - C[5] * C[6]) +
               C[2] * (C[3] * C[7] - C[4] * C[6]));
}

// current positions -> frame of the atom's build (FP64) by slot, species in .w
template <class P>
__global__ void k_vl_frame(const P *pos, const P *cell_row, const int64_t *sys,
                           const int32_t *species, int64_t n, const int32_t *perm,
                           const int32_t *rwrap, double4 *wpos, float4 *wpos32) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int64_t i = perm[p];
  const P *C = cell_row + 9 * sys[i];
  const int W0 = rwrap[3 * i], W1 = rwrap[3 * i + 1], W2 = rwrap[3 * i + 2];
  double w[3];
  for (int m = 0; m < 3; ++m)
    w[m] = (double)pos[3 * i + m] -
           (W0 * (double)C[m] + W1 * (double)C[3 + m] + W2 * (double)C[6 + m]);
  const unsigned long long hi = species ? (unsigned long long)(uint32_t)species[i] : 0ull;
  wpos[p] = make_double4(w[0], w[1], w[2], __longlong_as_double((long long)(hi << 32)));
  wpos32[p] = make_float4((float)w[0], (float)w[1], (float)w[2], __int_as_float((int)hi));
}

// Pruning of the systems marked in pexp: each slot's list is partitioned in
// place (stable for the front part) into the entries within r_c(ab) + prune of
// the slot's current frame position and the rest; the front count and the
// atom's position at the pruning are recorded.  FP64 distances.
__global__ void k_vl_prune(const double4 *__restrict__ wpos, uint32_t *list,
                           const int32_t *__restrict__ cnt, int64_t n,
                           const int32_t *__restrict__ perm, const int64_t *__restrict__ sys,
                           const double *__restrict__ sv, const double *__restrict__ table,
                           int pot, int nsp, double cutoff, double prune,
                           const int32_t *__restrict__ pexp, const uint8_t *active,
                           int32_t *pcnt, double4 *pref) {
  __shared__ double reach2[kMaxSpecies * kMaxSpecies];
  for (int k = threadIdx.x; k < nsp * nsp; k += blockDim.x) {
    const double r = sqrt(pair_rc2(pot, table + 5 * k, cutoff)) + prune;
    reach2[k] = r * r * (1.0 + 1e-10);
  }
  __syncthreads();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int64_t i = perm[p];
  const int64_t s = sys[i];
  if (!pexp[s] || (active && !active[s])) return;
  const double4 wi = wpos[p];
  const int si = min(max(tag_species(wi.w), 0), nsp - 1);
  const double *svs = sv + 81 * s;
  const int c = cnt[p];
  int front = 0;
  for (int k = 0; k < c; ++k) {
    const uint32_t e = list[(size_t)k * n + p];
    const double4 wj = wpos[e >> 5];
    const int code = (int)(e & 31u);
    const double dx = wj.x - wi.x + svs[3 * code];
    const double dy = wj.y - wi.y + svs[3 * code + 1];
    const double dz = wj.z - wi.z + svs[3 * code + 2];
    const int sj = min(max(tag_species(wj.w), 0), nsp - 1);
    if (dx * dx + dy * dy + dz * dz < reach2[si * nsp + sj]) {
      if (front != k) {
        list[(size_t)k * n + p] = list[(size_t)front * n + p];
        list[(size_t)front * n + p] = e;
      }
      ++front;
    }
  }
  pcnt[p] = front;
  pref[i] = make_double4(wi.x, wi.y, wi.z, 0.0);
}

// per pruned system: the cell's inverse at the pruning, and the mark cleared
template <class P>
__global__ void k_vl_sys_pruned(const P *cell_row, int64_t ns, const int32_t *rframe,
                                const uint8_t *active, double *pinv, int32_t *pexp) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns || !pexp[s] || (active && !active[s])) return;
  double C[9];
  for (int k = 0; k < 9; ++k) C[k] = (double)cell_row[9 * s + k];
  double inv[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (rframe[s]) {
    const double d = C[0] * (C[4] * C[8] - C[5] * C[7]) - C[1] * (C[3] * C[8] - C[5] * C[6]) +
                     C[2] * (C[3] * C[7] - C[4] * C[6]);
    const double id = 1.0 / d;
    inv[0] = (C[4] * C[8] - C[5] * C[7]) * id;
    inv[1] = (C[2] * C[7] - C[1] * C[8]) * id;
    inv[2] = (C[1] * C[5] - C[2] * C[4]) * id;
    inv[3] = (C[5] * C[6] - C[3] * C[8]) * id;
    inv[4] = (C[0] * C[8] - C[2] * C[6]) * id;
    inv[5] = (C[2] * C[3] - C[0] * C[5]) * id;
    inv[6] = (C[3] * C[7] - C[4] * C[6]) * id;
    inv[7] = (C[1] * C[6] - C[0] * C[7]) * id;
    inv[8] = (C[0] * C[4] - C[1] * C[3]) * id;
  }
  for (int k = 0; k < 9; ++k) pinv[9 * s + k] = inv[k];
  pexp[s] = 0;
}

__device__ __forceinline__ int vl_species(double w) { return tag_species(w); }
__device__ __forceinline__ int vl_species(float w) { return __float_as_int(w); }

template <int POT, class R, class P, int LANES>
__global__ void __launch_bounds__(kVlBlock)
    k_vl_forces(const double4 *__restrict__ wpos, const float4 *__restrict__ wpos32,
                const uint32_t *__restrict__ list, const int32_t *__restrict__ cnt, int64_t n,
                const int32_t *__restrict__ perm, const int64_t *__restrict__ sys,
                const double *__restrict__ sv, const float *__restrict__ svf,
                const float *__restrict__ band, const double *__restrict__ table,
                int ns_species, double cutoff, int flags, P *forces, P *energies, P *stresses,
                const SysGeom *__restrict__ cur, double *e_half, double *vir_half,
                const uint8_t *__restrict__ active) {
  constexpr bool F32 = sizeof(R) == 4;
  using Pos4 = std::conditional_t<F32, float4, double4>;
  using Sh = std::conditional_t<F32, float, double>;
  __shared__ PairPrm<R> prm[kMaxSpecies * kMaxSpecies];
  __shared__ double prc2[kMaxSpecies * kMaxSpecies];
  __shared__ float prc2f[kMaxSpecies * kMaxSpecies];
  __shared__ Sh ssv[kVlSmemSys * 81];
  __shared__ float sband[kVlSmemSys];
  for (int k = threadIdx.x; k < ns_species * ns_species; k += blockDim.x) {
    prm[k] = make_prm<R>(POT, table + 5 * k, cutoff);
    if constexpr (F32) prm_fast_extra(POT, table + 5 * k, prm[k]);
    prc2[k] = pair_rc2(POT, table + 5 * k, cutoff);
    prc2f[k] = (float)prc2[k];
  }
  // slots are grouped by system, so a block spans systems s_lo..s_hi; the shift
  // vectors (FP32 ones and the bands on the FP32 path) of the first kVlSmemSys of
  // them are staged in shared memory
  const Sh *shifts;
  const Pos4 *__restrict__ wg;
  if constexpr (F32) {
    shifts = svf;
    wg = wpos32;
  } else {
    shifts = sv;
    wg = wpos;
  }
  // LANES lanes per slot (small batches: more threads in flight; each lane takes
  // every LANES-th entry and a fixed butterfly sums the lanes), else one thread
  const int64_t p0 = (int64_t)blockIdx.x * (blockDim.x / LANES);
  const int64_t s_lo = sys[perm[p0]];
  const int64_t s_hi = sys[perm[min(p0 + (int64_t)(blockDim.x / LANES), n) - 1]];
  const int n_st = (int)min(s_hi - s_lo + 1, (int64_t)kVlSmemSys);
  for (int k = threadIdx.x; k < 81 * n_st; k += blockDim.x) ssv[k] = shifts[81 * s_lo + k];
  if constexpr (F32)
    for (int k = threadIdx.x; k < n_st; k += blockDim.x) sband[k] = band[s_lo + k];
  __syncthreads();
  const int64_t p = p0 + threadIdx.x / LANES;
  const int lane = threadIdx.x % LANES;
  // a group whose slot is past the end or inactive still takes part in the
  // lane sums (with no entries) and leaves before writing
  bool valid = p < n;
  int64_t i = 0, s = s_lo;
  if (valid) {
    i = perm[p];
    s = sys[i];
    valid = !active || active[s];
  }
  if (LANES == 1 && !valid) return;
  const Pos4 wi = wg[valid ? p : p0];
  const int si = min(max(vl_species(wi.w), 0), ns_species - 1);
  const PairPrm<R> *row = prm + si * ns_species;
  const double *rc2row = prc2 + si * ns_species;
  const float *rc2frow = prc2f + si * ns_species;
  const bool staged = s - s_lo < n_st;
  const Sh *svs = staged ? ssv + 81 * (s - s_lo) : shifts + 81 * s;
  float bnd = 0.f;
  if constexpr (F32) bnd = staged ? sband[s - s_lo] : band[s];
  const bool want_vir = flags & (TSB_OUT_STRESS | TSB_OUT_STRESSES);
  const int c = valid ? cnt[p] : 0;
  double fx = 0.0, fy = 0.0, fz = 0.0, ei = 0.0;
  double vxx = 0, vyy = 0, vzz = 0, vyz = 0, vxz = 0, vxy = 0;
  // one entry E with neighbour frame position WJ.  FP64 path: FP64 displacement
  // and cutoff test.  FP32 path: FP32 displacement and test, except within the
  // band around the cutoff, where both come from the FP64 positions.  Pair
  // function in R, FP64 accumulation.
#define TSB_VLPAIR(E, WJ)                                                                    \
  {                                                                                          \
    const int code = (int)((E) & 31u);                                                       \
    const int sj = min(max(vl_species((WJ).w), 0), ns_species - 1);                         \
    double dx, dy, dz;                                                                       \
    bool in_;                                                                                \
    R r2;                                                                                    \
    if constexpr (F32) {                                                                     \
      const float ax = (WJ).x - wi.x + svs[3 * code];                                        \
      const float ay = (WJ).y - wi.y + svs[3 * code + 1];                                    \
      const float az = (WJ).z - wi.z + svs[3 * code + 2];                                    \
      r2 = ax * ax + ay * ay + az * az;                                                      \
      in_ = r2 < rc2frow[sj];                                                                \
      dx = ax;                                                                               \
      dy = ay;                                                                               \
      dz = az;                                                                               \
      if (!(fabsf(r2 - rc2frow[sj]) >= bnd)) {                                               \
        const double4 di = wpos[p], dj = wpos[(E) >> 5];                                     \
        const double *sd = sv + 81 * s + 3 * code;                                           \
        dx = dj.x - di.x + sd[0];                                                            \
        dy = dj.y - di.y + sd[1];                                                            \
        dz = dj.z - di.z + sd[2];                                                            \
        const double d2 = dx * dx + dy * dy + dz * dz;                                       \
        in_ = d2 < rc2row[sj];                                                               \
        r2 = (float)d2;                                                                      \
      }                                                                                      \
    } else {                                                                                 \
      dx = (WJ).x - wi.x + svs[3 * code];                                                    \
      dy = (WJ).y - wi.y + svs[3 * code + 1];                                                \
      dz = (WJ).z - wi.z + svs[3 * code + 2];                                                \
      r2 = dx * dx + dy * dy + dz * dz;                                                      \
      in_ = r2 < rc2row[sj];                                                                 \
    }                                                                                        \
    if (F32 || in_) {                                                                        \
      R ep, fr;                                                                              \
      if constexpr (F32) {                                                                   \
        pair_eval_fast<POT>(row[sj], r2, ep, fr);                                            \
        fr = in_ ? fr : 0.f;                                                                 \
        ep = in_ ? ep : 0.f;                                                                 \
      } else {                                                                               \
        pair_eval<POT, R>(row[sj], r2, ep, fr);                                              \
      }                                                                                      \
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
  const uint32_t *lp = list + p;
  if constexpr (LANES > 1) {
    for (int k = lane; k < c; k += LANES) {
      const uint32_t e = lp[(size_t)k * n];
      const Pos4 wj = wg[e >> 5];
      TSB_VLPAIR(e, wj)
    }
    fx = group_sum<LANES>(fx);
    fy = group_sum<LANES>(fy);
    fz = group_sum<LANES>(fz);
    ei = group_sum<LANES>(ei);
    if (want_vir) {
      vxx = group_sum<LANES>(vxx);
      vyy = group_sum<LANES>(vyy);
      vzz = group_sum<LANES>(vzz);
      vyz = group_sum<LANES>(vyz);
      vxz = group_sum<LANES>(vxz);
      vxy = group_sum<LANES>(vxy);
    }
    if (!valid || lane != 0) return;
  } else {
  // four entries per iteration; the next four list words are loaded one
  // iteration ahead so their DRAM latency overlaps the current gathers and math
  int k = 0;
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
    const Pos4 w0 = wg[e0 >> 5], w1 = wg[e1 >> 5];
    const Pos4 w2 = wg[e2 >> 5], w3 = wg[e3 >> 5];
    TSB_VLPAIR(e0, w0)
    TSB_VLPAIR(e1, w1)
    TSB_VLPAIR(e2, w2)
    TSB_VLPAIR(e3, w3)
    e0 = f0;
    e1 = f1;
    e2 = f2;
    e3 = f3;
  }
  for (; k < c; ++k) {
    const uint32_t e = lp[(size_t)k * n];
    const Pos4 wj = wg[e >> 5];
    TSB_VLPAIR(e, wj)
  }
  }
#undef TSB_VLPAIR
  if (flags & TSB_OUT_FORCES) {
    forces[3 * i] = (P)fx;
    forces[3 * i + 1] = (P)fy;
    forces[3 * i + 2] = (P)fz;
  }
  // per-atom energies and stresses as the per-call search path writes them
  if (flags & TSB_OUT_ENERGIES) energies[i] = (P)ei;
  if (flags & TSB_OUT_STRESSES) {
    const double cf = -0.5 / cur[s].vol;
    P *o = stresses + 9 * i;
    o[0] = (P)(cf * vxx); o[1] = (P)(cf * vxy); o[2] = (P)(cf * vxz);
    o[3] = (P)(cf * vxy); o[4] = (P)(cf * vyy); o[5] = (P)(cf * vyz);
    o[6] = (P)(cf * vxz); o[7] = (P)(cf * vyz); o[8] = (P)(cf * vzz);
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

template <class P>
static int vl_check(const P *pos, const P *cell, const int64_t *sys, const uint8_t *active,
                    int64_t n, int64_t ns, double cutoff, double skin, double prune,
                    int32_t *flags, VlWork &w, cudaStream_t st) {
  cudaMemsetAsync(flags, 0, 2 * sizeof(int32_t), st);
  k_vl_sys_check<P><<<grid_for(ns), kBlock, 0, st>>>(cell, active, ns, cutoff, skin, w.rinv,
                                                     w.rframe, w.sys_built, w.fdef, w.dmax,
                                                     w.sys_exp, flags, prune, w.pinv, w.pfdef,
                                                     w.pdmax, w.pexp);
  k_vl_atom_check<P><<<grid_for(n), kBlock, 0, st>>>(pos, cell, sys, n, w.rwrap, w.ref, w.fdef,
                                                     w.dmax, w.sys_exp, flags, prune, w.pref,
                                                     w.pfdef, w.pdmax, w.pexp);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

template <class P>
static int vl_build(const P *pos, const P *cell, const uint8_t *pbc, const int64_t *sys,
                    const int32_t *species, int64_t n, int64_t ns, double cutoff, double skin,
                    uint32_t *list, int32_t *counts, int max_nb, int64_t max_sys,
                    int32_t *flags, VlWork &w, cudaStream_t st) {
  cudaMemsetAsync(flags + 1, 0, sizeof(int32_t), st);
  const double rcs = cutoff + skin;
  // batches of small systems rebin only the expired systems, one block each
  if (max_sys > 0 && max_sys <= kSysBinMaxAtoms)
    TSB_TRY(prepare_bins_sys<P>(pos, cell, pbc, sys, n, ns, rcs, w.b, st, species, w.sys_exp));
  else
    TSB_TRY(prepare_bins<P>(pos, cell, pbc, sys, n, ns, rcs, w.b, st, species));
  k_vl_exp_counts<<<grid_for(ns), kBlock, 0, st>>>(w.sys_exp, w.b.sys_lo, w.b.sys_hi, ns,
                                                   w.ecount);
  TSB_TRY(exclusive_scan(w.ecount, w.eoff, ns, w.b.scan_tmp, st));
  // a fixed grid of warps (8 blocks of 256 threads per SM) strides over the work
  int dev = 0, n_sm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  k_vl_build<<<(unsigned)(n_sm * 8), 256, 0, st>>>(w.b, n, ns, rcs * rcs, w.eoff, list, counts,
                                                    max_nb, flags, w.perm, w.ref, w.rwrap);
  k_vl_sys_built<<<grid_for(ns), kBlock, 0, st>>>(w.b.geom, ns, w.sys_exp, w.sys_built, skin,
                                                  w.rinv, w.rframe, w.rslack, w.pexp);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

template <int POT, class R, class P>
static void vl_launch(VlWork &w, const uint32_t *list, const int32_t *counts, int64_t n,
                      const int64_t *sys, const double *table, int nsp, double cutoff,
                      int flags, P *forces, P *energies, P *stresses, const uint8_t *active,
                      cudaStream_t st) {
  if (n <= kGroupSearchMaxAtoms)
    k_vl_forces<POT, R, P, kSearchGroup><<<grid_for(kSearchGroup * n, kVlBlock), kVlBlock, 0,
                                            st>>>(
        w.wpos, w.wpos32, list, counts, n, w.perm, sys, w.sv, w.svf, w.band, table, nsp,
        cutoff, flags, forces, energies, stresses, w.cur, w.e_half, w.vir_half, active);
  else
    k_vl_forces<POT, R, P, 1><<<grid_for(n, kVlBlock), kVlBlock, 0, st>>>(
        w.wpos, w.wpos32, list, counts, n, w.perm, sys, w.sv, w.svf, w.band, table, nsp,
        cutoff, flags, forces, energies, stresses, w.cur, w.e_half, w.vir_half, active);
}

template <class P>
static int vl_forces(int pot, const double *table, int nsp, const int32_t *species,
                     uint32_t *list, const int32_t *counts, const P *pos, const P *cell,
                     const int64_t *sys, const uint8_t *active, int64_t n, int64_t ns,
                     double cutoff, double prune, int flags, P *energy, P *forces, P *stress,
                     P *energies, P *stresses, VlWork &w, cudaStream_t st) {
  k_vl_sys_geom<P><<<grid_for(27 * ns), kBlock, 0, st>>>(cell, ns, w.b.sys_lo, w.b.sys_hi,
                                                         w.rslack, cutoff, w.sv, w.svf, w.band,
                                                         w.cur);
  k_vl_frame<P><<<grid_for(n), kBlock, 0, st>>>(pos, cell, sys, species, n, w.perm, w.rwrap,
                                                w.wpos, w.wpos32);
  if (prune > 0.0) {
    // systems marked by the check or rebuilt since their last pruning form their
    // front parts; the force kernel then reads the front counts
    k_vl_prune<<<grid_for(n), kBlock, 0, st>>>(w.wpos, list, counts, n, w.perm, sys, w.sv,
                                               table, pot, nsp, cutoff, prune, w.pexp, active,
                                               w.pcnt, w.pref);
    k_vl_sys_pruned<P><<<grid_for(ns), kBlock, 0, st>>>(cell, ns, w.rframe, active, w.pinv,
                                                        w.pexp);
    counts = w.pcnt;
  }
  const bool f64 = flags & TSB_MATH_FP64;
#define TSB_VLL(POT)                                                                        \
  if (f64)                                                                                  \
    vl_launch<POT, double, P>(w, list, counts, n, sys, table, nsp, cutoff, flags, forces,  \
                              energies, stresses, active, st);                              \
  else                                                                                      \
    vl_launch<POT, float, P>(w, list, counts, n, sys, table, nsp, cutoff, flags, forces,   \
                             energies, stresses, active, st);
  if (pot == TSB_POT_LJ) {
    TSB_VLL(TSB_POT_LJ)
  } else if (pot == TSB_POT_MORSE) {
    TSB_VLL(TSB_POT_MORSE)
  } else {
    TSB_VLL(TSB_POT_SOFT)
  }
#undef TSB_VLL
  k_sys_reduce<P><<<dim3((unsigned)ns, (unsigned)w.chunks), kBlock, 0, st>>>(
      w.cur, w.e_half, w.vir_half, flags, energy, stress, active, w.chunks, w.part);
  if (w.chunks > 1)
    k_sys_final<P><<<grid_for(ns), kBlock, 0, st>>>(w.cur, w.part, ns, w.chunks, flags, energy,
                                                     stress, active);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

// Lennard-Jones Hessian-vector product over the lists (the adjoint's HVP with the
// lists in place of the per-call search): lam_q -= coef (H v) per atom and the
// per-atom parameter partials, LANES lanes per slot over its entries (fixed-order
// butterfly reduction).  v is read in slot order (vs).
template <int LANES>
__global__ void __launch_bounds__(128)
    k_vl_lj_hvp(const double4 *__restrict__ wpos, const uint32_t *__restrict__ list,
                const int32_t *__restrict__ cnt, int64_t n, const int32_t *__restrict__ perm,
                const int64_t *__restrict__ sys, const double *__restrict__ sv,
                const double *__restrict__ table, int nsp, double cutoff,
                const double *__restrict__ vs, double coef, double *__restrict__ lam_q,
                double *__restrict__ gpart) {
  __shared__ LjHvpTable T;
  lj_hvp_table(T, table, nsp, cutoff);
  __syncthreads();
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t p = t / LANES;
  const int lane = (int)(t % LANES);
  if (p >= n) return;  // whole groups: LANES divides the block
  const int64_t i = perm[p];
  const int64_t s = sys[i];
  const double4 wi = wpos[p];
  const int si = min(max(tag_species(wi.w), 0), nsp - 1);
  const double vi0 = vs[3 * p], vi1 = vs[3 * p + 1], vi2 = vs[3 * p + 2];
  const double *svs = sv + 81 * s;
  double hx = 0, hy = 0, hz = 0;
  double gs[kAdjMaxSpecies], ge[kAdjMaxSpecies];
#pragma unroll
  for (int t2 = 0; t2 < kAdjMaxSpecies; ++t2) gs[t2] = ge[t2] = 0.0;
  const int c = cnt[p];
  for (int k = lane; k < c; k += LANES) {
    const uint32_t e = list[(size_t)k * n + p];
    const int64_t js = e >> 5;
    const int code = (int)(e & 31u);
    const double4 wj = wpos[js];
    const double dx = wj.x - wi.x + svs[3 * code];
    const double dy = wj.y - wi.y + svs[3 * code + 1];
    const double dz = wj.z - wi.z + svs[3 * code + 2];
    const int sj = min(max(tag_species(wj.w), 0), nsp - 1);
    lj_hvp_pair(T, si * nsp + sj, sj, dx, dy, dz, dx * dx + dy * dy + dz * dz, vi0, vi1, vi2,
                vs[3 * js], vs[3 * js + 1], vs[3 * js + 2], hx, hy, hz, gs, ge);
  }
  if constexpr (LANES > 1) {
    hx = group_sum<LANES>(hx);
    hy = group_sum<LANES>(hy);
    hz = group_sum<LANES>(hz);
#pragma unroll
    for (int t2 = 0; t2 < kAdjMaxSpecies; ++t2) {
      gs[t2] = group_sum<LANES>(gs[t2]);
      ge[t2] = group_sum<LANES>(ge[t2]);
    }
    if (lane != 0) return;
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

// v [N,3] by atom -> vs [N,3] by slot
__global__ void k_vl_gather3(const double *v, const int32_t *perm, int64_t n, double *vs) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < 3 * n) vs[k] = v[3 * (int64_t)perm[k / 3] + k % 3];
}

// out[s, k] += sum over the atoms of system s of part[i, k] (atom order)
__global__ void k_vl_sum_parts(const SysGeom *g, const double *part, int width, double *out) {
  const int s = blockIdx.x;
  const SysGeom &G = g[s];
  for (int k = threadIdx.x; k < width; k += blockDim.x) {
    double t = 0.0;
    for (int a = 0; a < G.count; ++a) t += part[(size_t)(G.start + a) * width + k];
    out[(size_t)s * width + k] += t;
  }
}

}  // namespace tsb

using namespace tsb;

extern "C" size_t tsb_vlist_hvp_scratch_size(int64_t n_atoms, int n_species) {
  return sizeof(double) * (size_t)n_atoms * (3 + 2 * (size_t)n_species * n_species) + 512;
}

extern "C" int tsb_vlist_lj_hvp(const double *table, int n_species, const int32_t *species,
                                const uint32_t *list, const int32_t *counts,
                                const double *positions, const double *cell_row,
                                const int64_t *system_idx, int64_t n_atoms, int64_t n_systems,
                                double cutoff, const double *v, double coef, double *lam_q,
                                double *grad_params, void *scratch, size_t scratch_bytes,
                                void *workspace, size_t workspace_bytes, void *stream) {
  if (n_species < 1 || n_species > kAdjMaxSpecies || !table || (n_species > 1 && !species) ||
      n_atoms < 1 || n_systems < 1 || !list || !counts || !positions || !cell_row ||
      !system_idx || !v || !lam_q || !grad_params || !(cutoff > 0.0))
    return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  VlWork w;
  carve_vl(c, w, n_atoms, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  const int width = 2 * n_species * n_species;
  Carver cs(scratch, scratch_bytes);
  double *vs = cs.take<double>(3 * n_atoms);
  double *part = cs.take<double>(n_atoms * width);
  if (!cs.ok || !scratch) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  k_vl_sys_geom<double><<<grid_for(27 * n_systems), kBlock, 0, st>>>(
      cell_row, n_systems, w.b.sys_lo, w.b.sys_hi, w.rslack, cutoff, w.sv, w.svf, w.band, w.cur);
  k_vl_frame<double><<<grid_for(n_atoms), kBlock, 0, st>>>(
      positions, cell_row, system_idx, species, n_atoms, w.perm, w.rwrap, w.wpos, w.wpos32);
  k_vl_gather3<<<grid_for(3 * n_atoms), kBlock, 0, st>>>(v, w.perm, n_atoms, vs);
  if (n_atoms <= kGroupSearchMaxAtoms)
    k_vl_lj_hvp<kSearchGroup><<<grid_for(kSearchGroup * n_atoms, 128), 128, 0, st>>>(
        w.wpos, list, counts, n_atoms, w.perm, system_idx, w.sv, table, n_species, cutoff, vs,
        coef, lam_q, part);
  else
    k_vl_lj_hvp<1><<<grid_for(n_atoms, 128), 128, 0, st>>>(
        w.wpos, list, counts, n_atoms, w.perm, system_idx, w.sv, table, n_species, cutoff, vs,
        coef, lam_q, part);
  k_vl_sum_parts<<<(unsigned)n_systems, 64, 0, st>>>(w.cur, part, width, grad_params);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" size_t tsb_vlist_workspace_size(int64_t n_atoms, int64_t n_systems) {
  Carver c(nullptr, (size_t)-1);
  VlWork w;
  carve_vl(c, w, n_atoms, n_systems);
  return c.off + 256;
}

extern "C" int tsb_vlist_reset(int64_t n_atoms, int64_t n_systems, void *workspace,
                               size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !workspace) return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  VlWork w;
  carve_vl(c, w, n_atoms, n_systems);
  if (!c.ok) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(w.sys_built, 0, sizeof(int32_t) * n_systems, st);
  cudaMemsetAsync(w.sys_exp, 0, sizeof(int32_t) * n_systems, st);
  cudaMemsetAsync(w.rslack, 0xff, sizeof(double) * n_systems, st);  // NaN: FP64 test
  cudaMemsetAsync(w.pexp, 0xff, sizeof(int32_t) * n_systems, st);    // nonzero: prune
  k_vl_iota<<<grid_for(n_atoms), kBlock, 0, st>>>(w.perm, n_atoms);
  TSB_CHECK_LAUNCH();
  return TSB_OK;
}

extern "C" int tsb_vlist_check(const void *positions, const void *cell_row,
                               const int64_t *system_idx, const uint8_t *sys_active,
                               int64_t n_atoms, int64_t n_systems, int dtype, double cutoff,
                               double skin, double prune_skin, int32_t *flags, void *workspace,
                               size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !positions || !cell_row || !system_idx || !flags ||
      !(cutoff > 0.0) || !(skin >= 0.0) || !(prune_skin >= 0.0))
    return TSB_ERR_INVALID_ARG;
  const double prune = prune_skin < skin ? prune_skin : 0.0;
  Carver c(workspace, workspace_bytes);
  VlWork w;
  carve_vl(c, w, n_atoms, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == TSB_F64)
    return vl_check<double>((const double *)positions, (const double *)cell_row, system_idx,
                            sys_active, n_atoms, n_systems, cutoff, skin, prune, flags, w, st);
  if (dtype == TSB_F32)
    return vl_check<float>((const float *)positions, (const float *)cell_row, system_idx,
                           sys_active, n_atoms, n_systems, cutoff, skin, prune, flags, w, st);
  return TSB_ERR_INVALID_ARG;
}

extern "C" int tsb_vlist_build(const void *positions, const void *cell_row, const uint8_t *pbc,
                               const int64_t *system_idx, const int32_t *species,
                               int64_t n_atoms, int64_t n_systems, int dtype, double cutoff,
                               double skin, uint32_t *list, int32_t *counts, int max_neighbors,
                               int64_t max_system_atoms, int32_t *flags, void *workspace,
                               size_t workspace_bytes, void *stream) {
  if (n_atoms < 1 || n_systems < 1 || !positions || !cell_row || !pbc || !system_idx ||
      !list || !counts || !flags || max_neighbors < 1 || !(cutoff > 0.0) || !(skin >= 0.0))
    return TSB_ERR_INVALID_ARG;
  if (n_atoms >= ((int64_t)1 << 27)) return TSB_ERR_UNSUPPORTED;
  Carver c(workspace, workspace_bytes);
  VlWork w;
  carve_vl(c, w, n_atoms, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == TSB_F64)
    return vl_build<double>((const double *)positions, (const double *)cell_row, pbc,
                            system_idx, species, n_atoms, n_systems, cutoff, skin, list,
                            counts, max_neighbors, max_system_atoms, flags, w, st);
  if (dtype == TSB_F32)
    return vl_build<float>((const float *)positions, (const float *)cell_row, pbc, system_idx,
                           species, n_atoms, n_systems, cutoff, skin, list, counts,
                           max_neighbors, max_system_atoms, flags, w, st);
  return TSB_ERR_INVALID_ARG;
}

extern "C" int tsb_vlist_forces(int potential, const double *table, int n_species,
                                const int32_t *species, uint32_t *list,
                                const int32_t *counts, const void *positions,
                                const void *cell_row, const int64_t *system_idx,
                                const uint8_t *sys_active, int64_t n_atoms, int64_t n_systems,
                                int dtype, double cutoff, double prune_skin, int out_flags,
                                void *energy,
                                void *forces, void *stress, void *energies, void *stresses,
                                void *workspace, size_t workspace_bytes, void *stream) {
  if (potential < TSB_POT_LJ || potential > TSB_POT_SOFT || n_species < 1 ||
      n_species > kMaxSpecies || !table || n_atoms < 1 || n_systems < 1 || !list || !counts ||
      !positions || !cell_row || !system_idx || !energy || !(prune_skin >= 0.0))
    return TSB_ERR_INVALID_ARG;
  if (n_species > 1 && !species) return TSB_ERR_INVALID_ARG;
  if (((out_flags & TSB_OUT_FORCES) && !forces) || ((out_flags & TSB_OUT_STRESS) && !stress) ||
      ((out_flags & TSB_OUT_ENERGIES) && !energies) ||
      ((out_flags & TSB_OUT_STRESSES) && !stresses))
    return TSB_ERR_INVALID_ARG;
  Carver c(workspace, workspace_bytes);
  VlWork w;
  carve_vl(c, w, n_atoms, n_systems);
  if (!c.ok || !workspace) return TSB_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == TSB_F64)
    return vl_forces<double>(potential, table, n_species, species, list, counts,
                             (const double *)positions, (const double *)cell_row, system_idx,
                             sys_active, n_atoms, n_systems, cutoff, prune_skin, out_flags,
                             (double *)energy, (double *)forces, (double *)stress,
                             (double *)energies, (double *)stresses, w, st);
  if (dtype == TSB_F32)
    return vl_forces<float>(potential, table, n_species, species, list, counts,
                            (const float *)positions, (const float *)cell_row, system_idx,
                            sys_active, n_atoms, n_systems, cutoff, prune_skin, out_flags,
                            (float *)energy,
                            (float *)forces, (float *)stress, (float *)energies,
                            (float *)stresses, w, st);
  return TSB_ERR_INVALID_ARG;
}
