// Lennard-Jones Hessian-vector product of one neighbour pair, shared by the
// cell-list and the Verlet-list HVP kernels (FP64).
//
// LJ: V = 4 eps (s^12 - s^6), s = sigma / r (lennard_jones.py:23-47)
//   V'  = -(24 eps / r)(2 s^12 - s^6)
//   V'' = (24 eps / r^2)(26 s^12 - 7 s^6)
//   dV'/deps = V' / eps ;  dV'/dsigma = -(144 eps / (r sigma))(4 s^12 - s^6)
// For d = r_j - r_i, u = d / r, the Hessian block is K = V'' u u^T + (V'/r)(I -
// u u^T); the pair adds K (v_i - v_j) to (H v)_i and (dV'/dtheta) (u . v_i) to
// the parameter gradients of its species pair.
#pragma once

#include "tsb_common.cuh"

namespace tsb {

constexpr int kAdjMaxSpecies = 4;

// per species pair: sigma^2, 1/sigma, epsilon, 1/epsilon, cutoff^2 (one FP64
// division per neighbour pair remains, 1/r)
struct LjHvpTable {
  double sig2[kAdjMaxSpecies * kAdjMaxSpecies], isig[kAdjMaxSpecies * kAdjMaxSpecies],
      eps[kAdjMaxSpecies * kAdjMaxSpecies], ieps[kAdjMaxSpecies * kAdjMaxSpecies],
      rc2[kAdjMaxSpecies * kAdjMaxSpecies];
};

// fill a shared-memory table from rows (sigma, epsilon, ., rc, .) of `table`
__device__ inline void lj_hvp_table(LjHvpTable &T, const double *table, int nsp, double cutoff) {
  for (int k = threadIdx.x; k < nsp * nsp; k += blockDim.x) {
    const double sg = table[5 * k], ep = table[5 * k + 1];
    T.sig2[k] = sg * sg;
    T.isig[k] = 1.0 / sg;
    T.eps[k] = ep;
    T.ieps[k] = 1.0 / ep;
    const double r = fmin(cutoff, table[5 * k + 3]);
    T.rc2[k] = r * r;
  }
}

// one pair (row k of the table, neighbour species sj): adds to h and to the
// register gradients gs / ge of species sj; pairs outside the cutoff add nothing
__device__ __forceinline__ void lj_hvp_pair(const LjHvpTable &T, int k, int sj, double dx,
                                            double dy, double dz, double d2, double vi0,
                                            double vi1, double vi2, double vj0, double vj1,
                                            double vj2, double &hx, double &hy, double &hz,
                                            double *gs, double *ge) {
  if (!(d2 < T.rc2[k]) || !(d2 > 0.0)) return;
  const double r = sqrt(d2), ir = 1.0 / r, ir2 = ir * ir;
  const double ux = dx * ir, uy = dy * ir, uz = dz * ir;
  const double s2 = T.sig2[k] * ir2, s6 = s2 * s2 * s2, s12 = s6 * s6;
  const double e = T.eps[k];
  const double vp = -(24.0 * e * ir) * (2.0 * s12 - s6);
  const double vpp = (24.0 * e * ir2) * (26.0 * s12 - 7.0 * s6);
  const double w0 = vi0 - vj0, w1 = vi1 - vj1, w2 = vi2 - vj2;
  const double uw = ux * w0 + uy * w1 + uz * w2;
  const double a = vpp - vp * ir;  // K w = a (u.w) u + (V'/r) w
  hx += a * uw * ux + vp * ir * w0;
  hy += a * uw * uy + vp * ir * w1;
  hz += a * uw * uz + vp * ir * w2;
  const double uvi = ux * vi0 + uy * vi1 + uz * vi2;
  const double dge = (vp * T.ieps[k]) * uvi;
  const double dgs = (-(144.0 * e * ir * T.isig[k]) * (4.0 * s12 - s6)) * uvi;
#pragma unroll
  for (int t2 = 0; t2 < kAdjMaxSpecies; ++t2)
    if (t2 == sj) {
      ge[t2] += dge;
      gs[t2] += dgs;
    }
}

}  // namespace tsb
