// FP64 3x3 matrix functions for the per-system cell filter (one thread per system).
//
// expm + Frechet derivative: scaling and squaring with the [13/13] Pade
// approximant (Higham 2005; Frechet form of Al-Mohy & Higham 2009, SIAM J.
// Matrix Anal. Appl. 30(4):1639-1657) -- the algorithm of
// torch_sim/math.py:107-189, with the scaling chosen per system instead of from
// the largest norm in the batch (results agree to rounding).
// logm: inverse scaling and squaring -- Denman-Beavers square roots until the
// matrix is within 0.05 of the identity, then the Mercator series of log(I + D).
#pragma once

namespace tsb {

struct M3 {
  double a[9];  // row-major
  __device__ double &operator()(int r, int c) { return a[3 * r + c]; }
  __device__ double operator()(int r, int c) const { return a[3 * r + c]; }
};

__device__ inline M3 m3_zero() {
  M3 m;
#pragma unroll
  for (int k = 0; k < 9; ++k) m.a[k] = 0.0;
  return m;
}

__device__ inline M3 m3_eye(double v = 1.0) {
  M3 m = m3_zero();
  m.a[0] = m.a[4] = m.a[8] = v;
  return m;
}

__device__ inline M3 m3_mul(const M3 &x, const M3 &y) {
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      r.a[3 * i + j] = x.a[3 * i] * y.a[j] + x.a[3 * i + 1] * y.a[3 + j] + x.a[3 * i + 2] * y.a[6 + j];
  return r;
}

__device__ inline M3 m3_add(const M3 &x, const M3 &y, double cx = 1.0, double cy = 1.0) {
  M3 r;
#pragma unroll
  for (int k = 0; k < 9; ++k) r.a[k] = cx * x.a[k] + cy * y.a[k];
  return r;
}

__device__ inline M3 m3_scale(const M3 &x, double c) {
  M3 r;
#pragma unroll
  for (int k = 0; k < 9; ++k) r.a[k] = c * x.a[k];
  return r;
}

__device__ inline M3 m3_T(const M3 &x) {
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.a[3 * i + j] = x.a[3 * j + i];
  return r;
}

__device__ inline double m3_det(const M3 &m) {
  const double *a = m.a;
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
         a[2] * (a[3] * a[7] - a[4] * a[6]);
}

__device__ inline M3 m3_inv(const M3 &m) {
  const double *a = m.a;
  const double id = 1.0 / m3_det(m);
  M3 r;
  r.a[0] = (a[4] * a[8] - a[5] * a[7]) * id;
  r.a[1] = (a[2] * a[7] - a[1] * a[8]) * id;
  r.a[2] = (a[1] * a[5] - a[2] * a[4]) * id;
  r.a[3] = (a[5] * a[6] - a[3] * a[8]) * id;
  r.a[4] = (a[0] * a[8] - a[2] * a[6]) * id;
  r.a[5] = (a[2] * a[3] - a[0] * a[5]) * id;
  r.a[6] = (a[3] * a[7] - a[4] * a[6]) * id;
  r.a[7] = (a[1] * a[6] - a[0] * a[7]) * id;
  r.a[8] = (a[0] * a[4] - a[1] * a[3]) * id;
  return r;
}

// X = A^-1 B  (A well conditioned here: Pade denominators, cell matrices)
__device__ inline M3 m3_solve(const M3 &A, const M3 &B) { return m3_mul(m3_inv(A), B); }

__device__ inline double m3_norm1_entrywise(const M3 &x) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) s += fabs(x.a[k]);
  return s;
}

__device__ inline double m3_maxabs(const M3 &x) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) s = fmax(s, fabs(x.a[k]));
  return s;
}

// exp(A) and its Frechet derivative L(A, E).  The scaling power uses the
// entrywise 1-norm against theta_13 = 4.74, as the reference does.
__device__ inline void m3_expm_frechet(const M3 &A_in, const M3 &E_in, M3 *R_out, M3 *L_out) {
  const double b0 = 64764752532480000.0, b1 = 32382376266240000.0, b2 = 7771770303897600.0,
               b3 = 1187353796428800.0, b4 = 129060195264000.0, b5 = 10559470521600.0,
               b6 = 670442572800.0, b7 = 33522128640.0, b8 = 1323241920.0, b9 = 40840800.0,
               b10 = 960960.0, b11 = 16380.0, b12 = 182.0, b13 = 1.0;
  double nrm = m3_norm1_entrywise(A_in);
  int s = 0;
  if (nrm > 4.74) s = (int)ceil(log2(fmin(nrm / 4.74, 1.8e19)));
  if (s > 64) s = 64;
  const double sc = ldexp(1.0, -s);
  const M3 A = m3_scale(A_in, sc), E = m3_scale(E_in, sc);
  const M3 I = m3_eye();
  const M3 A2 = m3_mul(A, A);
  const M3 M2 = m3_add(m3_mul(A, E), m3_mul(E, A));
  const M3 A4 = m3_mul(A2, A2);
  const M3 M4 = m3_add(m3_mul(A2, M2), m3_mul(M2, A2));
  const M3 A6 = m3_mul(A2, A4);
  const M3 M6 = m3_add(m3_mul(A4, M2), m3_mul(M4, A2));
  M3 W1, W2, Z1, Z2, Lw1, Lw2, Lz1, Lz2;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    W1.a[k] = b13 * A6.a[k] + b11 * A4.a[k] + b9 * A2.a[k];
    W2.a[k] = b7 * A6.a[k] + b5 * A4.a[k] + b3 * A2.a[k] + b1 * I.a[k];
    Z1.a[k] = b12 * A6.a[k] + b10 * A4.a[k] + b8 * A2.a[k];
    Z2.a[k] = b6 * A6.a[k] + b4 * A4.a[k] + b2 * A2.a[k] + b0 * I.a[k];
    Lw1.a[k] = b13 * M6.a[k] + b11 * M4.a[k] + b9 * M2.a[k];
    Lw2.a[k] = b7 * M6.a[k] + b5 * M4.a[k] + b3 * M2.a[k];
    Lz1.a[k] = b12 * M6.a[k] + b10 * M4.a[k] + b8 * M2.a[k];
    Lz2.a[k] = b6 * M6.a[k] + b4 * M4.a[k] + b2 * M2.a[k];
  }
  const M3 W = m3_add(m3_mul(A6, W1), W2);
  const M3 U = m3_mul(A, W);
  const M3 V = m3_add(m3_mul(A6, Z1), Z2);
  const M3 Lw = m3_add(m3_add(m3_mul(A6, Lw1), m3_mul(M6, W1)), Lw2);
  const M3 Lu = m3_add(m3_mul(A, Lw), m3_mul(E, W));
  const M3 Lv = m3_add(m3_add(m3_mul(A6, Lz1), m3_mul(M6, Z1)), Lz2);
  const M3 Q = m3_add(V, U, 1.0, -1.0);
  const M3 Qi = m3_inv(Q);
  M3 R = m3_mul(Qi, m3_add(U, V));
  M3 L = m3_mul(Qi, m3_add(m3_add(Lu, Lv), m3_mul(m3_add(Lu, Lv, 1.0, -1.0), R)));
  for (int k = 0; k < s; ++k) {
    L = m3_add(m3_mul(R, L), m3_mul(L, R));
    R = m3_mul(R, R);
  }
  *R_out = R;
  if (L_out) *L_out = L;
}

__device__ inline M3 m3_expm(const M3 &A) {
  M3 R;
  m3_expm_frechet(A, m3_zero(), &R, nullptr);
  return R;
}

// principal square root by the Denman-Beavers iteration
__device__ inline M3 m3_sqrtm(const M3 &X) {
  M3 Y = X, Z = m3_eye();
  for (int it = 0; it < 40; ++it) {
    const M3 Yi = m3_inv(Y), Zi = m3_inv(Z);
    const M3 Yn = m3_scale(m3_add(Y, Zi), 0.5);
    const M3 Zn = m3_scale(m3_add(Z, Yi), 0.5);
    const double d = m3_maxabs(m3_add(Yn, Y, 1.0, -1.0));
    Y = Yn;
    Z = Zn;
    if (d < 1e-15 * fmax(1.0, m3_maxabs(Y))) break;
  }
  return Y;
}

// principal matrix logarithm of a matrix with real positive spectrum near I
__device__ inline M3 m3_logm(const M3 &F) {
  M3 X = F;
  const M3 I = m3_eye();
  int k = 0;
  while (m3_maxabs(m3_add(X, I, 1.0, -1.0)) > 0.05 && k < 30) {
    X = m3_sqrtm(X);
    ++k;
  }
  const M3 D = m3_add(X, I, 1.0, -1.0);
  // log(I + D) = sum_{j>=1} (-1)^{j+1} D^j / j, |D| <= 0.05: 14 terms reach 1e-19
  M3 P = D, S = D;
  for (int j = 2; j <= 14; ++j) {
    P = m3_mul(P, D);
    const double c = ((j & 1) ? 1.0 : -1.0) / (double)j;
    S = m3_add(S, P, 1.0, c);
  }
  return m3_scale(S, ldexp(1.0, k));
}

}  // namespace tsb
