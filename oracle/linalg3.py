"""3x3 matrix-function oracle (TEST INFRASTRUCTURE ONLY; never the product path).

* ``expm_frechet`` <- torch_sim/math.py:107-189 (expm_frechet_sps): scaling and
  squaring with the [13/13] Pade approximant and its Frechet derivative
  (Al-Mohy & Higham 2009, SIAM J. Matrix Anal. Appl. 30(4):1639-1657).  Like
  the reference, the scaling power ``s`` is chosen from the largest 1-norm in
  the batch (math.py:133-137).
* ``expm``          the R factor of the same scheme (torch.matrix_exp in the
  reference, cell_filters.py / fire.py:440) -- agrees to rounding.
* ``logm``          scipy.linalg.logm, the reference's own fallback
  (math.py:416-445); its closed-form eigen-case path (math.py:615-745) agrees
  to rounding for the real-spectrum matrices used here.
"""

from __future__ import annotations

import numpy as np

# Pade [13/13] numerator coefficients b_0..b_13 (Higham 2005).
PADE13 = (64764752532480000.0, 32382376266240000.0, 7771770303897600.0,
          1187353796428800.0, 129060195264000.0, 10559470521600.0,
          670442572800.0, 33522128640.0, 1323241920.0, 40840800.0, 960960.0,
          16380.0, 182.0, 1.0)
THETA13 = 4.74  # ell_13 bound used by the reference (math.py:229-253, index 13)


def expm_frechet(A, E):
    """Return (expm(A), L_exp(A, E)) for batches [B,3,3] (or single [3,3])."""
    A = np.asarray(A, dtype=np.float64)
    E = np.asarray(E, dtype=np.float64)
    single = A.ndim == 2
    if single:
        A, E = A[None], E[None]
    b = PADE13
    # torch.norm(A, p=1, dim=(-2, -1)) is the ENTRYWISE 1-norm (math.py:132)
    norm1 = np.abs(A).sum(axis=(1, 2))
    sv = np.log2(np.clip(norm1.max() / THETA13, 1.0, 2.0 ** 64))
    s = max(0, min(int(np.ceil(sv)), 64))
    A = A * 2.0 ** -s
    E = E * 2.0 ** -s
    I = np.broadcast_to(np.eye(3), A.shape)
    A2 = A @ A
    M2 = A @ E + E @ A
    A4 = A2 @ A2
    M4 = A2 @ M2 + M2 @ A2
    A6 = A2 @ A4
    M6 = A4 @ M2 + M4 @ A2
    W1 = b[13] * A6 + b[11] * A4 + b[9] * A2
    W2 = b[7] * A6 + b[5] * A4 + b[3] * A2 + b[1] * I
    Z1 = b[12] * A6 + b[10] * A4 + b[8] * A2
    Z2 = b[6] * A6 + b[4] * A4 + b[2] * A2 + b[0] * I
    W = A6 @ W1 + W2
    U = A @ W
    V = A6 @ Z1 + Z2
    Lw1 = b[13] * M6 + b[11] * M4 + b[9] * M2
    Lw2 = b[7] * M6 + b[5] * M4 + b[3] * M2
    Lz1 = b[12] * M6 + b[10] * M4 + b[8] * M2
    Lz2 = b[6] * M6 + b[4] * M4 + b[2] * M2
    Lw = A6 @ Lw1 + M6 @ W1 + Lw2
    Lu = A @ Lw + E @ W
    Lv = A6 @ Lz1 + M6 @ Z1 + Lz2
    R = np.linalg.solve(-U + V, U + V)
    L = np.linalg.solve(-U + V, Lu + Lv + (Lu - Lv) @ R)
    for _ in range(s):
        L = R @ L + L @ R
        R = R @ R
    if single:
        return R[0], L[0]
    return R, L


def expm(A):
    return expm_frechet(A, np.zeros_like(np.asarray(A, dtype=np.float64)))[0]


def logm(T):
    import scipy.linalg

    T = np.asarray(T, dtype=np.float64)
    if T.ndim == 2:
        return np.real(scipy.linalg.logm(T))
    return np.stack([np.real(scipy.linalg.logm(t)) for t in T])
