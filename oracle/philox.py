"""Counter-based random draws of the CUDA kernels, restated in numpy (TEST
INFRASTRUCTURE ONLY; never the product path).

The reference draws its Langevin and V-rescale noise from
``torch.randn(generator=state.rng)`` (torch_sim/integrators/nvt.py:27-86,
594-654).  A persistent GPU kernel cannot share one sequential generator
between thousands of threads, so the tsb kernels draw from a stateless
counter-based generator instead: Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
"Parallel random numbers: as easy as 1, 2, 3", SC'11), keyed by the seed and
counted by (atom or system, step).  This module restates those draws so that
the oracle can replay a fused-kernel trajectory with the very same noise:

* ``philox4x32_10``   the generator: 10 rounds of two 32x32->64-bit products
  (multipliers 0xD2511F53, 0xCD9E8D57) with the Weyl key schedule
  (0x9E3779B9, 0xBB67AE85), as published.
* ``fused_normals``   the three Langevin normals per atom and step of the
  fused MD kernel: counter (atom, step), key = seed; Box-Muller on 24-bit
  uniforms u = (w >> 8 + 1) 2^-24 for the radii and t = (w >> 8) 2^-23 for the
  angles pi t.  The kernel evaluates these in FP32 with the hardware's
  approximate log2, sine and cosine (on pi (t - 1), negated); here they are
  evaluated in FP64 from the same integers, so the two agree to a few 1e-6
  absolute.
* ``step_normals``    the four FP64 normals per atom and step of the per-call
  BAOAB kernel (32-bit uniforms, FP64 Box-Muller).
* ``thermo_normal`` / ``gamma_deviate``  the per-system draws of the V-rescale
  (CSVR) factor: 53-bit uniforms from a tagged counter, Box-Muller, and
  Marsaglia-Tsang gamma deviates (ACM TOMS 26:363, 2000) with at most 64
  proposals.

Everything here is exact integer arithmetic on uint64 arrays up to the final
floating-point transforms.
"""

from __future__ import annotations

import numpy as np

_MASK = np.uint64(0xFFFFFFFF)
_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = 0x9E3779B9, 0xBB67AE85


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 of counter words (c0, c1, c2, c3) under key (k0, k1).

    All arguments broadcast; returns four uint64 arrays holding 32-bit words.
    """
    c0, c1, c2, c3 = (np.asarray(v, dtype=np.uint64) & _MASK for v in (c0, c1, c2, c3))
    k0 = int(k0) & 0xFFFFFFFF
    k1 = int(k1) & 0xFFFFFFFF
    for _ in range(10):
        p0 = _M0 * c0
        p1 = _M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK
        c0, c1, c2, c3 = (hi1 ^ c1 ^ np.uint64(k0), lo1, hi0 ^ c3 ^ np.uint64(k1), lo0)
        k0 = (k0 + _W0) & 0xFFFFFFFF
        k1 = (k1 + _W1) & 0xFFFFFFFF
    return c0, c1, c2, c3


def _split64(v):
    v = np.asarray(v, dtype=np.uint64)
    return v & _MASK, v >> np.uint64(32)


def fused_normals(seed: int, atoms, counter: int) -> np.ndarray:
    """[len(atoms), 3] Langevin normals of the fused kernel for global atom
    indices ``atoms`` at Philox counter ``counter`` (= start counter + step)."""
    atoms = np.asarray(atoms, dtype=np.uint64)
    a_lo, a_hi = _split64(atoms)
    c_lo, c_hi = _split64(np.full(atoms.shape, counter, dtype=np.uint64))
    seed = int(seed) & (2**64 - 1)
    x, y, z, w = philox4x32_10(a_lo, a_hi, c_lo, c_hi, seed & 0xFFFFFFFF, seed >> 32)
    k24 = 2.0 ** -24
    u1 = ((x >> np.uint64(8)) + np.uint64(1)).astype(np.float64) * k24
    u2 = ((z >> np.uint64(8)) + np.uint64(1)).astype(np.float64) * k24
    t1 = (y >> np.uint64(8)).astype(np.float64) * (2.0 * k24)
    t2 = (w >> np.uint64(8)).astype(np.float64) * (2.0 * k24)
    r1 = np.sqrt(-2.0 * np.log(u1))
    r2 = np.sqrt(-2.0 * np.log(u2))
    return np.stack([r1 * np.cos(np.pi * t1), r1 * np.sin(np.pi * t1),
                     r2 * np.cos(np.pi * t2)], axis=1)


def step_normals(seed: int, atoms, counter: int) -> np.ndarray:
    """[len(atoms), 3] normals of the per-call BAOAB kernel (first three of the
    four FP64 Box-Muller normals per atom and counter)."""
    atoms = np.asarray(atoms, dtype=np.uint64)
    a_lo, a_hi = _split64(atoms)
    c_lo, c_hi = _split64(np.full(atoms.shape, counter, dtype=np.uint64))
    seed = int(seed) & (2**64 - 1)
    x, y, z, w = philox4x32_10(a_lo, a_hi, c_lo, c_hi, seed & 0xFFFFFFFF, seed >> 32)
    k32 = 2.0 ** -32
    r1 = np.sqrt(-2.0 * np.log((x.astype(np.float64) + 1.0) * k32))
    r2 = np.sqrt(-2.0 * np.log((z.astype(np.float64) + 1.0) * k32))
    a1 = 2.0 * np.pi * (y.astype(np.float64) * k32)
    a2 = 2.0 * np.pi * (w.astype(np.float64) * k32)
    return np.stack([r1 * np.cos(a1), r1 * np.sin(a1), r2 * np.cos(a2)], axis=1)


def _u53(a, b):
    a, b = int(a), int(b)
    return (float((a >> 5) * 67108864 + (b >> 6)) + 1.0) * 2.0 ** -53


def _thermo_words(seed: int, system: int, counter: int, slot: int):
    seed = int(seed) & (2**64 - 1)
    counter = int(counter) & (2**64 - 1)
    r = philox4x32_10(int(system) & 0xFFFFFFFF, 0xC5A00000 ^ slot, counter & 0xFFFFFFFF,
                      counter >> 32, seed & 0xFFFFFFFF, seed >> 32)
    return [int(v) for v in r]


def thermo_normal(seed: int, system: int, counter: int, slot: int) -> float:
    """One standard normal of the thermostat stream (system, counter, slot)."""
    x, y, z, w = _thermo_words(seed, system, counter, slot)
    return float(np.sqrt(-2.0 * np.log(_u53(x, y))) * np.cos(np.pi * (2.0 * _u53(z, w))))


def gamma_deviate(a: float, seed: int, system: int, counter: int) -> float:
    """Gamma(a, 1) deviate of the thermostat stream (Marsaglia & Tsang 2000;
    a < 1 through Gamma(a + 1) U^(1/a)); at most 64 proposals."""
    boost = 1.0
    if a < 1.0:
        x, y, _, _ = _thermo_words(seed, system, counter, 1)
        boost = _u53(x, y) ** (1.0 / a)
        a += 1.0
    d = a - 1.0 / 3.0
    c = 1.0 / np.sqrt(9.0 * d)
    for k in range(64):
        xn = thermo_normal(seed, system, counter, 16 + 2 * k)
        v0 = 1.0 + c * xn
        if v0 <= 0.0:
            continue
        v = v0 * v0 * v0
        x, y, _, _ = _thermo_words(seed, system, counter, 17 + 2 * k)
        u = _u53(x, y)
        if u < 1.0 - 0.0331 * (xn * xn) * (xn * xn) or \
                np.log(u) < 0.5 * xn * xn + d * (1.0 - v + np.log(v)):
            return d * v * boost
    return d * boost


def vrescale_draws(seed: int, system: int, counter: int, dof: float):
    """(r1, gamma sample) of the V-rescale factor of one system and step."""
    return (thermo_normal(seed, system, counter, 0),
            gamma_deviate((dof - 1.0) / 2.0, seed, system, counter))
