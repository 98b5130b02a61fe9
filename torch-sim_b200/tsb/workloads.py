"""Seeded synthetic inputs for the classical-potential workloads.

The reference builds its structures with ASE (torch_sim/testing.py:246-253);
here every structure is built directly as numpy arrays so no ASE is needed.
All builders return plain dicts of numpy arrays in the SimState conventions
(state.py:138-142): ``positions [N,3]``, ``masses [N]``, ``cell`` column-vector
``[S,3,3]``, ``pbc [3]``, ``atomic_numbers [N]``, ``system_idx [N]``.

Workloads (units: Angstrom, eV, amu):

* ``argon_fcc``     LJ argon fcc n1 x n2 x n3 conventional cells, a = 5.26,
                    positions jittered by N(0, jitter)  (256-atom NVE case and the
                    500,000-atom single-system neighbour-list/force case)
* ``copper_batch``  Cu fcc supercells (a = 3.61) with atom counts drawn
                    uniformly in [n_min, n_max] and rounded to the nearest
                    4*n1*n2*n3, random diagonal strain and triclinic shear
                    (2048-system Morse NVT-Langevin case)
* ``kob_andersen_batch``  80:20 binary LJ boxes at number density 1.2 sigma_AA^-3
                    with uniform random positions (1024-system FIRE case)
* ``argon_species_batch`` fcc 3x3x3 argon systems with two species assigned
                    50:50 at random (differentiable-trajectory case)
"""

from __future__ import annotations

import math

import numpy as np

FCC_BASIS = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
AR_MASS, AR_Z = 39.948, 18
CU_MASS, CU_Z = 63.546, 29


def fcc_fractional(n1, n2, n3):
    """Fractional coordinates (in units of the supercell) of an fcc supercell."""
    g = np.stack(np.meshgrid(np.arange(n1), np.arange(n2), np.arange(n3), indexing="ij"),
                 -1).reshape(-1, 3)
    pts = (g[:, None, :] + FCC_BASIS[None]).reshape(-1, 3)
    return pts / np.array([n1, n2, n3], dtype=np.float64)


def _pack(systems, pbc=True):
    pos = np.concatenate([s["positions"] for s in systems])
    return {
        "positions": pos,
        "masses": np.concatenate([s["masses"] for s in systems]),
        "cell": np.stack([s["cell_row"].T for s in systems]),
        "pbc": np.array([pbc] * 3),
        "atomic_numbers": np.concatenate([s["atomic_numbers"] for s in systems]),
        "system_idx": np.concatenate([np.full(len(s["positions"]), k, dtype=np.int64)
                                      for k, s in enumerate(systems)]),
    }


def argon_fcc(n=(4, 4, 4), a=5.26, jitter=0.05, seed=0, n_systems=1):
    rng = np.random.default_rng(seed)
    cell_row = np.diag([n[0] * a, n[1] * a, n[2] * a]).astype(np.float64)
    frac = fcc_fractional(*n)
    systems = []
    for _ in range(n_systems):
        pos = frac @ cell_row + rng.normal(0.0, jitter, size=(len(frac), 3))
        systems.append({"positions": pos, "cell_row": cell_row,
                        "masses": np.full(len(pos), AR_MASS),
                        "atomic_numbers": np.full(len(pos), AR_Z, dtype=np.int64)})
    return _pack(systems)


def nearest_fcc_shape(target):
    """(n1, n2, n3) with 4*n1*n2*n3 closest to ``target`` (most cubic on ties)."""
    best = None
    for n1 in range(1, 9):
        for n2 in range(n1, 9):
            for n3 in range(n2, 17):
                n = 4 * n1 * n2 * n3
                key = (abs(n - target), n3 - n1)
                if best is None or key < best[0]:
                    best = (key, (n1, n2, n3))
    return best[1]


def strained_cell(n, a, rng, strain, shear_deg):
    """Row-vector cell of an n1 x n2 x n3 supercell with diagonal strain and shear."""
    base = np.diag([n[0] * a, n[1] * a, n[2] * a]).astype(np.float64)
    deform = np.eye(3) + np.diag(rng.uniform(-strain, strain, 3))
    t = np.tan(np.deg2rad(rng.uniform(-shear_deg, shear_deg, 3)))
    deform[0, 1], deform[0, 2], deform[1, 2] = t
    return base @ deform


def copper_batch(n_systems=2048, n_min=8, n_max=512, seed=0, a=3.61, strain=0.02,
                 shear_deg=3.0, jitter=0.0):
    rng = np.random.default_rng(seed)
    systems = []
    for _ in range(n_systems):
        shape = nearest_fcc_shape(int(rng.integers(n_min, n_max + 1)))
        perm = rng.permutation(3)
        shape = tuple(np.array(shape)[perm])
        cell_row = strained_cell(shape, a, rng, strain, shear_deg)
        pos = fcc_fractional(*shape) @ cell_row
        if jitter:
            pos = pos + rng.normal(0.0, jitter, pos.shape)
        systems.append({"positions": pos, "cell_row": cell_row,
                        "masses": np.full(len(pos), CU_MASS),
                        "atomic_numbers": np.full(len(pos), CU_Z, dtype=np.int64)})
    return _pack(systems)


def kob_andersen_batch(n_systems=1024, n_min=64, n_max=1000, seed=0, sigma_aa=3.4,
                       density=1.2):
    """Species A (Z=1) / B (Z=2) 80:20, cubic box L = (N / rho)^(1/3)."""
    rng = np.random.default_rng(seed)
    rho = density / sigma_aa ** 3
    systems = []
    for _ in range(n_systems):
        n = int(rng.integers(n_min, n_max + 1))
        L = (n / rho) ** (1.0 / 3.0)
        pos = rng.uniform(0.0, L, size=(n, 3))
        z = np.full(n, 1, dtype=np.int64)
        z[rng.permutation(n)[: int(round(0.2 * n))]] = 2
        systems.append({"positions": pos, "cell_row": np.eye(3) * L,
                        "masses": np.full(n, AR_MASS), "atomic_numbers": z})
    return _pack(systems)


def argon_species_batch(n_systems=256, n=(3, 3, 3), a=5.26, seed=0, jitter=0.0):
    rng = np.random.default_rng(seed)
    cell_row = np.diag([n[0] * a, n[1] * a, n[2] * a]).astype(np.float64)
    frac = fcc_fractional(*n)
    systems = []
    for _ in range(n_systems):
        m = len(frac)
        z = np.full(m, 1, dtype=np.int64)
        z[rng.permutation(m)[: m // 2]] = 2
        pos = frac @ cell_row
        if jitter:
            pos = pos + rng.normal(0.0, jitter, pos.shape)
        systems.append({"positions": pos, "cell_row": cell_row,
                        "masses": np.full(m, AR_MASS), "atomic_numbers": z})
    return _pack(systems)


def counts_of(system_idx):
    return np.bincount(np.asarray(system_idx))


def maxwell_boltzmann_normal(n_atoms, seed):
    """Standard normals used to draw initial momenta (shape [N,3])."""
    return np.random.default_rng(seed).standard_normal((n_atoms, 3))


# Same CODATA-2014 constants as torch_sim/units.py:50-59.
_E_CHARGE, _K_B, _AMU = 1.6021766208e-19, 1.38064852e-23, 1.660539040e-27
KB_EV = _K_B / _E_CHARGE  # eV/K (MetalUnits.temperature, units.py:112)
# internal time units per ps (MetalUnits.time, units.py:108): dt_internal = dt_ps * METAL_TIME
METAL_TIME = math.sqrt(_E_CHARGE / (_AMU * 1e-20)) * 1e-12
