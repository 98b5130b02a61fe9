"""Pair-potential oracle (TEST INFRASTRUCTURE ONLY; never the product path).

FP64 numpy restatement of the reference pair functions and of
``PairPotentialModel.forward`` on a half list:

* ``lj``          <- torch_sim/models/lennard_jones.py:23-47 (+ :50-71 force)
* ``morse``       <- torch_sim/models/morse.py:23-47 (+ :50-75 force)
* ``soft_sphere`` <- torch_sim/models/soft_sphere.py:35-59 (+ :62-87 force)
* species matrix  <- torch_sim/models/soft_sphere.py:90-167 (MultiSoftSpherePairFn);
  the Lennard-Jones species matrix (Kob-Andersen) uses the same lookup with the
  LJ pair function and a per-pair truncation radius.
* ``pair_forward`` <- torch_sim/models/pair_potential.py:351-464 with
  ``_prepare_pairs`` (:130-197), ``_virial_stress`` (:200-232) and
  ``_accumulate_stress`` (:235-274).

The reference takes dV/dr by autograd (pair_potential.py:420-425); here the
analytic derivative is used, which agrees to rounding.

Potential kinds and their per-species-pair parameter rows ``(p0, p1, p2, rc, eshift)``:
  LJ=0     p0=sigma p1=epsilon            V = 4 eps [(s/r)^12 - (s/r)^6]       (r > 0)
  MORSE=1  p0=sigma p1=epsilon p2=alpha   V = eps (1 - e^{-a(r-s)})^2 - eps    (r > 0)
  SOFT=2   p0=sigma p1=epsilon p2=alpha   V = eps/a (1 - r/s)^a               (r < s)
``rc`` is the per-pair truncation (pairs at r >= rc contribute nothing) and
``eshift`` is subtracted from V inside rc (0 for the reference's unshifted forms).
"""

from __future__ import annotations

import numpy as np

from . import neighbors as onl

LJ, MORSE, SOFT = 0, 1, 2


def pair_energy_dvdr(kind, r, p0, p1, p2):
    """Return (V(r), dV/dr) for arrays r and broadcastable parameters."""
    r = np.asarray(r, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        if kind == LJ:
            x6 = (p0 / r) ** 6
            e = 4.0 * p1 * (x6 * x6 - x6)
            dv = -24.0 * p1 / r * (2.0 * x6 * x6 - x6)
            ok = r > 0
        elif kind == MORSE:
            ex = np.exp(-p2 * (r - p0))
            e = p1 * (1.0 - ex) ** 2 - p1
            dv = 2.0 * p2 * p1 * ex * (1.0 - ex)
            ok = r > 0
        elif kind == SOFT:
            base = 1.0 - r / p0
            e = p1 / p2 * base ** p2
            dv = -(p1 / p0) * base ** (p2 - 1.0)
            ok = r < p0
        else:
            raise ValueError(kind)
    e = np.where(ok, e, 0.0)
    dv = np.where(ok, dv, 0.0)
    return e, dv


def pair_forward(kind, table, species, positions, cell_row, pbc, system_idx, cutoff,
                 *, per_atom=False, pairs=None):
    """Energy [S], forces [N,3], stress [S,3,3] (+ energies [N], stresses [N,3,3]).

    ``table`` is [n_species, n_species, 5] rows ``(p0, p1, p2, rc, eshift)``;
    ``species`` is the per-atom species index.  ``pairs`` may pass a precomputed
    full list (mapping, system_mapping, shifts).
    """
    positions = np.asarray(positions, dtype=np.float64)
    system_idx = np.asarray(system_idx, dtype=np.int64)
    n = positions.shape[0]
    n_sys = int(system_idx.max()) + 1 if n else 0
    cell_row, pbc = onl.normalize_inputs(cell_row, pbc, n_sys)
    if pairs is None:
        pairs = onl.neighbor_list(positions, cell_row, pbc, cutoff, system_idx)
    mapping, sysm, shifts = onl.full_to_half_list(*pairs)
    i, j = mapping
    cs = np.einsum("pk,pkm->pm", shifts, cell_row[sysm])
    dr = positions[j] - positions[i] + cs
    r = np.linalg.norm(dr, axis=1)
    table = np.asarray(table, dtype=np.float64)
    prm = table[species[i], species[j]]
    e, dv = pair_energy_dvdr(kind, r, prm[:, 0], prm[:, 1], prm[:, 2])
    inside = (r < cutoff) & (r < prm[:, 3])
    e = np.where(inside, e - prm[:, 4], 0.0)
    dv = np.where(inside, dv, 0.0)
    safe = np.where(r > 0, r, 1.0)
    fvec = (-dv / safe)[:, None] * dr
    energy = np.zeros(n_sys)
    np.add.at(energy, sysm, e)
    forces = np.zeros((n, 3))
    np.add.at(forces, i, -fvec)
    np.add.at(forces, j, fvec)
    vol = np.abs(np.linalg.det(cell_row))
    spp = np.einsum("pi,pj->pij", dr, fvec)
    stress = np.zeros((n_sys, 3, 3))
    np.add.at(stress, sysm, -spp)
    stress = stress / vol[:, None, None]
    out = {"energy": energy, "forces": forces, "stress": stress}
    if per_atom:
        ea = np.zeros(n)
        np.add.at(ea, i, e)
        np.add.at(ea, j, e)
        sa = np.zeros((n, 3, 3))
        np.add.at(sa, i, -0.5 * spp)
        np.add.at(sa, j, -0.5 * spp)
        out["energies"] = ea
        out["stresses"] = sa / vol[system_idx][:, None, None]
    return out


def single_table(kind, sigma, epsilon, alpha=0.0, rc=np.inf, eshift=0.0):
    """[1,1,5] parameter table for a one-species potential."""
    return np.array([[[sigma, epsilon, alpha, rc, eshift]]], dtype=np.float64)


def lj_shift(sigma, epsilon, rc):
    """V_LJ(rc) for the energy-shifted Lennard-Jones form."""
    e, _ = pair_energy_dvdr(LJ, np.array([rc]), sigma, epsilon, 0.0)
    return float(e[0])


def kob_andersen_table(sigma_aa=3.4, eps_aa=0.0104, trunc=2.5, shift=True):
    """Kob-Andersen 80:20 binary LJ table (species 0 = A, 1 = B).

    sigma_AB = 0.8, sigma_BB = 0.88, eps_AB = 1.5, eps_BB = 0.5 (reduced units of
    sigma_AA, eps_AA); each pair is truncated at ``trunc * sigma_ab`` and, with
    ``shift``, shifted to zero energy there.
    """
    sig = np.array([[1.0, 0.8], [0.8, 0.88]]) * sigma_aa
    eps = np.array([[1.0, 1.5], [1.5, 0.5]]) * eps_aa
    tab = np.zeros((2, 2, 5))
    for a in range(2):
        for b in range(2):
            rc = trunc * sig[a, b]
            tab[a, b] = [sig[a, b], eps[a, b], 0.0, rc,
                         lj_shift(sig[a, b], eps[a, b], rc) if shift else 0.0]
    return tab


def particle_life_force(r, A=1.0, beta=0.3, sigma=1.0):
    """Particle-life force magnitude (torch_sim/models/particle_life.py:24-54):
    r/beta - 1 for r < beta; A (1 - |2r - 1 - beta| / (1 - beta)) for beta <= r < sigma."""
    r = np.asarray(r, dtype=np.float64)
    inner = np.where(r < beta, r / beta - 1.0, 0.0)
    outer = np.where((r >= beta) & (r < sigma),
                     A * (1.0 - np.abs(2.0 * r - 1.0 - beta) / (1.0 - beta)), 0.0)
    return inner + outer


def pair_forces_forward(force_fn, positions, cell_row, pbc, system_idx, atomic_numbers, cutoff,
                        *, half=False):
    """PairForcesModel.forward (torch_sim/models/pair_potential.py:467-612): forces from
    a scalar pair force f(r, zi, zj); F_i -= f r_hat, F_j += f r_hat per listed pair;
    stress -1/V sum r (x) f_vec times 1 (half list) or 1/2 (full list); per-atom
    stresses w = 1/2 or 1/4 of each pair virial on both endpoints; energy zero."""
    positions = np.asarray(positions, dtype=np.float64)
    system_idx = np.asarray(system_idx, dtype=np.int64)
    z = np.asarray(atomic_numbers)
    n = positions.shape[0]
    n_sys = int(system_idx.max()) + 1
    cell_row, pbc = onl.normalize_inputs(cell_row, pbc, n_sys)
    mapping, sysm, shifts = onl.neighbor_list(positions, cell_row, pbc, cutoff, system_idx)
    if half:
        mapping, sysm, shifts = onl.full_to_half_list(mapping, sysm, shifts)
    i, j = mapping
    dr = positions[j] - positions[i] + np.einsum("pk,pkm->pm", shifts, cell_row[sysm])
    r = np.linalg.norm(dr, axis=1)
    f = np.where(r < cutoff, force_fn(r, z[i], z[j]), 0.0)
    safe = np.where(r > 0, r, 1.0)
    fv = (f / safe)[:, None] * dr
    forces = np.zeros((n, 3))
    np.add.at(forces, i, -fv)
    np.add.at(forces, j, fv)
    vol = np.abs(np.linalg.det(cell_row))
    spp = np.einsum("pi,pj->pij", dr, fv)
    stress = np.zeros((n_sys, 3, 3))
    np.add.at(stress, sysm, -spp)
    stress = stress / vol[:, None, None] * (1.0 if half else 0.5)
    w = 0.5 if half else 0.25
    sa = np.zeros((n, 3, 3))
    np.add.at(sa, i, -w * spp)
    np.add.at(sa, j, -w * spp)
    return {"energy": np.zeros(n_sys), "forces": forces, "stress": stress,
            "stresses": sa / vol[system_idx][:, None, None]}
