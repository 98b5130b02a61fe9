"""Lennard-Jones models (drop-in for torch_sim/models/lennard_jones.py:74-137).

V(r) = 4 eps [(sigma/r)^12 - (sigma/r)^6] (lennard_jones.py:23-47), default
cutoff 2.5 sigma, no energy shift unless ``shift_energy=True`` (then V - V(rc),
forces unchanged).  ``LennardJonesMultiModel`` is the species-matrix form used
for binary mixtures such as Kob-Andersen, with a per-pair truncation radius.
"""

from __future__ import annotations

import numpy as np
import torch

from .pair_potential import PairTableModel, lj_energy


class LennardJonesModel(PairTableModel):
    def __init__(self, sigma: float = 1.0, epsilon: float = 1.0, device=None,
                 dtype=torch.float64, *, compute_forces=True, compute_stress=False,
                 per_atom_energies=False, per_atom_stresses=False, neighbor_list_fn=None,
                 cutoff: float | None = None, retain_graph=False, shift_energy=False,
                 precision="mixed") -> None:
        self.sigma, self.epsilon = float(sigma), float(epsilon)
        rc = float(cutoff) if cutoff is not None else 2.5 * self.sigma
        eshift = lj_energy(rc, self.sigma, self.epsilon) if shift_energy else 0.0
        table = [[[self.sigma, self.epsilon, 0.0, np.inf, eshift]]]
        super().__init__("lj", table, cutoff=rc, device=device, dtype=dtype,
                         compute_forces=compute_forces, compute_stress=compute_stress,
                         per_atom_energies=per_atom_energies,
                         per_atom_stresses=per_atom_stresses,
                         neighbor_list_fn=neighbor_list_fn, retain_graph=retain_graph,
                         precision=precision)


UnbatchedLennardJonesModel = LennardJonesModel


class LennardJonesMultiModel(PairTableModel):
    """Species-matrix LJ: each pair (a, b) uses sigma_ab, epsilon_ab and is
    truncated at trunc_ab (default ``trunc * sigma_ab``), shifted to zero there
    when ``shift_energy``."""

    def __init__(self, atomic_numbers, sigma_matrix, epsilon_matrix, *, trunc=2.5,
                 cutoff_matrix=None, shift_energy=True, cutoff=None, device=None,
                 dtype=torch.float64, compute_forces=True, compute_stress=False,
                 per_atom_energies=False, per_atom_stresses=False, neighbor_list_fn=None,
                 precision="mixed") -> None:
        z = np.unique(np.asarray(torch.as_tensor(atomic_numbers).cpu()))
        sig = np.asarray(torch.as_tensor(sigma_matrix, dtype=torch.float64).cpu())
        eps = np.asarray(torch.as_tensor(epsilon_matrix, dtype=torch.float64).cpu())
        rcm = (trunc * sig if cutoff_matrix is None
               else np.asarray(torch.as_tensor(cutoff_matrix, dtype=torch.float64).cpu()))
        ns = len(z)
        tab = np.zeros((ns, ns, 5))
        for a in range(ns):
            for b in range(ns):
                sh = lj_energy(rcm[a, b], sig[a, b], eps[a, b]) if shift_energy else 0.0
                tab[a, b] = [sig[a, b], eps[a, b], 0.0, rcm[a, b], sh]
        rc = float(cutoff) if cutoff is not None else float(rcm.max())
        super().__init__("lj", tab, cutoff=rc, species_atomic_numbers=z, device=device,
                         dtype=dtype, compute_forces=compute_forces,
                         compute_stress=compute_stress, per_atom_energies=per_atom_energies,
                         per_atom_stresses=per_atom_stresses,
                         neighbor_list_fn=neighbor_list_fn, precision=precision)


def kob_andersen_model(sigma_aa=3.4, epsilon_aa=0.0104, atomic_numbers=(1, 2), **kw):
    """Kob-Andersen 80:20 binary LJ (A = first Z, B = second Z): sigma_AB = 0.8,
    sigma_BB = 0.88, eps_AB = 1.5, eps_BB = 0.5 in units of sigma_AA, eps_AA;
    truncated and shifted at 2.5 sigma_ab."""
    sig = np.array([[1.0, 0.8], [0.8, 0.88]]) * sigma_aa
    eps = np.array([[1.0, 1.5], [1.5, 0.5]]) * epsilon_aa
    return LennardJonesMultiModel(list(atomic_numbers), sig, eps, trunc=2.5,
                                  cutoff=2.5 * sigma_aa, **kw)
