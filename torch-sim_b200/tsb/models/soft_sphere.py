"""Soft-sphere models (drop-in for torch_sim/models/soft_sphere.py:175-377).

V(r) = eps/alpha (1 - r/sigma)^alpha for r < sigma, else 0 (soft_sphere.py:35-59);
the multi-species form looks sigma/epsilon/alpha up per species pair from
symmetric matrices indexed by the sorted unique atomic numbers (:90-167, :248-377).
Default cutoff: sigma (single) / max(sigma_matrix) (multi).

Unlike the reference, forces stay finite for non-integer alpha when a pair lies
between sigma_ab and the global cutoff: the reference differentiates
``(1 - r/sigma)^alpha`` of a negative base through ``torch.where`` and gets NaN
there; the analytic force is zero.
"""

from __future__ import annotations

import numpy as np
import torch

from .pair_potential import PairTableModel


class SoftSphereModel(PairTableModel):
    def __init__(self, sigma: float = 1.0, epsilon: float = 1.0, alpha: float = 2.0,
                 device=None, dtype=torch.float64, *, compute_forces=True,
                 compute_stress=False, per_atom_energies=False, per_atom_stresses=False,
                 neighbor_list_fn=None, use_neighbor_list=True, cutoff=None,
                 retain_graph=False, precision="mixed") -> None:
        self.sigma, self.epsilon, self.alpha = float(sigma), float(epsilon), float(alpha)
        rc = float(cutoff) if cutoff is not None else self.sigma
        table = [[[self.sigma, self.epsilon, self.alpha, np.inf, 0.0]]]
        super().__init__("soft_sphere", table, cutoff=rc, device=device, dtype=dtype,
                         compute_forces=compute_forces, compute_stress=compute_stress,
                         per_atom_energies=per_atom_energies,
                         per_atom_stresses=per_atom_stresses,
                         neighbor_list_fn=neighbor_list_fn, retain_graph=retain_graph,
                         precision=precision)


class SoftSphereMultiModel(PairTableModel):
    def __init__(self, atomic_numbers, sigma_matrix=None, epsilon_matrix=None,
                 alpha_matrix=None, device=None, dtype=torch.float64, *, pbc=True,
                 compute_forces=True, compute_stress=False, per_atom_energies=False,
                 per_atom_stresses=False, use_neighbor_list=True, neighbor_list_fn=None,
                 cutoff=None, retain_graph=False, precision="mixed") -> None:
        z = np.unique(np.asarray(torch.as_tensor(atomic_numbers).cpu()))
        ns = len(z)

        def mat(m, default):
            if m is None:
                return np.full((ns, ns), default)
            a = np.asarray(torch.as_tensor(m, dtype=torch.float64).detach().cpu())
            if a.shape != (ns, ns):
                raise ValueError(f"matrix must have shape ({ns}, {ns})")
            if not np.allclose(a, a.T):
                raise ValueError("parameter matrices must be symmetric")
            return a

        sig, eps, alp = mat(sigma_matrix, 1.0), mat(epsilon_matrix, 1.0), mat(alpha_matrix, 2.0)
        self.sigma_matrix, self.epsilon_matrix, self.alpha_matrix = sig, eps, alp
        tab = np.zeros((ns, ns, 5))
        tab[..., 0], tab[..., 1], tab[..., 2], tab[..., 3] = sig, eps, alp, np.inf
        rc = float(cutoff) if cutoff else float(sig.max())
        super().__init__("soft_sphere", tab, cutoff=rc, species_atomic_numbers=z,
                         device=device, dtype=dtype, compute_forces=compute_forces,
                         compute_stress=compute_stress, per_atom_energies=per_atom_energies,
                         per_atom_stresses=per_atom_stresses,
                         neighbor_list_fn=neighbor_list_fn, retain_graph=retain_graph,
                         precision=precision)
