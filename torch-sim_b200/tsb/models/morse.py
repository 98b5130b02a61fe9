"""Morse model (drop-in for torch_sim/models/morse.py:78-144).

V(r) = eps (1 - exp(-alpha (r - sigma)))^2 - eps (morse.py:23-47), default
cutoff 2.5 sigma.
"""

from __future__ import annotations

import numpy as np
import torch

from .pair_potential import PairTableModel


class MorseModel(PairTableModel):
    def __init__(self, sigma: float = 1.0, epsilon: float = 5.0, alpha: float = 5.0,
                 device=None, dtype=torch.float64, *, compute_forces=True,
                 compute_stress=False, per_atom_energies=False, per_atom_stresses=False,
                 neighbor_list_fn=None, cutoff: float | None = None, retain_graph=False,
                 precision="mixed") -> None:
        self.sigma, self.epsilon, self.alpha = float(sigma), float(epsilon), float(alpha)
        rc = float(cutoff) if cutoff is not None else 2.5 * self.sigma
        table = [[[self.sigma, self.epsilon, self.alpha, np.inf, 0.0]]]
        super().__init__("morse", table, cutoff=rc, device=device, dtype=dtype,
                         compute_forces=compute_forces, compute_stress=compute_stress,
                         per_atom_energies=per_atom_energies,
                         per_atom_stresses=per_atom_stresses,
                         neighbor_list_fn=neighbor_list_fn, retain_graph=retain_graph,
                         precision=precision)
