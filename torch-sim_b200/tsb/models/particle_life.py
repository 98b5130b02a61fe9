"""Force-defined pair models (drop-ins for torch_sim/models/pair_potential.py:467-612
and torch_sim/models/particle_life.py).

* ``ParticleLifeModel``      -- the particle-life force on the fused
  neighbour-search + force kernel (``tsb_pair_forward`` with TSB_POT_PLIFE).  The
  reference evaluates it on a full neighbour list, so every pair acts in both
  directions; the kernel's thread for atom i adds f(i <- j) and f(j <- i), and the
  stress carries the full-list weight 1/2 (per-atom stresses 1/4), as the
  reference does.  Energies are zero.
* ``ParticleLifeMultiModel`` -- the same with per-species-pair (A, beta, sigma)
  matrices, which may be asymmetric: row (a, b) is the force an atom of species a
  feels from a neighbour of species b.
* ``PairForcesModel``        -- any Python force function ``f(r, zi, zj)``: the
  pairs come from the tsb neighbour-list kernel (``torchsim_nl``) and the user's
  function runs as torch operations, as in the reference.
"""

from __future__ import annotations

import torch

from .. import _lib as L
from ..neighbors import full_to_half_list, torchsim_nl
from .interface import ModelInterface
from .pair_potential import PairTableModel


class ParticleLifeModel(PairTableModel):
    """Particle life with amplitude ``epsilon`` (the reference's ``A``), inner radius
    ``beta`` and outer radius ``sigma``; cutoff defaults to 2.5 sigma."""

    def __init__(self, sigma: float = 1.0, epsilon: float = 1.0, beta: float = 0.3,
                 device=None, dtype=torch.float64, *, compute_stress: bool = False,
                 per_atom_stresses: bool = False, neighbor_list_fn=None,
                 cutoff: float | None = None, precision: str = "mixed", **_kwargs) -> None:
        cutoff = 2.5 * sigma if cutoff is None else float(cutoff)
        self.sigma_param, self.epsilon, self.beta = sigma, epsilon, beta
        super().__init__("particle_life", [[[sigma, epsilon, beta, cutoff, 0.0]]],
                         cutoff=cutoff, device=device, dtype=dtype,
                         compute_stress=compute_stress, per_atom_stresses=per_atom_stresses,
                         neighbor_list_fn=neighbor_list_fn, precision=precision)


class ParticleLifeMultiModel(PairTableModel):
    """Particle life with [n_species, n_species] matrices ``A``, ``beta``, ``sigma``
    (row a, column b: the force on an atom of species a from one of species b)."""

    def __init__(self, atomic_numbers, A, beta, sigma, *, cutoff: float, device=None,
                 dtype=torch.float64, compute_stress: bool = False,
                 per_atom_stresses: bool = False, precision: str = "mixed") -> None:
        import numpy as np

        A, beta, sigma = (np.asarray(x, dtype=np.float64) for x in (A, beta, sigma))
        ns = len(atomic_numbers)
        tab = np.zeros((ns, ns, 5))
        tab[..., 0], tab[..., 1], tab[..., 2] = sigma, A, beta
        tab[..., 3] = cutoff
        z = np.asarray(atomic_numbers)
        order = np.argsort(z)
        tab = tab[order][:, order]
        super().__init__("particle_life", tab, cutoff=cutoff,
                         species_atomic_numbers=z[order].tolist(), device=device,
                         dtype=dtype, compute_stress=compute_stress,
                         per_atom_stresses=per_atom_stresses, precision=precision)


class PairForcesModel(ModelInterface):
    """Forces from a scalar pair force ``force_fn(distances, zi, zj)`` (1-D tensors
    over pairs) within ``cutoff``: F_i -= f r_hat_ij, F_j += f r_hat_ij per listed
    pair (full list unless ``reduce_to_half_list``)."""

    def __init__(self, force_fn, *, cutoff: float, device=None, dtype=torch.float64,
                 compute_stress: bool = False, per_atom_stresses: bool = False,
                 neighbor_list_fn=torchsim_nl, reduce_to_half_list: bool = False) -> None:
        super().__init__()
        self._device = torch.device(device) if device is not None else torch.device("cuda")
        self._dtype = dtype
        self._compute_forces = True
        self._compute_stress = compute_stress
        self.per_atom_stresses = per_atom_stresses
        self.force_fn = force_fn
        self.neighbor_list_fn = neighbor_list_fn
        self.cutoff = float(cutoff)
        self.reduce_to_half_list = reduce_to_half_list

    def forward(self, state, **_kwargs) -> dict[str, torch.Tensor]:
        if state.dtype != self._dtype:
            raise TypeError(
                f"SimState dtype {state.dtype} does not match model dtype {self._dtype}.")
        pos = state.positions
        n_sys = state.n_systems
        row_cell = state.cell.mT
        pbc = L.pbc_rows(state.pbc, n_sys, pos.device).bool()
        mapping, sysm, shifts = self.neighbor_list_fn(
            positions=pos, cell=row_cell, pbc=pbc, cutoff=self.cutoff,
            system_idx=state.system_idx)
        if self.reduce_to_half_list:
            mapping, sysm, shifts = full_to_half_list(mapping, sysm, shifts)
        i, j = mapping[0], mapping[1]
        dr = pos[j] - pos[i] + torch.einsum("pk,pkm->pm", shifts.to(pos.dtype), row_cell[sysm])
        r = dr.norm(dim=1)
        z = state.atomic_numbers
        f = self.force_fn(r, z[i], z[j])
        f = torch.where(r < self.cutoff, f, torch.zeros_like(f))
        safe = torch.where(r > 0, r, torch.ones_like(r))
        fv = (f / safe)[:, None] * dr
        forces = torch.zeros_like(pos).index_add(0, i, -fv).index_add(0, j, fv)
        out = {"energy": torch.zeros(n_sys, dtype=pos.dtype, device=pos.device),
               "forces": forces}
        if self._compute_stress or self.per_atom_stresses:
            vol = torch.linalg.det(row_cell).abs()
            spp = torch.einsum("pi,pj->pij", dr, fv)
            if self._compute_stress:
                st = torch.zeros((n_sys, 3, 3), dtype=pos.dtype, device=pos.device)
                st = st.index_add(0, sysm, -spp) / vol[:, None, None]
                out["stress"] = st * (1.0 if self.reduce_to_half_list else 0.5)
            if self.per_atom_stresses:
                w = 0.5 if self.reduce_to_half_list else 0.25
                sa = torch.zeros((pos.shape[0], 3, 3), dtype=pos.dtype, device=pos.device)
                sa = sa.index_add(0, i, -w * spp).index_add(0, j, -w * spp)
                out["stresses"] = sa / vol[state.system_idx][:, None, None]
        return out
