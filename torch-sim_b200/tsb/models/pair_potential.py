"""Pair-potential models on the fused GPU neighbour-search + force kernel.

``PairTableModel`` is the drop-in for torch_sim/models/pair_potential.py:277-464
(PairPotentialModel with reduce_to_half_list=True) restricted to the analytic
pair functions the kernels implement: Lennard-Jones, Morse and soft sphere,
each with an optional species matrix (soft_sphere.py:90-167).  Outputs follow
the reference exactly:

* ``energy [S]``        sum of pair energies per system (:402-409)
* ``forces [N,3]``      -dE/dr_i (:420-441)
* ``stress [S,3,3]``    -1/V sum_pairs r_ij (x) f_ij (:200-232)
* ``energies [N]``      each endpoint receives the full pair energy (:411-417)
* ``stresses [N,3,3]``  each endpoint receives half the pair virial (:262-272)

Precision: ``precision="mixed"`` (default) evaluates the pair function in FP32
from FP64 displacements and accumulates per-system energy/virial in FP64;
``precision="fp64"`` runs the pair function in FP64 as well.
"""

from __future__ import annotations

import numpy as np
import torch

from .. import _lib as L
from .. import ops as _ops  # noqa: F401  (registers torch.ops.tsb.*)
from .interface import ModelInterface

KIND = {"lj": L.POT_LJ, "morse": L.POT_MORSE, "soft_sphere": L.POT_SOFT,
        "particle_life": L.POT_PLIFE}


class PairTableModel(ModelInterface):
    """Species-matrix pair potential evaluated by ``tsb_pair_forward``.

    Args:
        potential: "lj", "morse" or "soft_sphere".
        table: [n_species, n_species, 5] rows (p0, p1, p2, rc, eshift), see
            include/tsb.h (LJ: sigma, epsilon; Morse/soft sphere: sigma, epsilon,
            alpha; rc per-pair truncation; eshift subtracted inside rc).
        species_atomic_numbers: atomic number of each species row (sorted unique
            Z, as SoftSphereMultiModel does, soft_sphere.py:308-312); None means a
            single species for every atom.
        cutoff: neighbour cutoff (pairs at r >= cutoff are ignored, pair_potential.py:194).
    """

    def __init__(self, potential: str, table, *, cutoff: float,
                 species_atomic_numbers=None, device=None, dtype=torch.float64,
                 compute_forces: bool = True, compute_stress: bool = False,
                 per_atom_energies: bool = False, per_atom_stresses: bool = False,
                 neighbor_list_fn=None, retain_graph: bool = False,
                 precision: str = "mixed") -> None:
        super().__init__()
        if retain_graph:
            raise NotImplementedError(
                "retain_graph: tsb kernels are not traced by autograd; use "
                "tsb.adjoint for differentiable trajectories")
        if precision not in ("mixed", "fp64"):
            raise ValueError(f"precision must be 'mixed' or 'fp64', got {precision!r}")
        self._device = torch.device(device) if device is not None else torch.device("cuda")
        self._dtype = dtype
        self._compute_forces = compute_forces
        self._compute_stress = compute_stress
        self.per_atom_energies = per_atom_energies
        self.per_atom_stresses = per_atom_stresses
        self.potential = potential
        self.kind = KIND[potential]
        self.cutoff = float(cutoff)
        self.precision = precision
        # neighbor_list_fn is accepted for signature compatibility: the kernel
        # builds the identical pair set itself (fused search + force).
        self.neighbor_list_fn = neighbor_list_fn
        tab = np.asarray(table, dtype=np.float64)
        if tab.ndim != 3 or tab.shape[0] != tab.shape[1] or tab.shape[2] != 5:
            raise ValueError("table must have shape [n_species, n_species, 5]")
        if tab.shape[0] > 16:
            raise ValueError("at most 16 species are supported")
        self.n_species = tab.shape[0]
        self.table_np = tab
        self.register_buffer("table", torch.as_tensor(tab, device=self._device), persistent=False)
        if species_atomic_numbers is None:
            self.z_lut = None
        else:
            z = torch.as_tensor(species_atomic_numbers, dtype=torch.int64).cpu()
            lut = torch.full((int(z.max()) + 1,), -1, dtype=torch.int32)
            lut[z] = torch.arange(len(z), dtype=torch.int32)
            self.z_lut = lut.to(self._device)
        self._species_cache = (None, None)

    def _species(self, atomic_numbers: torch.Tensor):
        if self.z_lut is None:
            return None
        key = (atomic_numbers.data_ptr(), atomic_numbers._version, atomic_numbers.shape[0])
        if self._species_cache[0] == key:
            return self._species_cache[1]
        z = atomic_numbers.to(self.z_lut.device)
        if bool((z < 0).any() | (z >= len(self.z_lut)).any()):
            raise ValueError("atomic number outside the model's species table")
        sp = self.z_lut[z].contiguous()
        if bool((sp < 0).any()):
            raise ValueError("atomic number not in the model's species table")
        self._species_cache = (key, sp)
        return sp

    def forward(self, state, **_kwargs) -> dict[str, torch.Tensor]:
        if state.dtype != self._dtype:
            raise TypeError(
                f"SimState dtype {state.dtype} does not match model dtype {self._dtype}.")
        L.require_cuda(state.positions, "state.positions")
        n_sys = state.n_systems
        flags = self._flags(self._compute_forces, self._compute_stress, self.per_atom_energies,
                            self.per_atom_stresses)
        energy, forces, stress, energies, stresses = torch.ops.tsb.pair_forward(
            *self._inputs(state), self.kind, self.n_species, self.cutoff, flags, n_sys,
            L.max_system_atoms(state.system_idx, n_sys))
        out = {"energy": energy}
        if self._compute_forces:
            out["forces"] = forces
        if self._compute_stress:
            out["stress"] = stress
        if self.per_atom_energies:
            out["energies"] = energies
        if self.per_atom_stresses:
            out["stresses"] = stresses
        return out

    def forward_into(self, state, *, energy, forces, stress=None, sys_active=None):
        """Write energy/forces(/stress) of the systems with ``sys_active`` != 0 into
        existing contiguous buffers; the other systems' entries are left untouched."""
        if state.dtype != self._dtype:
            raise TypeError(
                f"SimState dtype {state.dtype} does not match model dtype {self._dtype}.")
        L.require_cuda(state.positions, "state.positions")
        for t in (energy, forces, stress):
            if t is not None and not t.is_contiguous():
                raise ValueError("forward_into needs contiguous output buffers")
        self._launch(state, energy, forces, stress if self._compute_stress else None, None,
                     None, sys_active)

    def _inputs(self, state):
        """(positions, cell_row, pbc, system_idx, species, table) as the operators take them."""
        pos = state.positions.contiguous()
        dev = pos.device
        n_sys = state.n_systems
        table = self.table if self.table.device == dev else self.table.to(dev)
        return (pos, state.cell.mT.contiguous(), L.pbc_rows(state.pbc, n_sys, dev),
                state.system_idx.contiguous(), self._species(state.atomic_numbers), table)

    def _flags(self, forces, stress, energies, stresses):
        flags = 0
        if forces:
            flags |= L.OUT_FORCES
        if stress:
            flags |= L.OUT_STRESS
        if energies:
            flags |= L.OUT_ENERGIES
        if stresses:
            flags |= L.OUT_STRESSES
        if self.precision == "fp64":
            flags |= L.MATH_FP64
        return flags

    def _launch(self, state, energy, forces, stress, energies, stresses, sys_active):
        if energies is not None or stresses is not None:
            raise ValueError("per-atom outputs are returned by forward(), not written into")
        n_sys = state.n_systems
        flags = self._flags(forces is not None, stress is not None, False, False)
        torch.ops.tsb.pair_forward_into_(
            *self._inputs(state), self.kind, self.n_species, self.cutoff, flags, n_sys,
            L.max_system_atoms(state.system_idx, n_sys), energy, forces, stress, sys_active)


def single_species_table(sigma, epsilon, alpha=0.0, rc=np.inf, eshift=0.0):
    return np.array([[[sigma, epsilon, alpha, rc, eshift]]], dtype=np.float64)


def lj_energy(r, sigma, epsilon):
    x6 = (sigma / r) ** 6
    return 4.0 * epsilon * (x6 * x6 - x6)
