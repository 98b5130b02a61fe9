"""Batched simulation-state containers mirroring TorchSim's SimState family.

Field names, shapes and conventions follow the reference so that code written
against ``torch_sim.SimState`` works unchanged:

* ``SimState``      <- torch_sim/state.py:120-860 (positions [N,3], masses [N],
  cell [S,3,3] in the COLUMN-vector convention (state.py:138-142), pbc [3],
  atomic_numbers [N], system_idx [N] contiguous)
* ``MDState``       <- torch_sim/integrators/md.py:31-110 (+ momenta, energy, forces)
* ``FireState``     <- torch_sim/optimizers/state.py:38-51
* ``CellFireState`` <- torch_sim/optimizers/cell_filters.py:457-467

The tsb models and step functions only read attributes, so a reference
``torch_sim.SimState`` can be passed in directly as well.
"""

from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field

import torch


@dataclass(kw_only=True)
class SimState:
    positions: torch.Tensor
    masses: torch.Tensor
    cell: torch.Tensor
    pbc: torch.Tensor | bool | list = True
    atomic_numbers: torch.Tensor
    system_idx: torch.Tensor | None = None
    _rng: object = field(default=None, repr=False)
    _n_systems: int | None = field(default=None, repr=False)

    def __post_init__(self) -> None:
        dev = self.positions.device
        if not isinstance(self.pbc, torch.Tensor):
            p = [self.pbc] * 3 if isinstance(self.pbc, bool) else list(self.pbc)
            self.pbc = torch.tensor(p, dtype=torch.bool, device=dev)
        if self.system_idx is None:
            self.system_idx = torch.zeros(self.positions.shape[0], dtype=torch.int64,
                                          device=dev)
        if self.cell.ndim == 2:
            self.cell = self.cell.unsqueeze(0)
        n = {self.positions.shape[0], self.masses.shape[0], self.atomic_numbers.shape[0]}
        if len(n) != 1:
            raise ValueError(f"Incompatible shapes: {n}")

    # --- reference properties -------------------------------------------------
    @property
    def device(self) -> torch.device:
        return self.positions.device

    @property
    def dtype(self) -> torch.dtype:
        return self.positions.dtype

    @property
    def n_atoms(self) -> int:
        return self.positions.shape[0]

    @property
    def n_systems(self) -> int:
        if self._n_systems is None:
            self._n_systems = self.cell.shape[0]
        return self._n_systems

    @property
    def n_atoms_per_system(self) -> torch.Tensor:
        return self.system_idx.bincount(minlength=self.n_systems)

    @property
    def row_vector_cell(self) -> torch.Tensor:
        return self.cell.mT

    @row_vector_cell.setter
    def row_vector_cell(self, value: torch.Tensor) -> None:
        self.cell = value.mT

    @property
    def volume(self) -> torch.Tensor:
        return torch.det(self.cell)

    @property
    def rng(self) -> torch.Generator:
        if not isinstance(self._rng, torch.Generator):
            g = torch.Generator(device=self.device)
            if isinstance(self._rng, int):
                g.manual_seed(self._rng)
            self._rng = g
        return self._rng

    @rng.setter
    def rng(self, value) -> None:
        self._rng = value

    @property
    def constraints(self) -> list:
        return []

    def set_constrained_positions(self, new_positions: torch.Tensor) -> None:
        self.positions = new_positions

    def clone(self):
        kw = {f.name: (getattr(self, f.name).clone()
                       if isinstance(getattr(self, f.name), torch.Tensor)
                       else getattr(self, f.name))
              for f in dataclasses.fields(self)}
        return type(self)(**kw)

    def to(self, device=None, dtype=None):
        kw = {}
        for f in dataclasses.fields(self):
            v = getattr(self, f.name)
            if isinstance(v, torch.Tensor):
                v = v.to(device=device) if device is not None else v
                if dtype is not None and v.is_floating_point():
                    v = v.to(dtype=dtype)
            kw[f.name] = v
        return type(self)(**kw)

    @classmethod
    def from_state(cls, state, **extra):
        """Build ``cls`` from any SimState-like object (tsb or torch_sim)."""
        names = {f.name for f in dataclasses.fields(cls)}
        kw = {}
        for k in ("positions", "masses", "cell", "pbc", "atomic_numbers", "system_idx"):
            kw[k] = getattr(state, k)
        if "_rng" in names:
            kw["_rng"] = getattr(state, "_rng", None)
        for k in names:
            if k not in kw and k not in extra and hasattr(state, k) and not k.startswith("_"):
                kw[k] = getattr(state, k)
        kw.update(extra)
        return cls(**kw)


@dataclass(kw_only=True)
class MDState(SimState):
    momenta: torch.Tensor
    energy: torch.Tensor
    forces: torch.Tensor

    @property
    def velocities(self) -> torch.Tensor:
        return self.momenta / self.masses.unsqueeze(-1)

    def set_constrained_momenta(self, new_momenta: torch.Tensor) -> None:
        self.momenta = new_momenta


@dataclass
class NoseHooverChain:
    """Per-system Nose-Hoover chain variables (torch_sim/integrators/md.py:249-273):
    positions / momenta / masses [S, M], tau, kinetic_energy, degrees_of_freedom [S]."""

    positions: torch.Tensor
    momenta: torch.Tensor
    masses: torch.Tensor
    tau: torch.Tensor
    kinetic_energy: torch.Tensor
    degrees_of_freedom: torch.Tensor

    def clone(self) -> "NoseHooverChain":
        return NoseHooverChain(*(getattr(self, f.name).clone()
                                 for f in dataclasses.fields(self)))


@dataclass(kw_only=True)
class NVTNoseHooverState(MDState):
    """MDState + Nose-Hoover chain (torch_sim/integrators/nvt.py:244-290).  The
    chain integrates with ``chain_dt`` [S], the time step it was set up with."""

    chain: NoseHooverChain
    chain_steps: int = 3
    sy_steps: int = 3
    chain_dt: torch.Tensor | None = None

    def clone(self):
        c = super().clone()
        c.chain = self.chain.clone()
        return c

    def get_number_of_degrees_of_freedom(self) -> torch.Tensor:
        return self.chain.degrees_of_freedom


@dataclass(kw_only=True)
class NVTVRescaleState(MDState):
    """MDState for the V-rescale thermostat (torch_sim/integrators/nvt.py:565-591)."""


@dataclass(kw_only=True)
class NPTLangevinIsotropicState(MDState):
    """MDState + strain-based isotropic barostat (torch_sim/integrators/npt.py:653-703):
    stress [S,3,3]; per system alpha, cell_alpha, b_tau, strain ``cell_positions``
    (eps = ln(V/V0)/3), ``cell_velocities`` (d eps/dt), ``cell_masses``;
    ``reference_cell`` [S,3,3] (cell = exp(eps) reference_cell)."""

    stress: torch.Tensor
    alpha: torch.Tensor
    cell_alpha: torch.Tensor
    b_tau: torch.Tensor
    reference_cell: torch.Tensor
    cell_positions: torch.Tensor
    cell_velocities: torch.Tensor
    cell_masses: torch.Tensor

    @property
    def current_cell(self) -> torch.Tensor:
        return torch.exp(self.cell_positions)[:, None, None] * self.reference_cell

    @property
    def volume(self) -> torch.Tensor:
        return torch.linalg.det(self.reference_cell) * torch.exp(3 * self.cell_positions)


@dataclass(kw_only=True)
class NPTLangevinAnisotropicState(MDState):
    """MDState + per-axis strain barostat (torch_sim/integrators/npt.py:62-131):
    stress [S,3,3]; per system alpha, cell_alpha, b_tau, cell_masses; per-axis
    strains ``cell_positions`` [S,3] (eps_k = ln(L_k/L0_k)) and ``cell_velocities``
    [S,3]; ``reference_cell`` [S,3,3] (cell row k = exp(eps_k) reference row k)."""

    stress: torch.Tensor
    alpha: torch.Tensor
    cell_alpha: torch.Tensor
    b_tau: torch.Tensor
    reference_cell: torch.Tensor
    cell_positions: torch.Tensor
    cell_velocities: torch.Tensor
    cell_masses: torch.Tensor

    @property
    def current_cell(self) -> torch.Tensor:
        return torch.exp(self.cell_positions).unsqueeze(-1) * self.reference_cell

    @property
    def volume(self) -> torch.Tensor:
        return torch.linalg.det(self.cell)


@dataclass(kw_only=True)
class NPTNoseHooverIsotropicState(MDState):
    """MDState + MTK isotropic barostat with Nose-Hoover chains
    (torch_sim/integrators/npt.py:1110-1219): stress [S,3,3]; reference_cell
    [S,3,3]; log-volume ``cell_position`` [S] (ln(V/V0)/3), ``cell_momentum`` [S,1],
    ``cell_mass`` [S]; particle ``thermostat`` and cell ``barostat`` chains; the
    chains integrate with ``chain_dt`` [S]."""

    stress: torch.Tensor
    reference_cell: torch.Tensor
    cell_position: torch.Tensor
    cell_momentum: torch.Tensor
    cell_mass: torch.Tensor
    thermostat: NoseHooverChain
    barostat: NoseHooverChain
    chain_steps: int = 2
    sy_steps: int = 3
    chain_dt: torch.Tensor | None = None

    @property
    def current_cell(self) -> torch.Tensor:
        v0 = torch.linalg.det(self.reference_cell)
        v = v0 * torch.exp(3 * self.cell_position)
        return torch.pow(v / v0, 1.0 / 3.0)[:, None, None] * self.reference_cell

    def clone(self):
        c = super().clone()
        c.thermostat = self.thermostat.clone()
        c.barostat = self.barostat.clone()
        return c


@dataclass(kw_only=True)
class NPTCRescaleState(MDState):
    """MDState + stochastic cell rescaling (torch_sim/integrators/npt.py:2062-2090):
    stress [S,3,3]; per system isothermal_compressibility and tau_p; the initial cell
    [S,3,3], its inverse and volume."""

    stress: torch.Tensor
    isothermal_compressibility: torch.Tensor
    tau_p: torch.Tensor
    initial_cell: torch.Tensor
    initial_cell_inv: torch.Tensor
    initial_volume: torch.Tensor


@dataclass(kw_only=True)
class FireState(SimState):
    forces: torch.Tensor
    energy: torch.Tensor
    stress: torch.Tensor | None
    velocities: torch.Tensor
    dt: torch.Tensor
    alpha: torch.Tensor
    n_pos: torch.Tensor

    def set_constrained_forces(self, new_forces: torch.Tensor) -> None:
        self.forces = new_forces


@dataclass(kw_only=True)
class CellFireState(FireState):
    reference_cell: torch.Tensor
    cell_filter: str = "frechet"
    cell_factor: torch.Tensor | None = None
    pressure: torch.Tensor | None = None
    cell_positions: torch.Tensor | None = None
    cell_forces: torch.Tensor | None = None
    cell_velocities: torch.Tensor | None = None
    cell_masses: torch.Tensor | None = None
    hydrostatic_strain: bool = False
    constant_volume: bool = False


def state_from_arrays(d: dict, device="cuda", dtype=torch.float64) -> SimState:
    """SimState from the numpy dicts produced by :mod:`tsb.workloads`."""
    t = lambda x, dt=dtype: torch.as_tensor(x, dtype=dt, device=device)  # noqa: E731
    return SimState(positions=t(d["positions"]), masses=t(d["masses"]), cell=t(d["cell"]),
                    pbc=torch.as_tensor(d["pbc"], dtype=torch.bool, device=device),
                    atomic_numbers=t(d["atomic_numbers"], torch.int64),
                    system_idx=t(d["system_idx"], torch.int64))


# per-atom fields of the state classes above (first dimension n_atoms)
_ATOM_FIELDS = {"positions", "masses", "atomic_numbers", "system_idx", "momenta", "forces",
                "velocities"}


def select_systems(state, systems):
    """The systems ``systems`` (indices, any order) of a batched state, as a new
    state of the same class with systems renumbered 0..k-1 in ascending order of
    their old index (as ``SimState.__getitem__`` in torch_sim/state.py selects
    systems).  Per-atom fields are masked, per-system fields indexed, the rest
    copied by reference."""
    dev = state.device
    n_sys = state.n_systems
    sel = torch.unique(torch.as_tensor(systems, dtype=torch.long, device=dev))
    if sel.numel() == 0 or int(sel.min()) < 0 or int(sel.max()) >= n_sys:
        raise IndexError(f"system indices must lie in [0, {n_sys})")
    keep = torch.zeros(n_sys, dtype=torch.bool, device=dev)
    keep[sel] = True
    atom_mask = keep[state.system_idx]
    renum = torch.full((n_sys,), -1, dtype=torch.long, device=dev)
    renum[sel] = torch.arange(sel.numel(), device=dev)
    n_atoms = state.n_atoms
    kw = {}
    for f in dataclasses.fields(state):
        v = getattr(state, f.name)
        if f.name == "system_idx":
            v = renum[v[atom_mask]]
        elif f.name == "_n_systems":
            v = None
        elif isinstance(v, torch.Tensor) and v.ndim > 0:
            if f.name in _ATOM_FIELDS or (v.shape[0] == n_atoms and n_atoms != n_sys):
                v = v[atom_mask]
            elif v.shape[0] == n_sys and not (f.name == "pbc" and v.ndim == 1):
                v = v[sel]
        kw[f.name] = v
    return type(state)(**kw)
