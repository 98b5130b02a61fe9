"""Trajectory oracle for the persistent fused MD kernel (TEST INFRASTRUCTURE
ONLY; never the product path).

Replays, in FP64 numpy, what one launch of the fused kernel computes for every
system of a batch: ``n_steps`` of the reference integrator with forces from the
reference pair model, using the fused kernel's own random draws
(``oracle.philox``) so that the two trajectories can be compared step for step.

* Langevin: B(dt/2) A(dt/2) O(dt) A(dt/2) F B(dt/2) = ``oracle.md.nvt_langevin_step``
  (torch_sim/integrators/nvt.py:144-240), normals = ``philox.fused_normals``
  with counter (global atom index, start counter + step).
* NVE: ``oracle.md.nve_step`` (torch_sim/integrators/nve.py:74-130).
* Nose-Hoover chain: ``oracle.thermostats.nvt_nose_hoover_step``
  (torch_sim/integrators/nvt.py:381-488), the first half step with the
  kinetic energy carried from the previous step.
* V-rescale (CSVR): ``oracle.thermostats.nvt_vrescale_step``
  (torch_sim/integrators/nvt.py:715-741) with (r1, gamma) from
  ``philox.vrescale_draws`` keyed by (system, start counter + step).

Forces are the reference pair model restated in ``oracle.pair.pair_forward``
(torch_sim/models/pair_potential.py:351-464).  For speed the full pair list is
built once at ``cutoff + skin`` with ``oracle.neighbors.neighbor_list`` (the
restatement of torch_nl.py:156-215) and rebuilt whenever an atom moved more
than skin/2 since the build; every step evaluates the pairs of that list with
the strict test r < cutoff.  Pairs closer than the cutoff are always in such a
list, so the forces are those of a fresh neighbour list at every step (checked
in tests/test_oracle_golden.py).

The initial forces are taken from the caller, as the kernel takes them from the
state it is given.
"""

from __future__ import annotations

import numpy as np

from . import md as omd
from . import neighbors as onl
from . import pair as opair
from . import philox
from . import thermostats as oth


class VerletForces:
    """FP64 forces, energies and stresses of the reference pair model over a
    full pair list at cutoff + skin, rebuilt after moves beyond skin/2."""

    def __init__(self, kind, table, species, cell_row, system_idx, cutoff, skin=1.0):
        self.kind, self.table = kind, np.asarray(table, dtype=np.float64)
        self.species = np.asarray(species)
        self.cell_row = np.asarray(cell_row, dtype=np.float64)
        self.system_idx = np.asarray(system_idx, dtype=np.int64)
        self.cutoff, self.skin = float(cutoff), float(skin)
        self.pbc = np.ones((self.cell_row.shape[0], 3), dtype=bool)
        self.x_build = None
        self.pairs = None
        self.n_builds = 0

    def _maybe_rebuild(self, x):
        if self.x_build is not None:
            d2 = ((x - self.x_build) ** 2).sum(1)
            if d2.max() <= (0.5 * self.skin) ** 2:
                return
        self.pairs = onl.neighbor_list(x, self.cell_row, self.pbc, self.cutoff + self.skin,
                                       self.system_idx)
        self.x_build = x.copy()
        self.n_builds += 1

    def __call__(self, x):
        x = np.asarray(x, dtype=np.float64)
        self._maybe_rebuild(x)
        return opair.pair_forward(self.kind, self.table, self.species, x, self.cell_row,
                                  self.pbc, self.system_idx, self.cutoff, pairs=self.pairs)


def run(kind, table, species, positions, momenta, forces, masses, cell_row, system_idx,
        cutoff, n_steps, dt, *, integrator="nvt_langevin", kT=None, gamma=None, seed=0,
        counter=0, skin=1.0, tau=None, chain=None, chain_steps=1, sy_steps=1):
    """Advance every system by ``n_steps``; returns a dict with positions,
    momenta, forces (FP64 at the final positions), energy [S], stress [S,3,3]
    and, for the Nose-Hoover chain, the final chain state.

    ``dt``, ``kT``, ``gamma`` and ``tau`` are per-system arrays or scalars;
    ``chain`` is a dict ``xi, p_xi, ke, dof, tau`` ([S, M] / [S]).
    """
    system_idx = np.asarray(system_idx, dtype=np.int64)
    n_sys = int(system_idx.max()) + 1
    per_sys = lambda v: np.broadcast_to(np.asarray(v, dtype=np.float64), (n_sys,))  # noqa: E731
    dt_s = per_sys(dt)
    if not np.all(dt_s == dt_s[0]):
        raise ValueError("the oracle replays one time step for the whole batch")
    h = float(dt_s[0])
    fn = VerletForces(kind, table, species, cell_row, system_idx, cutoff, skin)
    state = {"positions": np.array(positions, dtype=np.float64),
             "momenta": np.array(momenta, dtype=np.float64),
             "masses": np.asarray(masses, dtype=np.float64),
             "forces": np.array(forces, dtype=np.float64), "energy": np.zeros(n_sys)}
    last = {}

    def force_fn(q):
        out = fn(q)
        last.update(out)
        return out["energy"], out["forces"]

    atoms = np.arange(len(system_idx), dtype=np.uint64)
    counts = np.bincount(system_idx, minlength=n_sys)
    dof = 3.0 * counts - 3.0
    for step in range(n_steps):
        c = int(counter) + step
        if integrator == "nvt_langevin":
            g = (1.0 / (100.0 * h)) if gamma is None else gamma
            z = philox.fused_normals(seed, atoms, c)
            state = omd.nvt_langevin_step(state, force_fn, h, per_sys(kT), per_sys(g), z,
                                          system_idx)
        elif integrator == "nve":
            state = omd.nve_step(state, force_fn, h)
        elif integrator == "nvt_nose_hoover":
            state, chain = oth.nvt_nose_hoover_step(state, chain, force_fn, h, per_sys(kT),
                                                    chain_steps, sy_steps, system_idx)
        elif integrator == "nvt_vrescale":
            tau_s = per_sys(10.0 * h if tau is None else tau)
            draws = [philox.vrescale_draws(seed, s, c, dof[s]) for s in range(n_sys)]
            r1 = np.array([d[0] for d in draws])
            gs = np.array([d[1] for d in draws])
            state = oth.nvt_vrescale_step(state, force_fn, h, per_sys(kT), tau_s, r1, gs,
                                          system_idx)
        else:
            raise ValueError(integrator)
    if n_steps == 0 or not last:
        force_fn(state["positions"])
    out = {"positions": state["positions"], "momenta": state["momenta"],
           "forces": last["forces"], "energy": last["energy"], "stress": last["stress"],
           "n_builds": fn.n_builds}
    if integrator == "nvt_nose_hoover":
        out["chain"] = chain
    return out
