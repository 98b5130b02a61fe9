"""Molecular-dynamics step oracle (TEST INFRASTRUCTURE ONLY; never the product path).

FP64 numpy restatement of the reference integrators.  Random numbers are passed
in explicitly (the reference draws them from ``torch.randn(generator=state.rng)``)
so one step can be compared exactly.

* ``initialize_momenta`` <- torch_sim/integrators/md.py:113-166
* ``momentum_step``      <- md.py:169-187       p += F dt
* ``position_step``      <- md.py:190-208       q += p/m dt
* ``nve_step``           <- torch_sim/integrators/nve.py:74-130  (B(dt/2) A(dt) F B(dt/2))
* ``ou_step``            <- torch_sim/integrators/nvt.py:27-86
* ``nvt_langevin_step``  <- nvt.py:144-240       (B A O A F B, gamma default 1/(100 dt))
* ``calc_kT``            <- torch_sim/quantities.py:16-66
* ``kinetic_energy``     <- quantities.py:104-139
"""

from __future__ import annotations

import numpy as np


def _per_atom(x, system_idx):
    x = np.asarray(x, dtype=np.float64)
    return x[system_idx] if x.ndim > 0 else x


def initialize_momenta(masses, system_idx, kT, normal):
    """p = sqrt(m kT) * normal, minus the per-system mean when the system has >1 atom."""
    kT_a = _per_atom(kT, system_idx)
    p = normal * np.sqrt(masses * kT_a)[:, None]
    n_sys = int(system_idx.max()) + 1
    counts = np.bincount(system_idx, minlength=n_sys)
    mean = np.zeros((n_sys, 3))
    np.add.at(mean, system_idx, p)
    mean = mean / counts[:, None]
    multi = (counts > 1)[system_idx][:, None]
    return np.where(multi, p - mean[system_idx], p)


def momentum_step(momenta, forces, dt):
    return momenta + forces * dt


def position_step(positions, momenta, masses, dt):
    return positions + momenta / masses[:, None] * dt


def nve_step(state, force_fn, dt):
    """state: dict positions, momenta, masses, forces, energy. force_fn(pos)->(E, F)."""
    p = momentum_step(state["momenta"], state["forces"], dt / 2)
    q = position_step(state["positions"], p, state["masses"], dt)
    e, f = force_fn(q)
    p = momentum_step(p, f, dt / 2)
    return dict(state, positions=q, momenta=p, forces=f, energy=e)


def ou_step(momenta, masses, system_idx, dt, kT, gamma, normal):
    """p <- c1 p + c2 sqrt(m) normal, c1 = exp(-gamma dt), c2 = sqrt(kT (1 - c1^2))."""
    c1 = np.exp(-np.asarray(gamma, dtype=np.float64) * dt)
    kT_a = _per_atom(kT, system_idx)
    c1_a = _per_atom(c1, system_idx)
    c2 = np.sqrt(kT_a * (1.0 - c1_a ** 2))
    c2 = c2[:, None] if np.ndim(c2) else c2
    c1_b = c1_a[:, None] if np.ndim(c1_a) else c1_a
    return c1_b * momenta + c2 * np.sqrt(masses)[:, None] * normal


def nvt_langevin_step(state, force_fn, dt, kT, gamma, normal, system_idx):
    if gamma is None:
        gamma = 1.0 / (100.0 * dt)
    p = momentum_step(state["momenta"], state["forces"], dt / 2)
    q = position_step(state["positions"], p, state["masses"], dt / 2)
    p = ou_step(p, state["masses"], system_idx, dt, kT, gamma, normal)
    q = position_step(q, p, state["masses"], dt / 2)
    e, f = force_fn(q)
    p = momentum_step(p, f, dt / 2)
    return dict(state, positions=q, momenta=p, forces=f, energy=e)


def calc_kT(masses, momenta, system_idx, dof=None):
    sq = (momenta ** 2 / masses[:, None]).sum(1)
    n_sys = int(system_idx.max()) + 1
    s = np.zeros(n_sys)
    np.add.at(s, system_idx, sq)
    if dof is None:
        dof = 3 * np.bincount(system_idx, minlength=n_sys)
    return s / dof


def kinetic_energy(masses, momenta, system_idx):
    sq = (momenta ** 2 / masses[:, None]).sum(1)
    n_sys = int(system_idx.max()) + 1
    s = np.zeros(n_sys)
    np.add.at(s, system_idx, sq)
    return 0.5 * s
