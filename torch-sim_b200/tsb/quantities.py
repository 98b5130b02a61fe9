"""Per-system reductions used by reporters and convergence checks.

* ``calc_kinetic_energy`` <- torch_sim/quantities.py:104-139 (1/2 sum p^2/m)
* ``calc_kT``             <- quantities.py:16-66 (sum p^2/m / dof, dof = 3 n)
* ``system_wise_max_force`` <- quantities.py:327-342
"""

from __future__ import annotations

import torch


def _seg_sum(v: torch.Tensor, system_idx: torch.Tensor, n_sys: int) -> torch.Tensor:
    return torch.zeros(n_sys, dtype=v.dtype, device=v.device).index_add_(0, system_idx, v)


def calc_kinetic_energy(*, masses, momenta, system_idx, n_systems=None):
    n = n_systems if n_systems is not None else int(system_idx.max()) + 1
    return 0.5 * _seg_sum((momenta ** 2 / masses[:, None]).sum(1), system_idx, n)


def calc_kT(*, masses, momenta, system_idx, dof_per_system=None, n_systems=None):
    n = n_systems if n_systems is not None else int(system_idx.max()) + 1
    s = _seg_sum((momenta ** 2 / masses[:, None]).sum(1), system_idx, n)
    if dof_per_system is None:
        dof_per_system = 3 * torch.bincount(system_idx, minlength=n)
    return s / dof_per_system


def system_wise_max_force(forces, system_idx, n_systems=None):
    n = n_systems if n_systems is not None else int(system_idx.max()) + 1
    out = torch.zeros(n, dtype=forces.dtype, device=forces.device)
    return out.scatter_reduce(0, system_idx, forces.norm(dim=1), reduce="amax")
