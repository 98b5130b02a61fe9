"""Per-system reductions used by reporters and convergence checks.

* ``calc_kinetic_energy`` <- torch_sim/quantities.py:104-139 (1/2 sum p^2/m)
* ``calc_kT``             <- quantities.py:16-66 (sum p^2/m / dof, dof = 3 n)
* ``system_wise_max_force`` <- quantities.py:327-342

The sums run in the ``tsb_kinetic_energy`` kernel: one block per system, FP64,
a fixed summation order, so repeated calls give bitwise equal results (a
float atomic scatter such as ``index_add_`` sums in a run-dependent order).
The maximum is order-independent and stays a torch ``scatter_reduce``.
"""

from __future__ import annotations

import torch

from . import _lib as L


def _sum_p2m(masses, momenta, system_idx, n_sys: int) -> torch.Tensor:
    """FP64 per-system sum of p^2/m in a fixed order."""
    L.require_cuda(momenta, "momenta")
    p = momenta.contiguous()
    dt = p.dtype
    m = masses.to(dt).contiguous()
    sysi = system_idx.contiguous()
    ke = torch.empty(n_sys, dtype=torch.float64, device=p.device)
    ws = L.Workspace.get(p.device, L.load().tsb_thermostat_workspace_size(n_sys))
    L.call("tsb_kinetic_energy", L.ptr(p), L.ptr(m), L.ptr(sysi), p.shape[0], n_sys,
           L.dtype_code(dt), L.ptr(ke), L.ptr(ws), ws.numel(), L.stream_ptr(p.device))
    return 2.0 * ke


def calc_kinetic_energy(*, masses, momenta, system_idx, n_systems=None):
    n = n_systems if n_systems is not None else int(system_idx.max()) + 1
    return (0.5 * _sum_p2m(masses, momenta, system_idx, n)).to(momenta.dtype)


def calc_kT(*, masses, momenta, system_idx, dof_per_system=None, n_systems=None):
    n = n_systems if n_systems is not None else int(system_idx.max()) + 1
    s = _sum_p2m(masses, momenta, system_idx, n).to(momenta.dtype)
    if dof_per_system is None:
        dof_per_system = 3 * torch.bincount(system_idx, minlength=n)
    return s / dof_per_system


def system_wise_max_force(forces, system_idx, n_systems=None):
    n = n_systems if n_systems is not None else int(system_idx.max()) + 1
    out = torch.zeros(n, dtype=forces.dtype, device=forces.device)
    return out.scatter_reduce(0, system_idx, forces.norm(dim=1), reduce="amax")
