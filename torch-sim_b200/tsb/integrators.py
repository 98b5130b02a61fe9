"""MD step functions on the tsb kernels (drop-ins for torch_sim.integrators).

Signatures follow the reference registry entries (internal units, runners.py
converts user units, torch_sim/integrators/__init__.py:193-255):

* ``nve_init(state, model, *, kT)`` / ``nve_step(state, model, *, dt)``
  <- torch_sim/integrators/nve.py:19-130 (velocity Verlet)
* ``nvt_langevin_init(state, model, *, kT)`` /
  ``nvt_langevin_step(state, model, *, dt, kT, gamma=None)``
  <- torch_sim/integrators/nvt.py:89-240 (BAOAB, gamma default 1/(100 dt))
* ``initialize_momenta`` <- md.py:113-166
* ``nvt_nose_hoover_init/step/invariant`` <- nvt.py:244-562 (Nose-Hoover chains,
  md.py:249-563)
* ``nvt_vrescale_init/step`` <- nvt.py:565-741 (CSVR; ``step(model, state, ...)``)
* ``npt_langevin_isotropic_init/step`` <- npt.py:653-1107 (strain-based GJF barostat)

Steps mutate ``state`` in place and return it (md.py:184-187).  ``dt``, ``kT``
and ``gamma`` may be scalars or per-system tensors.

Langevin noise: by default the O-step draws counter-based Philox4x32-10
normals on the device (key = the state's seed, counter = its step count), so a
trajectory is reproducible from (seed, step).  Passing ``noise=[N,3]`` uses
those normals instead -- e.g. the reference's own ``torch.randn`` draws, which
makes one step agree with the reference to rounding.

``run_md`` is the persistent fused path: many steps of many systems in one
kernel launch (see csrc/tsb_fused.cu).
"""

from __future__ import annotations

import math

import torch

from . import _lib as L
from . import ops as _ops  # noqa: F401  (registers torch.ops.tsb.*)
from .state import MDState


def _per_system(x, n_sys: int, device) -> torch.Tensor:
    """Per-system float64 [S] on the device.  A scalar (Python number or a
    one-element CPU tensor) becomes a fill on the device, with no host-to-device
    copy, so the step functions can be captured in a CUDA graph."""
    if torch.is_tensor(x) and x.device.type == "cpu" and x.numel() == 1:
        x = float(x)
    if isinstance(x, (int, float)):
        return torch.full((n_sys,), float(x), dtype=torch.float64, device=device)
    t = torch.as_tensor(x, dtype=torch.float64, device=device)
    if t.ndim == 0:
        t = t.expand(n_sys)
    return t.contiguous()


def initialize_momenta(positions, masses, system_idx, kT, generator=None):
    """p = sqrt(m kT) N(0,1) minus the per-system mean (md.py:113-166).

    The normals are drawn on the generator's device (the positions' device when
    ``generator`` is None) and moved to the positions' device, so a CPU generator
    seeded as the reference seeds ``state.rng`` replays the reference's draw for
    a state that lives on the GPU."""
    kT = torch.as_tensor(kT, device=positions.device, dtype=positions.dtype)
    if kT.ndim > 0:
        kT = kT[system_idx]
    draw_dev = generator.device if generator is not None else positions.device
    z = torch.randn(positions.shape, device=draw_dev, dtype=positions.dtype,
                    generator=generator).to(positions.device)
    p = z * torch.sqrt(masses * kT).unsqueeze(-1)
    n_sys = int(system_idx[-1]) + 1
    counts = torch.bincount(system_idx, minlength=n_sys)
    # per-system sums from an FP64 prefix sum over the contiguous systems: a fixed
    # summation order (index_add_ on the GPU sums in a run-dependent order); the
    # scan runs along the contiguous dimension of p^T (a scan down the 3 columns
    # of p would be three long serial scans)
    cs = torch.cat([torch.zeros((3, 1), dtype=torch.float64, device=p.device),
                    p.to(torch.float64).T.contiguous().cumsum(1)], dim=1)
    ends = counts.cumsum(0)
    mean = ((cs[:, ends] - cs[:, ends - counts]) / counts.view(1, -1)).T.to(p.dtype)
    return torch.where((counts > 1)[system_idx].view(-1, 1), p - mean[system_idx], p)


def _i64(v: int) -> int:
    """A uint64 (seed, counter) as the signed int64 an operator argument holds."""
    v = int(v) & (2**64 - 1)
    return v - 2**64 if v >= 2**63 else v


def _seed_of(state) -> int:
    rng = getattr(state, "_rng", None)
    if isinstance(rng, int):
        return rng
    if isinstance(rng, torch.Generator):
        return int(rng.initial_seed())
    return 0


def _md_init(state, model, kT):
    out = model(state)
    kT_t = torch.as_tensor(kT, device=state.device, dtype=state.dtype)
    momenta = getattr(state, "momenta", None)
    if momenta is None:
        momenta = initialize_momenta(state.positions, state.masses, state.system_idx, kT_t,
                                     state.rng)
    md = MDState.from_state(state, momenta=momenta, energy=out["energy"],
                            forces=out["forces"])
    md._philox_seed = _seed_of(state)
    md._philox_counter = 0
    return md


def nve_init(state, model, *, kT, **_kw) -> MDState:
    return _md_init(state, model, kT)


def nvt_langevin_init(state, model, *, kT, **_kw) -> MDState:
    return _md_init(state, model, kT)


def _kick(state, dt_s, scale):
    torch.ops.tsb.md_kick_(state.momenta, state.forces, state.system_idx, dt_s, float(scale))


def _drift(state, dt_s, scale):
    torch.ops.tsb.md_drift_(state.positions, state.momenta, state.masses, state.system_idx,
                            dt_s, float(scale))


def use_device_counter(state, counter_dev: torch.Tensor | None = None):
    """Keep the state's Langevin noise counter on the device: every
    ``nvt_langevin_step`` then draws with counter ``state._philox_counter +
    counter_dev`` and advances ``counter_dev`` on the stream, so a step loop
    captured in a CUDA graph draws fresh noise on every replay.  Returns the
    counter tensor (int64 [1])."""
    if counter_dev is None:
        counter_dev = torch.zeros(1, dtype=torch.int64, device=state.device)
    state._philox_counter_dev = counter_dev
    return counter_dev


def _prepare(state):
    L.require_cuda(state.positions, "state.positions")
    for name in ("positions", "momenta", "forces", "masses"):
        t = getattr(state, name)
        if not t.is_contiguous() or t.dtype != state.dtype:
            setattr(state, name, t.to(state.dtype).contiguous())
    if not state.system_idx.is_contiguous():
        state.system_idx = state.system_idx.contiguous()


def _apply_model(state, model):
    out = model(state)
    state.energy = out["energy"]
    state.forces = out["forces"].contiguous()
    return out


def _update_forces(state, model):
    """Forces and energy of the new positions written into the state's own
    tensors when the model can (``forward_into``), so the tensors a step reads
    and writes keep their identity from step to step -- what lets a captured CUDA
    graph of several steps be replayed; otherwise the model's outputs replace
    them, as the reference's steps do (``state.forces = model_output["forces"]``)."""
    f, e = getattr(state, "forces", None), getattr(state, "energy", None)
    n_sys = state.n_systems
    if (hasattr(model, "forward_into") and torch.is_tensor(f) and torch.is_tensor(e)
            and f.is_contiguous() and e.is_contiguous() and f.shape == state.positions.shape
            and tuple(e.shape) == (n_sys,) and f.dtype == e.dtype == state.dtype
            and f.device == e.device == state.device):
        model.forward_into(state, energy=e, forces=f)
        return
    _apply_model(state, model)


def nve_step(state, model, *, dt, **_kw):
    """B(dt/2) A(dt) force B(dt/2) (nve.py:74-130)."""
    _prepare(state)
    dt_s = _per_system(dt, state.n_systems, state.device)
    _kick(state, dt_s, 0.5)
    _drift(state, dt_s, 1.0)
    _update_forces(state, model)
    _kick(state, dt_s, 0.5)
    return state


def nvt_langevin_step(state, model, *, dt, kT, gamma=None, noise=None, **_kw):
    """BAOAB: B(dt/2) A(dt/2) O(dt) A(dt/2) force B(dt/2) (nvt.py:144-240)."""
    _prepare(state)
    n_sys = state.n_systems
    dt_s = _per_system(dt, n_sys, state.device)
    kT_s = _per_system(kT, n_sys, state.device)
    if gamma is None:
        gamma = 1.0 / (100.0 * torch.as_tensor(dt, dtype=torch.float64))
    g_s = _per_system(gamma, n_sys, state.device)
    if noise is not None:
        noise = noise.to(device=state.device, dtype=state.dtype).contiguous()
    seed = getattr(state, "_philox_seed", _seed_of(state))
    counter = getattr(state, "_philox_counter", 0)
    counter_dev = getattr(state, "_philox_counter_dev", None)
    torch.ops.tsb.md_baoab_boa_(state.positions, state.momenta, state.forces, state.masses,
                                state.system_idx, dt_s, kT_s, g_s, noise, _i64(seed),
                                _i64(counter), counter_dev)
    state._philox_seed = seed
    if counter_dev is None:
        state._philox_counter = counter + 1
    _update_forces(state, model)
    _kick(state, dt_s, 0.5)
    return state


# ---------------------------------------------------------------------------
# NVT Nose-Hoover chains and V-rescale (CSVR)
# ---------------------------------------------------------------------------
def _dof(state) -> torch.Tensor:
    """3N - 3 per system (the COM motion removed, nvt.py:287-290, 355-357)."""
    counts = torch.bincount(state.system_idx, minlength=state.n_systems)
    dof = 3 * counts - 3
    if bool((dof <= 0).any()):
        raise ValueError("Degrees of freedom cannot be zero or negative")
    return dof.to(torch.float64)


def _thermo_ws(state):
    return L.Workspace.get(state.device,
                           L.load().tsb_thermostat_workspace_size(state.n_systems))


def kinetic_energy(state) -> torch.Tensor:
    """Per-system 1/2 sum p^2/m in FP64 on the device (quantities.py:104-139)."""
    ke = torch.empty(state.n_systems, dtype=torch.float64, device=state.device)
    ws = _thermo_ws(state)
    L.call("tsb_kinetic_energy", L.ptr(state.momenta), L.ptr(state.masses),
           L.ptr(state.system_idx), state.n_atoms, state.n_systems,
           L.dtype_code(state.dtype), L.ptr(ke), L.ptr(ws), ws.numel(),
           L.stream_ptr(state.device))
    return ke


def nvt_nose_hoover_init(state, model, *, kT, dt, tau=None, chain_length: int = 3,
                         chain_steps: int = 3, sy_steps: int = 3, **kwargs):
    """NVT Nose-Hoover-chain state (nvt.py:293-378): tau defaults to 10 dt, chain
    positions and momenta start at zero, Q_j = kT tau^2, Q_1 = dof kT tau^2."""
    from .state import NoseHooverChain, NVTNoseHooverState

    if not 1 <= chain_length <= 16:
        raise ValueError("chain_length must lie in 1..16")
    if sy_steps not in (1, 3, 5, 7):
        raise ValueError("sy_steps must be 1, 3, 5 or 7")
    if kwargs.get("momenta") is not None:
        state = MDState.from_state(state, momenta=kwargs["momenta"],
                                   energy=torch.zeros(state.n_systems, dtype=state.dtype,
                                                      device=state.device),
                                   forces=torch.zeros_like(state.positions))
    md = _md_init(state, model, kT)
    _prepare(md)
    n_sys, dev = md.n_systems, md.device
    dt_s = _per_system(dt, n_sys, dev)
    kT_s = _per_system(kT, n_sys, dev)
    tau_s = _per_system(10.0 * dt_s if tau is None else tau, n_sys, dev)
    dof = _dof(md)
    q = (kT_s * tau_s * tau_s).unsqueeze(-1).repeat(1, chain_length)
    q[:, 0] *= dof
    zeros = torch.zeros((n_sys, chain_length), dtype=torch.float64, device=dev)
    chain = NoseHooverChain(positions=zeros.clone(), momenta=zeros.clone(),
                            masses=q.contiguous(), tau=tau_s.clone(),
                            kinetic_energy=kinetic_energy(md), degrees_of_freedom=dof)
    out = NVTNoseHooverState.from_state(md, chain=chain, chain_steps=int(chain_steps),
                                        sy_steps=int(sy_steps), chain_dt=dt_s.clone())
    out._philox_seed, out._philox_counter = md._philox_seed, 0
    return out


def _nhc_half(state, kT_s, recompute: bool):
    c = state.chain
    ws = _thermo_ws(state)
    L.call("tsb_nhc_half_step", L.ptr(state.momenta), L.ptr(state.masses),
           L.ptr(state.system_idx), state.n_atoms, state.n_systems,
           L.dtype_code(state.dtype), L.ptr(c.positions), L.ptr(c.momenta), L.ptr(c.masses),
           L.ptr(c.kinetic_energy), L.ptr(c.degrees_of_freedom), L.ptr(kT_s), L.ptr(c.tau),
           L.ptr(state.chain_dt), c.positions.shape[1], state.chain_steps, state.sy_steps,
           int(recompute), L.ptr(ws), ws.numel(), L.stream_ptr(state.device))


def nvt_nose_hoover_step(state, model, *, dt, kT, **_kw):
    """NHC(dt/2) . velocity Verlet . NHC(dt/2) (nvt.py:381-488).  The chain
    masses follow kT on every step; the chain's own time step is the one it was
    initialised with."""
    _prepare(state)
    c = state.chain
    for name in ("positions", "momenta", "masses", "tau", "kinetic_energy",
                 "degrees_of_freedom"):
        t = getattr(c, name)
        if t.dtype != torch.float64 or not t.is_contiguous():
            setattr(c, name, t.to(torch.float64).contiguous())
    dt_s = _per_system(dt, state.n_systems, state.device)
    kT_s = _per_system(kT, state.n_systems, state.device)
    _nhc_half(state, kT_s, recompute=False)
    _kick(state, dt_s, 0.5)
    _drift(state, dt_s, 1.0)
    _update_forces(state, model)
    _kick(state, dt_s, 0.5)
    _nhc_half(state, kT_s, recompute=True)
    return state


def nvt_nose_hoover_invariant(state, kT) -> torch.Tensor:
    """Extended-system energy: E_pot + E_kin + sum_j p_xi_j^2 / (2 Q_j) + dof kT xi_1
    + kT sum_{j>1} xi_j (nvt.py:491-562)."""
    c = state.chain
    kT_s = _per_system(kT, state.n_systems, state.device)
    e = state.energy.to(torch.float64) + kinetic_energy(state)
    e = e + c.momenta[:, 0] ** 2 / (2 * c.masses[:, 0]) + c.degrees_of_freedom * kT_s * c.positions[:, 0]
    for j in range(1, c.positions.shape[1]):
        e = e + c.momenta[:, j] ** 2 / (2 * c.masses[:, j]) + kT_s * c.positions[:, j]
    return e


def nvt_vrescale_init(state, model, *, kT, **_kw):
    """V-rescale (CSVR) state (nvt.py:657-712)."""
    from .state import NVTVRescaleState

    md = _md_init(state, model, kT)
    out = NVTVRescaleState.from_state(md)
    out._philox_seed, out._philox_counter = md._philox_seed, 0
    return out


def nvt_vrescale_step(model, state, *, dt, kT, tau=None, noise=None, **_kw):
    """Rescale the momenta by the CSVR factor, then velocity Verlet
    (nvt.py:715-741; note the reference's argument order, model first).  tau
    defaults to 10 dt.  The normal r1 and the Gamma((dof - 1)/2) deviate are drawn
    on the device from the Philox stream (seed, system, step); ``noise`` [S, 2]
    = (r1, gamma deviate) supplies them instead, e.g. the reference's own draws."""
    _prepare(state)
    n_sys, dev = state.n_systems, state.device
    dt_s = _per_system(dt, n_sys, dev)
    kT_s = _per_system(kT, n_sys, dev)
    tau_s = _per_system(10.0 * dt_s if tau is None else tau, n_sys, dev)
    dof = _dof(state)
    if noise is not None:
        noise = torch.as_tensor(noise, dtype=torch.float64, device=dev).reshape(n_sys, 2)
        noise = noise.contiguous()
    seed = getattr(state, "_philox_seed", _seed_of(state))
    counter = getattr(state, "_philox_counter", 0)
    ws = _thermo_ws(state)
    L.call("tsb_vrescale", L.ptr(state.momenta), L.ptr(state.masses), L.ptr(state.system_idx),
           state.n_atoms, n_sys, L.dtype_code(state.dtype), L.ptr(dof), L.ptr(kT_s),
           L.ptr(tau_s), L.ptr(dt_s), L.ptr(noise), seed & (2**64 - 1), counter, None,
           L.ptr(ws), ws.numel(), L.stream_ptr(dev))
    state._philox_seed, state._philox_counter = seed, counter + 1
    _kick(state, dt_s, 0.5)
    _drift(state, dt_s, 1.0)
    _update_forces(state, model)
    _kick(state, dt_s, 0.5)
    return state


# ---------------------------------------------------------------------------
# Isotropic NPT Langevin
# ---------------------------------------------------------------------------
# ---------------------------------------------------------------------------
# Isotropic stochastic cell rescaling (C-rescale)
# ---------------------------------------------------------------------------
# eV / A^3 per bar (MetalUnits.pressure, torch_sim/units.py:100-113)
METAL_PRESSURE_BAR = 1e5 * 1e-30 / 1.6021766208e-19


def npt_crescale_init(state, model, *, kT, dt, tau_p=None, isothermal_compressibility=None,
                      **_kw):
    """C-rescale state (npt.py:2904-2986): tau_p = 3 dt and the isothermal
    compressibility 1e-6 bar^-1 by default; ``model`` must compute the stress."""
    from .state import NPTCRescaleState

    md = _md_init(state, model, kT)
    out = model(md)
    if "stress" not in out:
        raise ValueError("NPT needs a model with compute_stress=True")
    n_sys, dev = md.n_systems, md.device
    dt_s = _per_system(dt, n_sys, dev)
    tau_p = _per_system(3 * dt_s if tau_p is None else tau_p, n_sys, dev).clone()
    beta = _per_system(1e-6 / METAL_PRESSURE_BAR if isothermal_compressibility is None
                       else isothermal_compressibility, n_sys, dev).clone()
    cell0 = md.cell.clone()
    st = NPTCRescaleState.from_state(
        md, stress=out["stress"], isothermal_compressibility=beta, tau_p=tau_p,
        initial_cell=cell0, initial_cell_inv=torch.linalg.inv(cell0),
        initial_volume=torch.linalg.det(cell0))
    st._philox_seed, st._philox_counter = md._philox_seed, 0
    return st


def _vrescale(state, kT_s, tau_s, dt_s, noise, seed, counter):
    dev, n_sys = state.device, state.n_systems
    if noise is not None:
        noise = torch.as_tensor(noise, dtype=torch.float64, device=dev).reshape(n_sys, 2)
        noise = noise.contiguous()
    ws = _thermo_ws(state)
    L.call("tsb_vrescale", L.ptr(state.momenta), L.ptr(state.masses), L.ptr(state.system_idx),
           state.n_atoms, n_sys, L.dtype_code(state.dtype), L.ptr(_dof(state)), L.ptr(kT_s),
           L.ptr(tau_s), L.ptr(dt_s), L.ptr(noise), seed, counter, None, L.ptr(ws),
           ws.numel(), L.stream_ptr(dev))


def _crescale_step(state, model, *, dt, kT, external_pressure, tau, noise, n_baro, barostat):
    """V-rescale(dt/2), kick(dt/2), ``barostat``, forces, kick(dt/2), V-rescale(dt/2)."""
    _prepare(state)
    n_sys, dev = state.n_systems, state.device
    dt_s = _per_system(dt, n_sys, dev)
    kT_s = _per_system(kT, n_sys, dev)
    tau_s = _per_system(tau, n_sys, dev)
    half = (dt_s / 2).contiguous()
    for name in ("isothermal_compressibility", "tau_p"):
        v = getattr(state, name)
        if v.dtype != torch.float64 or not v.is_contiguous():
            setattr(state, name, v.to(torch.float64).contiguous())
    state.cell = state.cell.to(state.dtype).contiguous()
    state.stress = state.stress.to(state.dtype).contiguous()
    v1 = cn = v2 = None
    if noise is not None:
        v1, v2 = noise[0], noise[2]
        cn = torch.as_tensor(noise[1], dtype=torch.float64, device=dev)
        cn = cn.reshape(n_sys, n_baro).contiguous()
    seed = getattr(state, "_philox_seed", _seed_of(state)) & (2**64 - 1)
    counter = getattr(state, "_philox_counter", 0)
    _vrescale(state, kT_s, tau_s, half, v1, seed, counter)
    _kick(state, dt_s, 0.5)
    ws = L.Workspace.get(dev, L.load().tsb_npt_workspace_size(n_sys))
    barostat(state, kT_s, dt_s, cn, seed, counter, ws)
    out = _apply_model(state, model)
    state.stress = out["stress"].to(state.dtype).contiguous()
    _kick(state, dt_s, 0.5)
    _vrescale(state, kT_s, tau_s, half, v2, seed, counter + 1)
    state._philox_seed, state._philox_counter = seed, counter + 2
    return state


def _crescale_simple(entry, external_pressure):
    """Barostat call of the isotropic / anisotropic C-rescale entry points."""

    def call(state, kT_s, dt_s, cn, seed, counter, ws):
        p_s = _per_system(external_pressure, state.n_systems, state.device)
        L.call(entry, L.ptr(state.positions), L.ptr(state.momenta), L.ptr(state.masses),
               L.ptr(state.system_idx), state.n_atoms, state.n_systems,
               L.dtype_code(state.dtype), L.ptr(state.stress), L.ptr(state.cell),
               L.ptr(state.isothermal_compressibility), L.ptr(state.tau_p), L.ptr(kT_s),
               L.ptr(p_s), L.ptr(dt_s), L.ptr(cn), seed, counter, L.ptr(ws), ws.numel(),
               L.stream_ptr(state.device))

    return call


def _crescale_triclinic(external_pressure, average):
    """Barostat call of tsb_npt_crescale_tri; a [3, 3] or [S, 3, 3] external pressure
    takes the deviatoric correction (npt.py:2145-2183)."""

    def call(state, kT_s, dt_s, cn, seed, counter, ws):
        n_sys, dev = state.n_systems, state.device
        pe = torch.as_tensor(external_pressure, dtype=torch.float64, device=dev)
        pt = None
        if pe.ndim >= 2:
            if average:
                raise ValueError("the average-pressure variant takes a scalar pressure")
            pt = pe.expand(n_sys, 3, 3).reshape(n_sys, 9).contiguous()
            p_s = torch.zeros(n_sys, dtype=torch.float64, device=dev)
        else:
            p_s = _per_system(pe, n_sys, dev)
        ci = state.initial_cell_inv.to(torch.float64).reshape(n_sys, 9).contiguous()
        v0 = state.initial_volume.to(torch.float64).contiguous()
        L.call("tsb_npt_crescale_tri", L.ptr(state.positions), L.ptr(state.momenta),
               L.ptr(state.masses), L.ptr(state.system_idx), state.n_atoms, n_sys,
               L.dtype_code(state.dtype), L.ptr(state.stress), L.ptr(state.cell),
               L.ptr(state.isothermal_compressibility), L.ptr(state.tau_p), L.ptr(kT_s),
               L.ptr(p_s), L.ptr(pt), L.ptr(ci), L.ptr(v0), L.ptr(dt_s), int(average),
               L.ptr(cn), seed, counter, L.ptr(ws), ws.numel(), L.stream_ptr(dev))

    return call


def npt_crescale_triclinic_step(state, model, *, dt, kT, external_pressure, tau=None,
                                noise=None, **_kw):
    """One triclinic C-rescale step (npt.py:2517-2644; Del Tatto et al. 2022):
    matrix deformation from the traceless pressure tensor, Gram-Schmidt rotated to
    lower-triangular form; a tensor ``external_pressure`` takes the deviatoric
    correction.  tau defaults to dt.  ``noise = (vrescale_1 [S, 2], barostat
    [S, 11], vrescale_2 [S, 2])``, barostat = (volume normal, 3x3 normals
    row-major, volume normal)."""
    dt_s = _per_system(dt, state.n_systems, state.device)
    return _crescale_step(state, model, dt=dt, kT=kT, external_pressure=external_pressure,
                          tau=dt_s if tau is None else tau, noise=noise, n_baro=11,
                          barostat=_crescale_triclinic(external_pressure, False))


def npt_crescale_triclinic_average_step(state, model, *, dt, kT, external_pressure,
                                        tau=None, noise=None, **_kw):
    """One triclinic C-rescale step with the average kinetic pressure
    (3N - 3)/3 kT / V in place of the instantaneous one and unscaled momenta
    (npt.py:2376-2452, 2721-2796).  Arguments as npt_crescale_triclinic_step."""
    dt_s = _per_system(dt, state.n_systems, state.device)
    return _crescale_step(state, model, dt=dt, kT=kT, external_pressure=external_pressure,
                          tau=dt_s if tau is None else tau, noise=noise, n_baro=11,
                          barostat=_crescale_triclinic(external_pressure, True))


def npt_crescale_anisotropic_step(state, model, *, dt, kT, external_pressure, tau=None,
                                  noise=None, **_kw):
    """One anisotropic C-rescale step (npt.py:2645-2720): as the isotropic step with
    per-axis cell factors; the thermostat's tau defaults to 100 dt, as the reference's
    code does.  ``noise = (vrescale_1 [S, 2], barostat [S, 5], vrescale_2 [S, 2])``,
    barostat = (volume normal, z_x, z_y, z_z, volume normal)."""
    dt_s = _per_system(dt, state.n_systems, state.device)
    return _crescale_step(state, model, dt=dt, kT=kT, external_pressure=external_pressure,
                          tau=100 * dt_s if tau is None else tau, noise=noise, n_baro=5,
                          barostat=_crescale_simple("tsb_npt_crescale_aniso",
                                                    external_pressure))


def npt_crescale_isotropic_step(state, model, *, dt, kT, external_pressure, tau=None,
                                noise=None, **_kw):
    """One isotropic C-rescale step (npt.py:2797-2901; Bernetti & Bussi 2020):
    V-rescale(dt/2), kick(dt/2), barostat(dt), forces, kick(dt/2), V-rescale(dt/2).
    The thermostat's tau defaults to dt, as the reference's code does.  The draws
    (two V-rescale pairs (r1, Gamma deviate) and the barostat normal) come from
    the device Philox stream (seed, system, step); ``noise = (vrescale_1 [S, 2],
    cell [S], vrescale_2 [S, 2])`` supplies them instead."""
    dt_s = _per_system(dt, state.n_systems, state.device)
    return _crescale_step(state, model, dt=dt, kT=kT, external_pressure=external_pressure,
                          tau=dt_s if tau is None else tau, noise=noise, n_baro=1,
                          barostat=_crescale_simple("tsb_npt_crescale_iso", external_pressure))


# ---------------------------------------------------------------------------
# Isotropic NPT Nose-Hoover (MTK)
# ---------------------------------------------------------------------------
def _new_chain(n_sys, chain_length, dof, kT_s, tau_s, ke, dev):
    from .state import NoseHooverChain

    q = (kT_s * tau_s * tau_s).unsqueeze(-1).repeat(1, chain_length)
    q[:, 0] *= dof
    z = torch.zeros((n_sys, chain_length), dtype=torch.float64, device=dev)
    return NoseHooverChain(positions=z.clone(), momenta=z.clone(), masses=q.contiguous(),
                           tau=tau_s.clone(), kinetic_energy=ke.to(torch.float64).clone(),
                           degrees_of_freedom=dof.to(torch.float64).clone())


def npt_nose_hoover_isotropic_init(state, model, *, kT, dt, chain_length: int = 3,
                                   chain_steps: int = 2, sy_steps: int = 3, t_tau=None,
                                   b_tau=None, **kwargs):
    """MTK isotropic NPT state (npt.py:1642-1809): t_tau = 10 dt, b_tau = 100 dt,
    cell mass W = 3 (N + 1) kT b_tau^2, log volume and cell momentum zero; the
    particle chain sees 3N - 3 degrees of freedom, the cell chain 1."""
    from .state import NPTNoseHooverIsotropicState

    if not 1 <= chain_length <= 16:
        raise ValueError("chain_length must lie in 1..16")
    if sy_steps not in (1, 3, 5, 7):
        raise ValueError("sy_steps must be 1, 3, 5 or 7")
    if kwargs.get("momenta") is not None:
        state = MDState.from_state(state, momenta=kwargs["momenta"],
                                   energy=torch.zeros(state.n_systems, dtype=state.dtype,
                                                      device=state.device),
                                   forces=torch.zeros_like(state.positions))
    md = _md_init(state, model, kT)
    out = model(md)
    if "stress" not in out:
        raise ValueError("NPT needs a model with compute_stress=True")
    _prepare(md)
    n_sys, dev = md.n_systems, md.device
    dt_s = _per_system(dt, n_sys, dev)
    kT_s = _per_system(kT, n_sys, dev)
    t_tau_s = _per_system(10 * dt_s if t_tau is None else t_tau, n_sys, dev)
    b_tau_s = _per_system(100 * dt_s if b_tau is None else b_tau, n_sys, dev)
    n_at = torch.bincount(md.system_idx, minlength=n_sys).to(torch.float64)
    zs = torch.zeros(n_sys, dtype=torch.float64, device=dev)
    thermo = _new_chain(n_sys, chain_length, _dof(md), kT_s, t_tau_s, kinetic_energy(md), dev)
    baro = _new_chain(n_sys, chain_length, torch.ones_like(zs), kT_s, b_tau_s, zs, dev)
    st = NPTNoseHooverIsotropicState.from_state(
        md, stress=out["stress"], reference_cell=md.cell.to(torch.float64).clone(),
        cell_position=zs.clone(), cell_momentum=zs.clone().unsqueeze(-1),
        cell_mass=3 * (n_at + 1) * kT_s * b_tau_s * b_tau_s, thermostat=thermo,
        barostat=baro, chain_steps=int(chain_steps), sy_steps=int(sy_steps),
        chain_dt=dt_s.clone())
    return st


def _chain_half(c, momenta, masses, system_idx, n_items, n_sys, dtype, kT_s, chain_dt,
                chain_steps, sy_steps, recompute, dev):
    ws = L.Workspace.get(dev, L.load().tsb_thermostat_workspace_size(n_sys))
    L.call("tsb_nhc_half_step", L.ptr(momenta), L.ptr(masses), L.ptr(system_idx), n_items,
           n_sys, L.dtype_code(dtype), L.ptr(c.positions), L.ptr(c.momenta), L.ptr(c.masses),
           L.ptr(c.kinetic_energy), L.ptr(c.degrees_of_freedom), L.ptr(kT_s), L.ptr(c.tau),
           L.ptr(chain_dt), c.positions.shape[1], chain_steps, sy_steps, int(recompute),
           L.ptr(ws), ws.numel(), L.stream_ptr(dev))


def npt_nose_hoover_isotropic_step(state, model, *, dt, kT, external_pressure, **_kw):
    """One MTK isotropic NPT step (npt.py:1812-1963): cell chain and particle chain
    half steps, the inner step (cell-momentum half kick, exp(iL2) momenta, log-volume
    and exp(iL1) position updates, forces, exp(iL2), half kick), then the particle
    and cell chain half steps with freshly summed kinetic energies."""
    _prepare(state)
    n_sys, n, dev = state.n_systems, state.n_atoms, state.device
    dt_s = _per_system(dt, n_sys, dev)
    kT_s = _per_system(kT, n_sys, dev)
    p_s = _per_system(external_pressure, n_sys, dev)
    for c in (state.thermostat, state.barostat):
        for name in ("positions", "momenta", "masses", "tau", "kinetic_energy",
                     "degrees_of_freedom"):
            t = getattr(c, name)
            if t.dtype != torch.float64 or not t.is_contiguous():
                setattr(c, name, t.to(torch.float64).contiguous())
    for name in ("reference_cell", "cell_position"):
        setattr(state, name, getattr(state, name).to(torch.float64).contiguous())
    state.cell = state.cell.to(state.dtype).contiguous()
    state.stress = state.stress.to(state.dtype).contiguous()
    n_at = torch.bincount(state.system_idx, minlength=n_sys).to(torch.float64)
    b_tau = state.barostat.tau
    state.cell_mass = (3 * (n_at + 1) * kT_s * b_tau * b_tau).contiguous()
    # the cell momentum as a [S, 3] momentum array (p_eps, 0, 0) with mass W, one
    # item per system, for the chain kernel
    p3 = torch.zeros((n_sys, 3), dtype=state.dtype, device=dev)
    p3[:, 0] = state.cell_momentum.reshape(n_sys).to(state.dtype)
    w_mass = state.cell_mass.to(state.dtype).contiguous()
    sys_items = torch.arange(n_sys, dtype=torch.int64, device=dev)
    cd = state.chain_dt if state.chain_dt is not None else dt_s
    _chain_half(state.barostat, p3, w_mass, sys_items, n_sys, n_sys, state.dtype, kT_s, cd,
                state.chain_steps, state.sy_steps, False, dev)
    _chain_half(state.thermostat, state.momenta, state.masses, state.system_idx, n, n_sys,
                state.dtype, kT_s, cd, state.chain_steps, state.sy_steps, False, dev)
    p_eps = p3[:, 0].to(torch.float64).contiguous()
    v_eps = torch.empty(n_sys, dtype=torch.float64, device=dev)
    ws = L.Workspace.get(dev, L.load().tsb_npt_workspace_size(n_sys))
    dtc, stp = L.dtype_code(state.dtype), L.stream_ptr(dev)
    L.call("tsb_npt_nh_iso_pre", L.ptr(state.positions), L.ptr(state.momenta),
           L.ptr(state.forces), L.ptr(state.masses), L.ptr(state.system_idx), n, n_sys, dtc,
           L.ptr(state.stress), L.ptr(state.reference_cell), L.ptr(state.cell),
           L.ptr(state.cell_position), L.ptr(p_eps), L.ptr(state.cell_mass), L.ptr(p_s),
           L.ptr(dt_s), L.ptr(v_eps), L.ptr(ws), ws.numel(), stp)
    out = _apply_model(state, model)
    state.stress = out["stress"].to(state.dtype).contiguous()
    L.call("tsb_npt_nh_iso_post", L.ptr(state.momenta), L.ptr(state.forces),
           L.ptr(state.masses), L.ptr(state.system_idx), n, n_sys, dtc, L.ptr(state.stress),
           L.ptr(state.reference_cell), L.ptr(state.cell_position), L.ptr(p_eps), L.ptr(p_s),
           L.ptr(dt_s), L.ptr(v_eps), L.ptr(ws), ws.numel(), stp)
    _chain_half(state.thermostat, state.momenta, state.masses, state.system_idx, n, n_sys,
                state.dtype, kT_s, cd, state.chain_steps, state.sy_steps, True, dev)
    p3 = torch.zeros((n_sys, 3), dtype=state.dtype, device=dev)
    p3[:, 0] = p_eps.to(state.dtype)
    _chain_half(state.barostat, p3, w_mass, sys_items, n_sys, n_sys, state.dtype, kT_s, cd,
                state.chain_steps, state.sy_steps, True, dev)
    state.cell_momentum = p3[:, :1].to(torch.float64).clone()
    return state


def npt_nose_hoover_isotropic_invariant(state, kT, external_pressure) -> torch.Tensor:
    """Extended energy (npt.py:1966-2059): E_pot + E_kin + both chains' energies
    (particle chain with 3N - 3 degrees of freedom, cell chain with 1) + P V +
    p_eps^2 / (2 W)."""
    n_sys, dev = state.n_systems, state.device
    kT_s = _per_system(kT, n_sys, dev)
    p_s = _per_system(external_pressure, n_sys, dev)
    e = state.energy.to(torch.float64) + kinetic_energy(state)
    for c, dof in ((state.thermostat, _dof(state)),
                   (state.barostat, torch.ones(n_sys, dtype=torch.float64, device=dev))):
        e = e + c.momenta[:, 0] ** 2 / (2 * c.masses[:, 0]) + dof * kT_s * c.positions[:, 0]
        for j in range(1, c.positions.shape[1]):
            e = e + c.momenta[:, j] ** 2 / (2 * c.masses[:, j]) + kT_s * c.positions[:, j]
    e = e + p_s * torch.linalg.det(state.cell.to(torch.float64))
    return e + state.cell_momentum.reshape(n_sys) ** 2 / (2 * state.cell_mass)


def npt_langevin_anisotropic_init(state, model, *, kT, dt, alpha=None, cell_alpha=None,
                                  b_tau=None, **_kw):
    """Per-axis strain NPT Langevin state (npt.py:409-510): eps = 0 [S,3], alpha =
    1/(5 dt), cell_alpha = 1/(30 dt), b_tau = 300 dt by default.  ``model`` must
    compute the stress."""
    from .state import NPTLangevinAnisotropicState

    md = _md_init(state, model, kT)
    out = model(md)
    if "stress" not in out:
        raise ValueError("NPT needs a model with compute_stress=True")
    n_sys, dev = md.n_systems, md.device
    dt_s = _per_system(dt, n_sys, dev)
    kT_s = _per_system(kT, n_sys, dev)
    alpha = _per_system(1.0 / (5 * dt_s) if alpha is None else alpha, n_sys, dev).clone()
    cell_alpha = _per_system(1.0 / (30 * dt_s) if cell_alpha is None else cell_alpha,
                             n_sys, dev).clone()
    b_tau = _per_system(300 * dt_s if b_tau is None else b_tau, n_sys, dev).clone()
    n_at = torch.bincount(md.system_idx, minlength=n_sys).to(torch.float64)
    z = torch.zeros((n_sys, 3), dtype=torch.float64, device=dev)
    st = NPTLangevinAnisotropicState.from_state(
        md, stress=out["stress"], alpha=alpha, cell_alpha=cell_alpha, b_tau=b_tau,
        reference_cell=md.cell.to(torch.float64).clone(), cell_positions=z.clone(),
        cell_velocities=z.clone(), cell_masses=(n_at + 1) * kT_s * b_tau * b_tau)
    st._philox_seed, st._philox_counter = md._philox_seed, 0
    return st


def npt_langevin_anisotropic_step(state, model, *, dt, kT, external_pressure, noise=None,
                                  **_kw):
    """One per-axis NPT Langevin step (npt.py:513-650).  ``external_pressure`` is a
    scalar, a [3] vector or [S, 3]; the cell noise [S, 3] and particle noise [N, 3]
    come from the device Philox stream, or from ``noise = (cell_noise,
    particle_noise)``, e.g. the reference's own draws."""
    _prepare(state)
    n_sys, n, dev = state.n_systems, state.n_atoms, state.device
    dt_s = _per_system(dt, n_sys, dev)
    kT_s = _per_system(kT, n_sys, dev)
    pe = torch.as_tensor(external_pressure, dtype=torch.float64, device=dev)
    p3 = pe.reshape(1, 1).expand(n_sys, 3) if pe.ndim == 0 else pe.reshape(-1, 3).expand(n_sys, 3)
    p3 = p3.contiguous()
    for name in ("alpha", "cell_alpha", "b_tau", "reference_cell", "cell_positions",
                 "cell_velocities", "cell_masses"):
        v = getattr(state, name)
        if v.dtype != torch.float64 or not v.is_contiguous():
            setattr(state, name, v.to(torch.float64).contiguous())
    state.cell = state.cell.to(state.dtype).contiguous()
    state.stress = state.stress.to(state.dtype).contiguous()
    cn = pn = None
    if noise is not None:
        cn = torch.as_tensor(noise[0], dtype=torch.float64, device=dev).reshape(n_sys, 3)
        pn = torch.as_tensor(noise[1], dtype=torch.float64, device=dev).reshape(n, 3)
        cn, pn = cn.contiguous(), pn.contiguous()
    seed = getattr(state, "_philox_seed", _seed_of(state)) & (2**64 - 1)
    counter = getattr(state, "_philox_counter", 0)
    f_eps = torch.empty((n_sys, 3), dtype=torch.float64, device=dev)
    ws = L.Workspace.get(dev, L.load().tsb_npt_workspace_size(n_sys))
    dtc, stp = L.dtype_code(state.dtype), L.stream_ptr(dev)
    L.call("tsb_npt_langevin_aniso_pre", L.ptr(state.positions), L.ptr(state.momenta),
           L.ptr(state.forces), L.ptr(state.masses), L.ptr(state.system_idx), n, n_sys, dtc,
           L.ptr(state.stress), L.ptr(state.reference_cell), L.ptr(state.cell),
           L.ptr(state.cell_positions), L.ptr(state.cell_velocities), L.ptr(state.cell_masses),
           L.ptr(f_eps), L.ptr(state.alpha), L.ptr(state.cell_alpha), L.ptr(state.b_tau),
           L.ptr(kT_s), L.ptr(p3), L.ptr(dt_s), L.ptr(cn), L.ptr(pn), seed, counter,
           L.ptr(ws), ws.numel(), stp)
    forces_old = state.forces
    out = _apply_model(state, model)
    state.stress = out["stress"].to(state.dtype).contiguous()
    L.call("tsb_npt_langevin_aniso_post", L.ptr(state.momenta), L.ptr(state.masses),
           L.ptr(forces_old), L.ptr(state.forces), L.ptr(state.system_idx), n, n_sys, dtc,
           L.ptr(state.stress), L.ptr(state.cell), L.ptr(state.cell_velocities),
           L.ptr(state.cell_masses), L.ptr(f_eps), L.ptr(state.alpha), L.ptr(state.cell_alpha),
           L.ptr(kT_s), L.ptr(p3), L.ptr(dt_s), L.ptr(cn), L.ptr(pn), seed, counter,
           L.ptr(ws), ws.numel(), stp)
    state._philox_seed, state._philox_counter = seed, counter + 1
    return state


def npt_langevin_isotropic_init(state, model, *, kT, dt, alpha=None, cell_alpha=None,
                                b_tau=None, **_kw):
    """Strain-based isotropic NPT Langevin state (npt.py:888-985): eps = 0,
    alpha = 1/(5 dt), cell_alpha = 1/(30 dt), b_tau = 300 dt by default,
    Q = (N + 1) kT b_tau^2.  ``model`` must compute the stress."""
    from .state import NPTLangevinIsotropicState

    md = _md_init(state, model, kT)
    out = model(md)
    if "stress" not in out:
        raise ValueError("NPT needs a model with compute_stress=True")
    n_sys, dev = md.n_systems, md.device
    dt_s = _per_system(dt, n_sys, dev)
    kT_s = _per_system(kT, n_sys, dev)
    alpha = _per_system(1.0 / (5 * dt_s) if alpha is None else alpha, n_sys, dev).clone()
    cell_alpha = _per_system(1.0 / (30 * dt_s) if cell_alpha is None else cell_alpha,
                             n_sys, dev).clone()
    b_tau = _per_system(300 * dt_s if b_tau is None else b_tau, n_sys, dev).clone()
    n_at = torch.bincount(md.system_idx, minlength=n_sys).to(torch.float64)
    z = torch.zeros(n_sys, dtype=torch.float64, device=dev)
    st = NPTLangevinIsotropicState.from_state(
        md, stress=out["stress"], alpha=alpha, cell_alpha=cell_alpha, b_tau=b_tau,
        reference_cell=md.cell.to(torch.float64).clone(), cell_positions=z.clone(),
        cell_velocities=z.clone(), cell_masses=(n_at + 1) * kT_s * b_tau * b_tau)
    st._philox_seed, st._philox_counter = md._philox_seed, 0
    return st


def npt_langevin_isotropic_step(state, model, *, dt, kT, external_pressure, noise=None, **_kw):
    """One isotropic NPT Langevin step (npt.py:988-1107).  The cell noise [S] and the
    particle noise [N, 3] are drawn on the device from the Philox stream (seed,
    system / atom, step); ``noise = (cell_noise, particle_noise)`` supplies them
    instead, e.g. the reference's own draws."""
    _prepare(state)
    n_sys, n, dev = state.n_systems, state.n_atoms, state.device
    dt_s = _per_system(dt, n_sys, dev)
    kT_s = _per_system(kT, n_sys, dev)
    p_s = _per_system(external_pressure, n_sys, dev)
    for name in ("alpha", "cell_alpha", "b_tau", "reference_cell", "cell_positions",
                 "cell_velocities", "cell_masses"):
        v = getattr(state, name)
        if v.dtype != torch.float64 or not v.is_contiguous():
            setattr(state, name, v.to(torch.float64).contiguous())
    state.cell = state.cell.to(state.dtype).contiguous()
    state.stress = state.stress.to(state.dtype).contiguous()
    cn = pn = None
    if noise is not None:
        cn = torch.as_tensor(noise[0], dtype=torch.float64, device=dev).reshape(n_sys)
        pn = torch.as_tensor(noise[1], dtype=torch.float64, device=dev).reshape(n, 3)
        cn, pn = cn.contiguous(), pn.contiguous()
    seed = getattr(state, "_philox_seed", _seed_of(state)) & (2**64 - 1)
    counter = getattr(state, "_philox_counter", 0)
    f_eps = torch.empty(n_sys, dtype=torch.float64, device=dev)
    ws = L.Workspace.get(dev, L.load().tsb_npt_workspace_size(n_sys))
    dtc, stp = L.dtype_code(state.dtype), L.stream_ptr(dev)
    L.call("tsb_npt_langevin_iso_pre", L.ptr(state.positions), L.ptr(state.momenta),
           L.ptr(state.forces), L.ptr(state.masses), L.ptr(state.system_idx), n, n_sys, dtc,
           L.ptr(state.stress), L.ptr(state.reference_cell), L.ptr(state.cell),
           L.ptr(state.cell_positions), L.ptr(state.cell_velocities), L.ptr(state.cell_masses),
           L.ptr(f_eps), L.ptr(state.alpha), L.ptr(state.cell_alpha), L.ptr(state.b_tau),
           L.ptr(kT_s), L.ptr(p_s), L.ptr(dt_s), L.ptr(cn), L.ptr(pn), seed, counter,
           L.ptr(ws), ws.numel(), stp)
    forces_old = state.forces
    out = _apply_model(state, model)
    state.stress = out["stress"].to(state.dtype).contiguous()
    L.call("tsb_npt_langevin_iso_post", L.ptr(state.momenta), L.ptr(state.masses),
           L.ptr(forces_old), L.ptr(state.forces), L.ptr(state.system_idx), n, n_sys, dtc,
           L.ptr(state.stress), L.ptr(state.reference_cell), L.ptr(state.cell_positions),
           L.ptr(state.cell_velocities), L.ptr(state.cell_masses), L.ptr(f_eps),
           L.ptr(state.alpha), L.ptr(state.cell_alpha), L.ptr(kT_s), L.ptr(p_s), L.ptr(dt_s),
           L.ptr(cn), L.ptr(pn), seed, counter, L.ptr(ws), ws.numel(), stp)
    state._philox_seed, state._philox_counter = seed, counter + 1
    return state


# ---------------------------------------------------------------------------
# Persistent fused batched MD
# ---------------------------------------------------------------------------
class FusedMDError(RuntimeError):
    pass


def _system_order(state):
    """Largest systems first (longest-processing-time order balances the tail)."""
    cache = getattr(state, "_tsb_order", None)
    key = (state.system_idx.data_ptr(), state.n_atoms)
    if cache is not None and cache[0] == key:
        return cache[1], cache[2]
    counts = torch.bincount(state.system_idx, minlength=state.n_systems)
    order = torch.argsort(counts, descending=True, stable=True).to(torch.int32).contiguous()
    max_atoms = int(counts.max())
    try:
        state._tsb_order = (key, order, max_atoms)
    except AttributeError:
        pass
    return order, max_atoms


NARROW_MAX_ATOMS = 256      # systems the 256-thread blocks of the fused kernel take
PRUNE_FRACTION = 0.375      # default pruning skin of the fused kernel, relative to its skin
NARROW_MAX_IMAGES = 1968    # their table of atoms + periodic images


def _split_order(state, cutoff: float, skin: float):
    """(order, n_wide): systems for 512-thread blocks first, then those for the
    256-thread blocks (two per SM), each group largest first.  A system goes to
    the narrow blocks when it has at most 256 atoms and its atoms and images
    within cutoff + skin of the cell -- about n prod_k (1 + 2 R / d_k), d_k the
    cell's plane spacings -- fit 95 % of their table (an underestimate only
    costs that system a smaller skin: it shrinks until its tables fit)."""
    counts = torch.bincount(state.system_idx, minlength=state.n_systems).to(torch.float64)
    cell_row = state.cell.mT.to(torch.float64)
    recip = torch.linalg.inv(cell_row).mT          # rows: reciprocal vectors, |b_k| = 1/d_k
    h = (cutoff + skin) * recip.norm(dim=-1)       # [S, 3] image margins, fractional
    images = counts * torch.prod(1.0 + 2.0 * h, dim=-1)
    narrow = (counts <= NARROW_MAX_ATOMS) & (images <= 0.95 * NARROW_MAX_IMAGES)
    key = torch.where(narrow, counts, counts + 1e6)  # wide ones sort first
    order = torch.argsort(key, descending=True, stable=True).to(torch.int32).contiguous()
    return order, int((~narrow).sum())


class FusedMD:
    """Preallocated persistent fused-MD runner (no host synchronisation per launch).

    Holds FP64 copies of positions/momenta/forces and every buffer the C ABI
    needs, so :meth:`launch` is a single ``tsb_fused_md`` call that can be
    timed, overlapped or replayed; :meth:`check` synchronises and raises on a
    device-reported failure; :meth:`write_back` copies the results into the
    state.
    """

    def __init__(self, state, model, *, integrator: str = "nvt_langevin", dt, kT=None,
                 gamma=None, skin: float | str = 0.7, seed: int | None = None, tau=None,
                 lanes: int | str | None = None, shapes: str = "auto",
                 prune: float | str | None = None):
        from .models.pair_potential import PairTableModel

        if not isinstance(model, PairTableModel):
            raise TypeError("the fused path needs a tsb PairTableModel (LJ / Morse / soft sphere)")
        self.integ = {"nve": L.INT_NVE, "nvt_langevin": L.INT_LANGEVIN,
                      "nvt_nose_hoover": L.INT_NOSE_HOOVER,
                      "nvt_vrescale": L.INT_VRESCALE}[integrator]
        L.require_cuda(state.positions, "state.positions")
        if not bool(torch.as_tensor(state.pbc).all()):
            raise FusedMDError("the fused path requires periodic boundaries on all axes")
        self.state, self.model = state, model
        dev = self.dev = state.device
        self.n, self.n_sys = state.n_atoms, state.n_systems
        self.order, max_atoms = _system_order(state)
        self.lib = L.load()
        if max_atoms > self.lib.tsb_fused_max_atoms():
            raise FusedMDError(f"systems with {max_atoms} atoms exceed the fused-kernel "
                               f"limit of {self.lib.tsb_fused_max_atoms()}")
        self.dt_s = _per_system(dt, self.n_sys, dev)
        if self.integ in (L.INT_NOSE_HOOVER, L.INT_VRESCALE):
            if kT is None:
                raise ValueError(f"kT is required for {integrator}")
            _dof(state)  # every system needs >= 2 atoms (3N - 3 > 0)
            self.kT_s = _per_system(kT, self.n_sys, dev)
            self.g_s = None
            if self.integ == L.INT_NOSE_HOOVER:
                c = getattr(state, "chain", None)
                if c is None:
                    raise TypeError("nvt_nose_hoover needs a state from nvt_nose_hoover_init")
                f64c = lambda t: t.to(torch.float64).contiguous().clone()  # noqa: E731
                self.cxi, self.cpxi = f64c(c.positions), f64c(c.momenta)
                self.cQ, self.cke = f64c(c.masses), f64c(c.kinetic_energy)
                self.tau_s = f64c(c.tau)
                self.cdt = f64c(state.chain_dt)
                self.M, self.nc, self.nsy = c.positions.shape[1], state.chain_steps, state.sy_steps
            else:
                self.tau_s = _per_system(10.0 * self.dt_s if tau is None else tau,
                                         self.n_sys, dev)
        elif self.integ == L.INT_LANGEVIN:
            if kT is None:
                raise ValueError("kT is required for nvt_langevin")
            self.kT_s = _per_system(kT, self.n_sys, dev)
            if gamma is None:
                gamma = 1.0 / (100.0 * torch.as_tensor(dt, dtype=torch.float64))
            self.g_s = _per_system(gamma, self.n_sys, dev)
        else:
            self.kT_s = self.g_s = None
        f64 = torch.float64
        self.x = state.positions.to(f64).contiguous().clone()
        self.p = state.momenta.to(f64).contiguous().clone()
        self.f = state.forces.to(f64).contiguous().clone()
        self.m = state.masses.to(f64).contiguous()
        self.cell_row = state.cell.mT.to(f64).contiguous()
        self.sys_idx = state.system_idx.contiguous()
        self.species = model._species(state.atomic_numbers)
        self.table = model.table if model.table.device == dev else model.table.to(dev)
        self.energy = torch.zeros(self.n_sys, dtype=f64, device=dev)
        self.stress = torch.zeros((self.n_sys, 3, 3), dtype=f64, device=dev)
        self.rebuilds = torch.zeros(self.n_sys, dtype=torch.int32, device=dev)
        self.status = torch.zeros(4, dtype=torch.int32, device=dev)
        self.ws = torch.empty(self.lib.tsb_fused_workspace_size(self.n, self.n_sys),
                              dtype=torch.uint8, device=dev)
        if isinstance(skin, str):
            if skin != "auto":
                raise ValueError(f"skin must be a number or 'auto', got {skin!r}")
            from .autotune import tune_fused_skin

            skin = tune_fused_skin(state, model, integrator=integrator, dt=dt, kT=kT,
                                   gamma=gamma)
            if lanes is None:
                lanes = "auto"
            if prune is None:
                prune = "auto"
        self.skin = float(skin)
        # pruning skin of the list's shell (Angstrom; 0: off): None is a fixed
        # fraction of the skin, "auto" the project autotuner
        if prune is None:
            prune = PRUNE_FRACTION * self.skin
        elif prune == "auto":
            from .autotune import tune_fused_prune

            prune = tune_fused_prune(state, model, skin=self.skin, integrator=integrator,
                                     dt=dt, kT=kT, gamma=gamma)
        elif isinstance(prune, str):
            raise ValueError(f"prune must be a number, None or 'auto', got {prune!r}")
        if not (float(prune) >= 0.0 and math.isfinite(float(prune))):
            raise ValueError(f"prune must be >= 0, got {prune!r}")
        self.prune = float(prune)
        # threads per atom at most (small systems); "auto": the project autotuner
        self.lanes = 32 if lanes is None else lanes
        if self.lanes == "auto":
            from .autotune import tune_fused_lanes

            self.lanes = tune_fused_lanes(state, model, skin=self.skin, integrator=integrator,
                                          dt=dt, kT=kT, gamma=gamma, prune=self.prune)
        if self.lanes not in (1, 2, 4, 8, 16, 32):
            raise ValueError(f"lanes must be a power of two in 1..32, got {self.lanes!r}")
        # block shapes: "auto" puts small systems in 256-thread blocks (two per
        # SM) and the rest in 512-thread blocks; "wide" runs all in 512-thread blocks
        if shapes not in ("auto", "wide"):
            raise ValueError(f"shapes must be 'auto' or 'wide', got {shapes!r}")
        self.shapes = shapes
        if shapes == "auto":
            self.order, self.n_wide = _split_order(state, model.cutoff, self.skin)
        else:
            self.n_wide = -1
        self.seed = (seed if seed is not None
                     else getattr(state, "_philox_seed", _seed_of(state))) & (2**64 - 1)
        # Philox counter lives on the device so that graph replays advance it
        self.counter_dev = torch.tensor([getattr(state, "_philox_counter", 0)],
                                        dtype=torch.int64, device=dev)
        self._graphs = {}

    @property
    def counter(self) -> int:
        return int(self.counter_dev.item())

    def launch(self, n_steps: int, stream: int | None = None, frames=None) -> None:
        """Advance every system by n_steps in one persistent launch (on the current
        stream; ``stream`` is accepted for compatibility and must be None or the
        current stream).  ``frames`` = (frame_x float32 [F, N, 3], frame_e float64
        [F, S], report_every) makes the kernel write positions and potential
        energies every report_every steps (F frames at most)."""
        if stream is not None and stream != L.stream_ptr(self.dev):
            raise ValueError("FusedMD.launch runs on the current CUDA stream")
        m = self.model
        nh = self.integ == L.INT_NOSE_HOOVER
        g = (lambda name: getattr(self, name, None) if nh else None)  # noqa: E731
        fx, fe, every = frames if frames is not None else (None, None, 0)
        torch.ops.tsb.fused_md_(
            self.integ, m.kind, self.table, m.n_species, self.species, self.x, self.p, self.f,
            self.m, self.cell_row, self.sys_idx, self.order, m.cutoff, self.skin, int(n_steps),
            self.dt_s, self.kT_s, self.g_s, getattr(self, "tau_s", None), g("cxi"), g("cpxi"),
            g("cQ"), g("cke"), g("cdt"), self.M if nh else 0, self.nc if nh else 0,
            self.nsy if nh else 0, _i64(self.seed), 0, self.counter_dev, fx, fe, int(every),
            self.lanes, self.n_wide, self.prune, self.energy, self.stress, self.rebuilds,
            self.status, self.ws)

    def graph(self, n_steps: int) -> "torch.cuda.CUDAGraph":
        """CUDA graph of one ``launch(n_steps)``; ``g.replay()`` advances every system
        by n_steps with fresh Langevin noise (the device counter moves on)."""
        if n_steps not in self._graphs:
            torch.cuda.synchronize(self.dev)
            keep = [self.x, self.p, self.f, self.counter_dev]
            if self.integ == L.INT_NOSE_HOOVER:
                keep += [self.cxi, self.cpxi, self.cQ, self.cke]
            saved = [t.clone() for t in keep]
            s = torch.cuda.Stream(self.dev)
            s.wait_stream(torch.cuda.current_stream(self.dev))
            with torch.cuda.stream(s):  # warm-up outside capture (sets kernel attributes)
                self.launch(n_steps)
            torch.cuda.current_stream(self.dev).wait_stream(s)
            torch.cuda.synchronize(self.dev)
            for t, v in zip(keep, saved):
                t.copy_(v)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self.launch(n_steps)
            self._graphs[n_steps] = g
        return self._graphs[n_steps]

    def check(self) -> None:
        st = self.status.tolist()
        if st[0] != 0:
            what = {1: "periodic images", 2: "neighbour slots",
                    3: "system index of atom"}.get(st[2], "atoms")
            raise FusedMDError(f"fused MD: system {st[1]}: {L.status_string(st[0])} "
                               f"({what}: {st[3]})")

    def write_back(self):
        s = self.state
        dt_in = s.positions.dtype
        cast = (lambda t: t.clone()) if dt_in == torch.float64 else (lambda t: t.to(dt_in))
        s.positions, s.momenta, s.forces = cast(self.x), cast(self.p), cast(self.f)
        s.energy = cast(self.energy)
        s._philox_seed, s._philox_counter = self.seed, self.counter
        if self.integ == L.INT_NOSE_HOOVER:
            c = s.chain
            c.positions, c.momenta = self.cxi.clone(), self.cpxi.clone()
            c.masses, c.kinetic_energy = self.cQ.clone(), self.cke.clone()
        return s


def _scatter_back(state, sub, systems, chain: bool):
    """Write a sub-state's per-atom and per-system results into ``state``."""
    dev = state.device
    sel = torch.as_tensor(sorted(systems), dtype=torch.long, device=dev)
    keep = torch.zeros(state.n_systems, dtype=torch.bool, device=dev)
    keep[sel] = True
    atoms = keep[state.system_idx]
    for name in ("positions", "momenta", "forces"):
        getattr(state, name)[atoms] = getattr(sub, name).to(getattr(state, name).dtype)
    state.energy[sel] = sub.energy.to(state.energy.dtype)
    if chain:
        for name in ("positions", "momenta", "masses", "kinetic_energy"):
            getattr(state.chain, name)[sel] = getattr(sub.chain, name)


def _run_fused(state, model, n_steps, integrator, dt, kT, gamma, skin, seed, check, tau,
               prune=None):
    r = FusedMD(state, model, integrator=integrator, dt=dt, kT=kT, gamma=gamma, skin=skin,
                seed=seed, tau=tau, prune=prune)
    r.launch(n_steps)
    if check:
        r.check()
    r.write_back()
    return r.rebuilds


def _run_per_call(state, model, n_steps, integrator, dt, kT, gamma, seed, tau):
    """Systems too large for the fused kernel: the per-call step functions."""
    if seed is not None:
        state._philox_seed = seed
    for _ in range(n_steps):
        if integrator == "nve":
            nve_step(state, model, dt=dt)
        elif integrator == "nvt_langevin":
            nvt_langevin_step(state, model, dt=dt, kT=kT, gamma=gamma)
        elif integrator == "nvt_vrescale":
            nvt_vrescale_step(model, state, dt=dt, kT=kT, tau=tau)
        else:
            nvt_nose_hoover_step(state, model, dt=dt, kT=kT)
    return state


def run_md(state, model, n_steps: int, *, integrator: str = "nvt_langevin", dt, kT=None,
           gamma=None, skin: float | str = 0.7, seed: int | None = None, check: bool = True,
           return_rebuilds: bool = False, tau=None, max_memory_scaler: float | None = None,
           memory_scales_with: str = "n_atoms_x_density", prune: float | str | None = None):
    """Advance every system ``n_steps`` in ONE persistent kernel launch.

    Same update rules as ``nve_step`` / ``nvt_langevin_step`` (Langevin noise
    from the Philox stream) / ``nvt_nose_hoover_step`` (state from
    ``nvt_nose_hoover_init``; its chain is updated) / ``nvt_vrescale_step`` (``tau``,
    default 10 dt; same Philox draws as the step function), with a device-side
    Verlet list (cutoff + skin)
    rebuilt when any atom of a system moved more than skin/2; between builds only
    the list's pairs within cutoff + ``prune`` are evaluated (re-pruned when an
    atom moved more than prune/2; default a fixed fraction of the skin, 0 off,
    "auto" tuned).  ``model`` must be
    a :class:`tsb.models.PairTableModel` (LJ / Morse / soft sphere, any species
    table); all axes must be periodic.  ``state`` is updated in place
    (positions, momenta, forces, energy).

    Admission (the reference autobatcher's role, torch_sim/autobatching.py:475-765):
    systems with more atoms than ``tsb_fused_max_atoms()`` (512) advance through
    the per-call step functions instead of the fused kernel; with
    ``max_memory_scaler`` the other systems run in launches whose summed memory
    cost (``memory_scales_with``, see ``tsb.autobatching``) stays below it.
    ``return_rebuilds`` gives per-system list builds (-1 for systems advanced per
    call).
    """
    counts = torch.bincount(state.system_idx, minlength=state.n_systems)
    big = counts > L.load().tsb_fused_max_atoms()
    any_big = bool(big.any())
    if not any_big and max_memory_scaler is None:
        rebuilds = _run_fused(state, model, n_steps, integrator, dt, kT, gamma, skin, seed,
                              check, tau, prune)
        return (state, rebuilds) if return_rebuilds else state
    from .autobatching import BinningAutoBatcher
    from .state import select_systems

    if any_big and integrator == "nvt_nose_hoover":
        raise FusedMDError("systems above the fused-kernel limit need nve, nvt_langevin or "
                           "nvt_vrescale")
    chain = integrator == "nvt_nose_hoover"
    rebuilds = torch.full((state.n_systems,), -1, dtype=torch.int32, device=state.device)
    small_idx = torch.nonzero(~big).flatten().tolist()
    big_idx = torch.nonzero(big).flatten().tolist()
    if small_idx:
        sub = select_systems(state, small_idx) if any_big else state
        if max_memory_scaler is None:
            groups = [(sub, list(range(len(small_idx))))]
        else:
            ab = BinningAutoBatcher(model, memory_scales_with=memory_scales_with,
                                    max_memory_scaler=max_memory_scaler)
            ab.load_states(sub)
            groups = list(ab)
        for part, idx in groups:
            if part is not sub:
                for k in ("_philox_seed", "_philox_counter"):
                    if hasattr(sub, k):
                        setattr(part, k, getattr(sub, k))
            rb = _run_fused(part, model, n_steps, integrator, dt, kT, gamma, skin, seed, check,
                            tau, prune)
            if part is not sub:
                _scatter_back(sub, part, idx, chain)
            rebuilds[torch.as_tensor([small_idx[i] for i in idx], device=state.device)] = rb
        if sub is not state:
            _scatter_back(state, sub, small_idx, chain)
    if big_idx:
        sub = select_systems(state, big_idx)
        for k in ("_philox_seed", "_philox_counter"):
            if hasattr(state, k):
                setattr(sub, k, getattr(state, k))
        _run_per_call(sub, model, n_steps, integrator, dt, kT, gamma, seed, tau)
        _scatter_back(state, sub, big_idx, chain)
    return (state, rebuilds) if return_rebuilds else state
