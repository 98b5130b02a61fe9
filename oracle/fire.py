"""FIRE + Frechet-cell-filter oracle (TEST INFRASTRUCTURE ONLY; never the product path).

FP64 numpy restatement of:

* ``fire_init``          <- torch_sim/optimizers/fire.py:21-114
* ``frechet_init``       <- torch_sim/optimizers/cell_filters.py:230-284
* ``fire_step`` (ASE)    <- fire.py:288-499 (_ase_fire_step)
* ``fire_step`` (VV)     <- fire.py:179-285 (_vv_fire_step)
* ``compute_cell_forces`` (Frechet branch) <- cell_filters.py:353-391, with
  ``_frechet_cell_forces`` (:142-178) and ``_clamp_deform_grad_log`` (:26-60)
* ``converged``          <- torch_sim/runners.py:501-538 and quantities.py:327-342

State is a dict of numpy arrays.  ``cell`` is the column-vector cell [S,3,3]
(state.py:138-142); ``model(positions, cell_col) -> (energy, forces, stress)``.
"""

from __future__ import annotations

import numpy as np

from . import linalg3

MAX_LOG_DEFORM = 2.0  # cell_filters.py:23


def _vdot(x, y, system_idx, n_sys):
    out = np.zeros(n_sys)
    np.add.at(out, system_idx, (x * y).sum(1))
    return out


def deform_grad(ref_col, cell_col):
    """F = cell_col @ inv(ref_col): solve(ref_row, cell_row)^T (cell_filters.py:137-139)."""
    ref_row = np.transpose(ref_col, (0, 2, 1))
    cell_row = np.transpose(cell_col, (0, 2, 1))
    return np.transpose(np.linalg.solve(ref_row, cell_row), (0, 2, 1))


def frechet_cell_forces(log_F, ucf):
    """sum_ab L_exp(log_F, E_mu,nu)[a,b] * ucf[a,b] over the 9 unit directions."""
    S = log_F.shape[0]
    dirs = np.zeros((9, 3, 3))
    for k in range(9):
        dirs[k, k // 3, k % 3] = 1.0
    A = np.repeat(log_F[:, None], 9, axis=1).reshape(-1, 3, 3)
    E = np.broadcast_to(dirs[None], (S, 9, 3, 3)).reshape(-1, 3, 3)
    _, L = linalg3.expm_frechet(A, E)
    L = L.reshape(S, 9, 3, 3)
    return (L * ucf[:, None]).sum(axis=(2, 3)).reshape(S, 3, 3)


def compute_cell_forces(st):
    """Frechet branch of compute_cell_forces; writes st['cell_forces']."""
    vol = np.linalg.det(st["cell"])[:, None, None]
    virial = -vol * (st["stress"] + st["pressure"])
    F = deform_grad(st["reference_cell"], st["cell"])
    ucf = virial @ np.linalg.inv(np.transpose(F, (0, 2, 1)))
    logF = np.clip(linalg3.logm(F), -MAX_LOG_DEFORM, MAX_LOG_DEFORM)
    st["cell_forces"] = frechet_cell_forces(logF, ucf) / st["cell_factor"][:, None, None]


def fire_init(st, model, *, dt_start=0.1, alpha_start=0.1, cell_filter=None,
              scalar_pressure=0.0):
    st = dict(st)
    e, f, s = model(st["positions"], st["cell"])
    n_sys = st["cell"].shape[0]
    st.update(energy=e, forces=f, stress=s,
              velocities=np.full_like(st["positions"], np.nan),
              dt=np.full(n_sys, dt_start), alpha=np.full(n_sys, alpha_start),
              n_pos=np.zeros(n_sys, dtype=np.int64))
    if cell_filter == "frechet":
        counts = np.bincount(st["system_idx"], minlength=n_sys).astype(np.float64)
        st["cell_factor"] = counts
        st["pressure"] = np.broadcast_to(scalar_pressure * np.eye(3), (n_sys, 3, 3)).copy()
        st["reference_cell"] = st["cell"].copy()
        st["cell_positions"] = np.zeros((n_sys, 3, 3))
        vol = np.linalg.det(st["cell"])[:, None, None]
        virial = -vol * (s + st["pressure"])
        F = deform_grad(st["reference_cell"], st["cell"])
        ucf = virial @ np.linalg.inv(np.transpose(F, (0, 2, 1)))
        st["cell_forces"] = ucf / counts[:, None, None]
        st["cell_velocities"] = np.full((n_sys, 3, 3), np.nan)
        st["cell_filter"] = "frechet"
    return st


def fire_step(st, model, *, dt_max=1.0, n_min=5, f_inc=1.1, f_dec=0.5, alpha_start=0.1,
              f_alpha=0.99, max_step=0.2, flavor="ase_fire", eps=1e-16):
    if flavor == "ase_fire":
        return _ase_step(dict(st), model, dt_max, n_min, f_inc, f_dec, alpha_start,
                         f_alpha, max_step, eps)
    return _vv_step(dict(st), model, dt_max, n_min, f_inc, f_dec, alpha_start,
                    f_alpha, eps)


def _update_params(st, pos_mask, n_min, f_inc, f_dec, dt_max, alpha_start, f_alpha,
                   inc_before_count):
    dt, alpha, n_pos = st["dt"].copy(), st["alpha"].copy(), st["n_pos"].copy()
    if not inc_before_count:  # VV ordering: count first (fire.py:231-233)
        n_pos[pos_mask] += 1
    inc = (n_pos > n_min) & pos_mask
    dt[inc] = np.minimum(dt[inc] * f_inc, dt_max)
    alpha[inc] *= f_alpha
    if inc_before_count:  # ASE ordering (fire.py:340-343)
        n_pos[pos_mask] += 1
    neg = ~pos_mask
    dt[neg] *= f_dec
    alpha[neg] = alpha_start
    n_pos[neg] = 0
    st.update(dt=dt, alpha=alpha, n_pos=n_pos)


def _ase_step(st, model, dt_max, n_min, f_inc, f_dec, alpha_start, f_alpha, max_step,
              eps):
    sysi = st["system_idx"]
    n_sys = st["cell"].shape[0]
    is_cell = "cell_filter" in st
    v = st["velocities"].copy()
    nan_atoms = np.isnan(v).any(axis=1)
    v = np.nan_to_num(v, nan=0.0)
    if is_cell:
        st["cell_velocities"] = np.nan_to_num(st["cell_velocities"], nan=0.0)
    forces = st["forces"]
    if not nan_atoms.all():
        power = _vdot(forces, v, sysi, n_sys)
        if is_cell:
            power = power + (st["cell_forces"] * st["cell_velocities"]).sum(axis=(1, 2))
        pos = power > 0.0
        _update_params(st, pos, n_min, f_inc, f_dec, dt_max, alpha_start, f_alpha, True)
        vs = _vdot(v, v, sysi, n_sys)
        fs = _vdot(forces, forces, sysi, n_sys)
        if is_cell:
            cv = st["cell_velocities"]
            cf = st["cell_forces"]
            vs = vs + (cv ** 2).sum(axis=(1, 2))
            fs = fs + (cf ** 2).sum(axis=(1, 2))
            mix_c = cf / (np.sqrt(fs)[:, None, None] + eps) * np.sqrt(vs)[:, None, None]
            a = st["alpha"][:, None, None]
            st["cell_velocities"] = np.where(pos[:, None, None],
                                             (1 - a) * cv + a * mix_c, 0.0)
        mix = forces * (np.sqrt(vs)[sysi] / (np.sqrt(fs)[sysi] + eps))[:, None]
        a = st["alpha"][sysi][:, None]
        v = np.where(pos[sysi][:, None], (1 - a) * v + a * mix, 0.0)
    dt_a = st["dt"][sysi][:, None]
    v = v + forces * dt_a
    dr = v * dt_a
    drs = _vdot(dr, dr, sysi, n_sys)
    if is_cell:
        dtc = st["dt"][:, None, None]
        st["cell_velocities"] = st["cell_velocities"] + st["cell_forces"] * dtc
        dr_cell = st["cell_velocities"] * dtc
        drs = drs + (dr_cell ** 2).sum(axis=(1, 2))
        sc = np.sqrt(drs)[:, None, None]
        dr_cell = np.where(sc > max_step, max_step * dr_cell / (sc + eps), dr_cell)
    sa = np.sqrt(drs)[sysi][:, None]
    dr = np.where(sa > max_step, max_step * dr / (sa + eps), dr)
    st["velocities"] = v
    if is_cell:
        F = deform_grad(st["reference_cell"], st["cell"])
        frac = np.linalg.solve(F[sysi], st["positions"][..., None])[..., 0]
        new_frac = frac + dr
        cp = st["cell_positions"] + dr_cell
        cf = st["cell_factor"][:, None, None]
        logF = cp / cf
        if (np.abs(logF) > MAX_LOG_DEFORM).any():
            logF = np.clip(logF, -MAX_LOG_DEFORM, MAX_LOG_DEFORM)
            cp = logF * cf
        Fn = linalg3.expm(logF)
        st["cell"] = Fn @ st["reference_cell"]
        Fa = deform_grad(st["reference_cell"], st["cell"])
        st["cell_positions"] = linalg3.logm(Fa) * cf
        st["positions"] = np.einsum("nij,nj->ni", Fa[sysi], new_frac)
    else:
        st["positions"] = st["positions"] + dr
    e, f, s = model(st["positions"], st["cell"])
    st.update(energy=e, forces=f, stress=s)
    if is_cell:
        compute_cell_forces(st)
    return st


def _vv_step(st, model, dt_max, n_min, f_inc, f_dec, alpha_start, f_alpha, eps):
    sysi = st["system_idx"]
    n_sys = st["cell"].shape[0]
    m = st["masses"][:, None]
    v = st["velocities"].copy()
    nan_atoms = np.isnan(v).any(axis=1)
    v[nan_atoms] = 0.0
    dt_a = st["dt"][sysi][:, None]
    v = v + 0.5 * dt_a * st["forces"] / m
    st["positions"] = st["positions"] + dt_a * v
    e, f, s = model(st["positions"], st["cell"])
    st.update(energy=e, forces=f, stress=s)
    v = v + 0.5 * dt_a * f / m
    power = _vdot(f, v, sysi, n_sys)
    pos = power > 0.0
    _update_params(st, pos, n_min, f_inc, f_dec, dt_max, alpha_start, f_alpha, False)
    vs = _vdot(v, v, sysi, n_sys)
    fs = _vdot(f, f, sysi, n_sys)
    mix = f * (np.sqrt(vs)[sysi] / (np.sqrt(fs)[sysi] + eps))[:, None]
    a = st["alpha"][sysi][:, None]
    st["velocities"] = np.where(pos[sysi][:, None], (1 - a) * v + a * mix, 0.0)
    return st


def max_force(forces, system_idx, n_sys):
    out = np.zeros(n_sys)
    np.maximum.at(out, system_idx, np.linalg.norm(forces, axis=1))
    return out


def converged(st, fmax, include_cell_forces=False):
    n_sys = st["cell"].shape[0]
    ok = max_force(st["forces"], st["system_idx"], n_sys) < fmax
    if include_cell_forces:
        ok &= np.linalg.norm(st["cell_forces"], axis=2).max(axis=1) < fmax
    return ok
