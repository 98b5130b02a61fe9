"""Isotropic NPT Langevin oracle (TEST INFRASTRUCTURE ONLY; never the product path).

FP64 numpy restatement of the reference's strain-based isotropic NPT Langevin
step (Gronbech-Jensen & Farago GJF scheme), noise passed in:

* ``cell_force``          <- torch_sim/integrators/npt.py:704-749
                             F_eps = 3 V (P_avg - P_ext), P_avg = -tr(sigma)/3 + N kT / V
* ``npt_langevin_isotropic_step`` <- npt.py:988-1107 with the helpers
  ``_npt_langevin_isotropic_cell_position_step`` (:769-798),
  ``_npt_langevin_isotropic_position_step`` (:838-885),
  ``_npt_langevin_isotropic_cell_velocity_step`` (:801-835),
  ``_npt_langevin_particle_velocity_step`` (:316-367),
  cell = exp(eps) reference_cell, V = det(reference_cell) exp(3 eps) (:690-703)
* ``npt_langevin_anisotropic_step`` <- npt.py:513-650 (per-axis strains; cell
  force :370-406, strain steps :201-264, position step :267-313)
* ``npt_nose_hoover_isotropic_step`` <- npt.py:1812-1963 (MTK: chain half steps of
  md.py:388-514, inner step :1532-1639 with exp_iL1 :1346-1399, exp_iL2 :1402-1457,
  cell force :1460-1529, sinh(x)/x series :1312-1343)
* ``npt_crescale_isotropic_step`` <- npt.py:2797-2901 (V-rescale half steps of
  nvt.py:594-654, momentum half steps, ``_crescale_isotropic_barostat_step``
  :2455-2492 with the instantaneous pressure of quantities.py:156-198)
* ``npt_crescale_anisotropic_step`` <- npt.py:2645-2720 with
  ``_crescale_anisotropic_barostat_step`` (:2282-2343)
* ``npt_crescale_triclinic_step`` <- npt.py:2517-2644 with
  ``_crescale_triclinic_barostat_step`` (:2186-2280), ``_compute_deviatoric_correction``
  (:2145-2183), ``rotate_gram_schmidt`` (:2093-2126); ``average=True`` gives
  ``npt_crescale_triclinic_average_step`` (:2721-2796, barostat :2376-2452)
"""

from __future__ import annotations

import numpy as np

from . import md as omd
from . import thermostats as oth


def cell_force(stress, vol, n_atoms, kT, p_ext):
    p_avg = -np.einsum("sii->s", stress) / 3.0 + n_atoms * kT / vol
    return 3.0 * vol * (p_avg - p_ext)


def npt_langevin_isotropic_step(st, force_fn, dt, kT, p_ext, cell_noise, particle_noise,
                                system_idx):
    """st: dict positions, momenta, masses, forces, stress, cell_positions (eps),
    cell_velocities, alpha, cell_alpha, b_tau, reference_cell.  force_fn(q, cell)
    -> (energy, forces, stress)."""
    st = dict(st)
    n_sys = len(st["cell_positions"])
    n_at = np.bincount(system_idx, minlength=n_sys).astype(np.float64)
    q_mass = (n_at + 1) * kT * st["b_tau"] ** 2
    v0 = np.linalg.det(st["reference_cell"])
    eps_old = st["cell_positions"].copy()
    vol = v0 * np.exp(3 * eps_old)
    f_n = cell_force(st["stress"], vol, n_at, kT, p_ext)
    beta_c = np.sqrt(2.0 * st["cell_alpha"] * kT * dt) * cell_noise
    a_at = st["alpha"][system_idx]
    beta_p = np.sqrt(2 * a_at * kT * dt)[:, None] * particle_noise
    # strain position step
    q2 = 2 * q_mass
    cb = 1 / (1 + st["cell_alpha"] * dt / q2)
    eps = eps_old + cb * dt * st["cell_velocities"] + cb * dt * dt * f_n / q2 + cb * dt * beta_c / q2
    cell = np.exp(eps)[:, None, None] * st["reference_cell"]
    # particle position step with box scaling
    m = st["masses"]
    scale = np.exp(eps - eps_old)[system_idx]
    b = 1 / (1 + a_at * dt / (2 * m))
    vel = st["momenta"] / m[:, None]
    c3 = vel + dt * st["forces"] / (2 * m[:, None]) + beta_p / (2 * m[:, None])
    q = scale[:, None] * st["positions"] + ((2 * scale / (scale + 1)) * b * dt)[:, None] * c3
    forces_old = st["forces"]
    e, f, s = force_fn(q, cell)
    vol = v0 * np.exp(3 * eps)
    f_new = cell_force(s, vol, n_at, kT, p_ext)
    qm = q_mass
    ac = (1 - st["cell_alpha"] * dt / (2 * qm)) / (1 + st["cell_alpha"] * dt / (2 * qm))
    bc = 1 / (1 + st["cell_alpha"] * dt / (2 * qm))
    eps_dot = ac * st["cell_velocities"] + dt * (ac * f_n + f_new) / (2 * qm) + bc * beta_c / qm
    m2 = 2 * m
    ap = ((1 - a_at * dt / m2) / (1 + a_at * dt / m2))[:, None]
    bp = (1 / (1 + a_at * dt / m2))[:, None]
    v_new = ap * vel + dt * (ap * forces_old + f) / m2[:, None] + bp * beta_p / m[:, None]
    st.update(positions=q, momenta=v_new * m[:, None], forces=f, energy=e, stress=s, cell=cell,
              cell_positions=eps, cell_velocities=eps_dot, cell_masses=q_mass)
    return st


def _vrescale(st, kT, tau, dt, r1, gamma_sample, system_idx):
    n_sys = int(system_idx.max()) + 1
    dof = 3 * np.bincount(system_idx, minlength=n_sys) - 3
    kt_now = omd.calc_kT(st["masses"], st["momenta"], system_idx, dof)
    lam = oth.vrescale_factor(dof * kt_now / 2.0, dof, kT, tau, dt, r1, gamma_sample)
    return st["momenta"] * lam[system_idx][:, None]


def npt_crescale_isotropic_step(st, force_fn, dt, kT, p_ext, tau, noise, system_idx):
    """st: dict positions, momenta, masses, forces, stress, cell [S,3,3] (either
    convention), isothermal_compressibility [S], tau_p [S].  noise = (r1_a [S],
    gamma_a [S], cell [S], r1_b [S], gamma_b [S]) in the order the reference draws
    them.  force_fn(q, cell) -> (energy, forces, stress)."""
    st = dict(st)
    r1a, ga, zc, r1b, gb = noise
    m = st["masses"]
    st["momenta"] = _vrescale(st, kT, tau, dt / 2, r1a, ga, system_idx)
    st["momenta"] = st["momenta"] + st["forces"] * (dt / 2)
    vol = np.linalg.det(st["cell"])
    p = st["momenta"]
    n_sys = len(vol)
    two_k = np.zeros(n_sys)
    np.add.at(two_k, system_idx, (p * p / m[:, None]).sum(1))
    tr_p = two_k / vol - np.einsum("sii->s", st["stress"])
    bt, tp = st["isothermal_compressibility"], st["tau_p"]
    sqrt_vol = np.sqrt(vol)
    pre_random = np.sqrt(kT * bt * dt / (4 * tp))
    pre = bt * sqrt_vol / (2 * tp)
    change = -pre * (p_ext - tr_p / 3 - kT / (2 * vol)) * dt + np.sqrt(2.0) * pre_random * zc
    mu = ((sqrt_vol + change) / sqrt_vol) ** (2.0 / 3.0)
    mu_a = mu[system_idx][:, None]
    q = mu_a * st["positions"] + (mu_a + 1 / mu_a) * p * (0.5 * dt) / m[:, None]
    p = p / mu_a
    cell = mu[:, None, None] * st["cell"]
    e, f, s = force_fn(q, cell)
    st.update(positions=q, momenta=p, cell=cell, forces=f, energy=e, stress=s)
    st["momenta"] = st["momenta"] + st["forces"] * (dt / 2)
    st["momenta"] = _vrescale(st, kT, tau, dt / 2, r1b, gb, system_idx)
    return st


def npt_crescale_anisotropic_step(st, force_fn, dt, kT, p_ext, tau, noise, system_idx):
    """As npt_crescale_isotropic_step with per-axis factors; noise = (r1_a, gamma_a,
    baro [S, 5] = (volume normal, z_x, z_y, z_z, volume normal), r1_b, gamma_b)."""
    st = dict(st)
    r1a, ga, zb, r1b, gb = noise
    m = st["masses"]
    st["momenta"] = _vrescale(st, kT, tau, dt / 2, r1a, ga, system_idx)
    st["momenta"] = st["momenta"] + st["forces"] * (dt / 2)
    vol = np.linalg.det(st["cell"])
    p = st["momenta"]
    n_sys = len(vol)
    two_k = np.zeros((n_sys, 3))
    np.add.at(two_k, system_idx, p * p / m[:, None])
    p_diag = two_k / vol[:, None] - np.einsum("sii->si", st["stress"])
    tr_p = p_diag.sum(1)
    bt, tp = st["isothermal_compressibility"], st["tau_p"]
    sqrt_vol = np.sqrt(vol)
    pre_random = np.sqrt(kT * bt * dt / (4 * tp))
    pre = bt * sqrt_vol / (2 * tp)
    lam = sqrt_vol + (-pre * (p_ext - tr_p / 3 - kT / (2 * vol)) * dt / 2 + pre_random * zb[:, 0])
    c_rand = np.sqrt(2 * bt * kT * dt / (3 * tp)) / lam
    a_t = (bt / (3 * tp))[:, None] * (p_diag - tr_p[:, None] / 3)
    z = zb[:, 1:4]
    z = z - z.mean(1, keepdims=True)
    d = np.exp(a_t * dt + c_rand[:, None] * z)
    lam = lam + (-pre * (p_ext - tr_p / 3 - kT / (2 * vol)) * dt / 2 + pre_random * zb[:, 4])
    mu = d * ((lam / sqrt_vol) ** (2.0 / 3.0))[:, None]
    mu_a = mu[system_idx]
    q = mu_a * st["positions"] + (mu_a + 1 / mu_a) * p * dt / (2 * m[:, None])
    p = p / mu_a
    cell = mu[:, :, None] * st["cell"]
    e, f, s = force_fn(q, cell)
    st.update(positions=q, momenta=p, cell=cell, forces=f, energy=e, stress=s)
    st["momenta"] = st["momenta"] + st["forces"] * (dt / 2)
    st["momenta"] = _vrescale(st, kT, tau, dt / 2, r1b, gb, system_idx)
    return st


def _gram_schmidt_lower(box):
    out = np.zeros_like(box)
    a, b, c = box[:, :, 0], box[:, :, 1], box[:, :, 2]
    out[:, 0, 0] = np.linalg.norm(a, axis=1)
    out[:, 1, 0] = (a * b).sum(1) / out[:, 0, 0]
    out[:, 1, 1] = np.sqrt((b * b).sum(1) - out[:, 1, 0] ** 2)
    out[:, 2, 0] = (a * c).sum(1) / out[:, 0, 0]
    out[:, 2, 1] = ((b * c).sum(1) - out[:, 2, 0] * out[:, 1, 0]) / out[:, 1, 1]
    out[:, 2, 2] = np.sqrt((c * c).sum(1) - out[:, 2, 0] ** 2 - out[:, 2, 1] ** 2)
    return out


def npt_crescale_triclinic_step(st, force_fn, dt, kT, p_ext, tau, noise, system_idx,
                                average=False):
    """noise = (r1_a, gamma_a, baro [S, 11] = (volume normal, 3x3 normals row-major,
    volume normal), r1_b, gamma_b).  p_ext: scalar, or [3, 3] for the deviatoric
    correction (st then holds initial_cell_inv [S,3,3] and initial_volume [S])."""
    from scipy.linalg import expm

    st = dict(st)
    r1a, ga, zb, r1b, gb = noise
    m = st["masses"]
    st["momenta"] = _vrescale(st, kT, tau, dt / 2, r1a, ga, system_idx)
    st["momenta"] = st["momenta"] + st["forces"] * (dt / 2)
    cell = st["cell"]
    vol = np.linalg.det(cell)
    p = st["momenta"]
    n_sys = len(vol)
    eye = np.eye(3)
    if average:
        nat = np.bincount(system_idx, minlength=n_sys)
        pint = ((3 * nat - 3) / 3 * kT / vol)[:, None, None] * eye - st["stress"]
    else:
        kin = np.zeros((n_sys, 3, 3))
        np.add.at(kin, system_idx, np.einsum("ni,nj->nij", p, p) / m[:, None, None])
        pint = kin / vol[:, None, None] - st["stress"]
    tr_p = np.einsum("sii->s", pint)
    bt, tp = st["isothermal_compressibility"], st["tau_p"]
    sqrt_vol = np.sqrt(vol)
    pre_random = np.sqrt(kT * bt * dt / (4 * tp))
    pre = bt * sqrt_vol / (2 * tp)
    p_ext = np.asarray(p_ext, dtype=np.float64)
    pdrive = pint
    if p_ext.ndim >= 2:
        T = np.broadcast_to(p_ext, (n_sys, 3, 3))
        hydro = np.einsum("sii->s", T) / 3
        sdev = T - hydro[:, None, None] * eye
        ci = st["initial_cell_inv"]
        sig = st["initial_volume"][:, None, None] * (np.transpose(ci, (0, 2, 1)) @ sdev @ ci)
        sym = 0.5 * (sig + np.transpose(sig, (0, 2, 1)))
        pdev = np.transpose(cell, (0, 2, 1)) @ sym @ cell / vol[:, None, None]
        eff = hydro + np.einsum("sii->s", pdev) / 3
        pdrive = pint - pdev
    else:
        eff = p_ext
    drift = -pre * (eff - tr_p / 3 - kT / (2 * vol)) * dt / 2
    lam = sqrt_vol + (drift + pre_random * zb[:, 0])
    prm = np.sqrt(2 * bt * kT * dt / (3 * tp)) / lam
    tr_d = np.einsum("sii->s", pdrive)
    a_t = (bt / (3 * tp))[:, None, None] * (pdrive - (tr_d / 3)[:, None, None] * eye)
    Z = zb[:, 1:10].reshape(n_sys, 3, 3)
    Zt = Z - (np.einsum("sii->s", Z) / 3)[:, None, None] * eye
    D = np.stack([expm(x) for x in a_t * dt + prm[:, None, None] * Zt])
    D = _gram_schmidt_lower(D)
    lam = lam + (drift + pre_random * zb[:, 10])
    R = D * ((lam / sqrt_vol) ** (2.0 / 3.0))[:, None, None]
    M = np.broadcast_to(eye, R.shape) if average else np.transpose(np.linalg.inv(R), (0, 2, 1))
    Ra, Ma = R[system_idx], M[system_idx]
    q = np.einsum("nij,nj->ni", Ra, st["positions"]) + \
        np.einsum("nij,nj->ni", Ma + Ra, p) * dt / (2 * m[:, None])
    p = np.einsum("nij,nj->ni", Ma, p)
    cell = cell @ np.transpose(R, (0, 2, 1))
    e, f, s = force_fn(q, cell)
    st.update(positions=q, momenta=p, cell=cell, forces=f, energy=e, stress=s)
    st["momenta"] = st["momenta"] + st["forces"] * (dt / 2)
    st["momenta"] = _vrescale(st, kT, tau, dt / 2, r1b, gb, system_idx)
    return st


def npt_langevin_anisotropic_step(st, force_fn, dt, kT, p_ext, cell_noise, particle_noise,
                                  system_idx):
    """st: dict positions, momenta, masses, forces, stress, cell, cell_positions
    [S,3], cell_velocities [S,3], alpha, cell_alpha, b_tau, reference_cell; p_ext
    [3] or [S, 3]; cell_noise [S, 3]."""
    st = dict(st)
    n_sys = len(st["cell_positions"])
    n_at = np.bincount(system_idx, minlength=n_sys).astype(np.float64)
    q_mass = (n_at + 1) * kT * st["b_tau"] ** 2
    p3 = np.broadcast_to(np.asarray(p_ext, dtype=np.float64), (n_sys, 3))

    def force(stress, cell):
        vol = np.linalg.det(cell)
        p_diag = -np.einsum("sii->si", stress) + (n_at * kT / vol)[:, None]
        return vol[:, None] * (p_diag - p3)

    eps_old = st["cell_positions"].copy()
    f_n = force(st["stress"], st["cell"])
    beta_c = np.sqrt(2.0 * st["cell_alpha"] * kT * dt)[:, None] * cell_noise
    a_at = st["alpha"][system_idx]
    beta_p = np.sqrt(2 * a_at * kT * dt)[:, None] * particle_noise
    q2 = (2 * q_mass)[:, None]
    cb = 1 / (1 + st["cell_alpha"][:, None] * dt / q2)
    eps = eps_old + cb * dt * st["cell_velocities"] + cb * dt * dt * f_n / q2 + cb * dt * beta_c / q2
    cell = np.exp(eps)[:, :, None] * st["reference_cell"]
    m = st["masses"]
    scale = np.exp(eps - eps_old)[system_idx]
    b = 1 / (1 + a_at * dt / (2 * m))
    vel = st["momenta"] / m[:, None]
    c3 = vel + dt * st["forces"] / (2 * m[:, None]) + beta_p / (2 * m[:, None])
    q = scale * st["positions"] + (2 * scale / (scale + 1)) * (b * dt)[:, None] * c3
    forces_old = st["forces"]
    e, f, s = force_fn(q, cell)
    f_new = force(s, cell)
    qm = q_mass[:, None]
    ca = st["cell_alpha"][:, None]
    ac = (1 - ca * dt / (2 * qm)) / (1 + ca * dt / (2 * qm))
    bc = 1 / (1 + ca * dt / (2 * qm))
    eps_dot = ac * st["cell_velocities"] + dt * (ac * f_n + f_new) / (2 * qm) + bc * beta_c / qm
    m2 = 2 * m
    ap = ((1 - a_at * dt / m2) / (1 + a_at * dt / m2))[:, None]
    bp = (1 / (1 + a_at * dt / m2))[:, None]
    v_new = ap * vel + dt * (ap * forces_old + f) / m2[:, None] + bp * beta_p / m[:, None]
    st.update(positions=q, momenta=v_new * m[:, None], forces=f, energy=e, stress=s, cell=cell,
              cell_positions=eps, cell_velocities=eps_dot, cell_masses=q_mass)
    return st


def _sinhx_x(x):
    return 1 + x ** 2 / 6 + x ** 4 / 120 + x ** 6 / 5040 + x ** 8 / 362_880 + x ** 10 / 39_916_800


def npt_nose_hoover_isotropic_step(st, force_fn, dt, kT, p_ext, system_idx):
    """st: dict positions, momenta, masses, forces, stress, reference_cell,
    cell_position [S], cell_momentum [S], and per chain ("t" particles, "b" cell)
    xi / p_xi [S, M], ke [S], tau [S], chain_steps, sy_steps.  Returns the updated
    dict (cell, cell_mass and the chains' masses included)."""
    st = dict(st)
    n_sys = len(st["cell_position"])
    nat = np.bincount(system_idx, minlength=n_sys).astype(np.float64)
    dof_t, dof_b = 3 * nat - 3, np.ones(n_sys)
    m = st["masses"]
    M = st["t_xi"].shape[1]
    qt = oth.chain_masses(dof_t, kT, st["t_tau"], M)
    qb = oth.chain_masses(dof_b, kT, st["b_tau"], M)
    w = 3 * (nat + 1) * kT * st["b_tau"] ** 2
    cs, ss = st["chain_steps"], st["sy_steps"]
    sidx = np.arange(n_sys)
    pc, b_xi, b_pxi, b_ke = oth.nhc_half_step(st["cell_momentum"][:, None], st["b_xi"],
                                              st["b_pxi"], qb, st["b_ke"], dof_b, kT, dt, cs,
                                              ss, sidx)
    p, t_xi, t_pxi, t_ke = oth.nhc_half_step(st["momenta"], st["t_xi"], st["t_pxi"], qt,
                                             st["t_ke"], dof_t, kT, dt, cs, ss, system_idx)
    pc = pc[:, 0]
    alpha = 1 + 3 / dof_t
    v0 = np.linalg.det(st["reference_cell"])

    def cell_force(p, stress, vol):
        ke = omd.kinetic_energy(m, p, system_idx)
        return alpha * 2 * ke - np.einsum("sii->s", stress) * vol - p_ext * vol * 3

    vol = v0 * np.exp(3 * st["cell_position"])
    pc = pc + dt / 2 * cell_force(p, st["stress"], vol)
    v = pc / w
    dt2 = dt / 2

    def il2(p, f):
        x = (alpha * v)[system_idx] * dt2
        return p * np.exp(-x)[:, None] + dt2 * f * _sinhx_x(x / 2)[:, None] * np.exp(-x / 2)[:, None]

    p = il2(p, st["forces"])
    eps = st["cell_position"] + v * dt
    vol = v0 * np.exp(3 * eps)
    cell = ((vol / v0) ** (1.0 / 3.0))[:, None, None] * st["reference_cell"]
    x = (v * dt)[system_idx]
    q = st["positions"]
    q = q + (q * (np.exp(x) - 1)[:, None] + dt * (p / m[:, None]) * np.exp(x / 2)[:, None] *
             _sinhx_x(x / 2)[:, None])
    e, f, s = force_fn(q, cell)
    p = il2(p, f)
    pc = pc + dt / 2 * cell_force(p, s, vol)
    t_ke = omd.kinetic_energy(m, p, system_idx)
    p, t_xi, t_pxi, t_ke = oth.nhc_half_step(p, t_xi, t_pxi, qt, t_ke, dof_t, kT, dt, cs, ss,
                                             system_idx)
    b_ke = pc ** 2 / (2 * w)
    pc, b_xi, b_pxi, b_ke = oth.nhc_half_step(pc[:, None], b_xi, b_pxi, qb, b_ke, dof_b, kT,
                                              dt, cs, ss, sidx)
    st.update(positions=q, momenta=p, forces=f, energy=e, stress=s, cell=cell,
              cell_position=eps, cell_momentum=pc[:, 0], cell_mass=w, t_xi=t_xi, t_pxi=t_pxi,
              t_ke=t_ke, t_q=qt, b_xi=b_xi, b_pxi=b_pxi, b_ke=b_ke, b_q=qb)
    return st
