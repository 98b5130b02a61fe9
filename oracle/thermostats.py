"""Deterministic-thermostat oracle (TEST INFRASTRUCTURE ONLY; never the product path).

FP64 numpy restatement of the reference's NVT Nose-Hoover-chain and V-rescale
(CSVR) steps, per system, with the random numbers of CSVR passed in.

* ``chain_masses``    <- torch_sim/integrators/md.py:379-386, 534-559
                         Q_j = kT tau^2, Q_1 = N_f kT tau^2
* ``nhc_half_step``   <- md.py:388-514  (Martyna-Tuckerman-Tobias-Klein 1996:
                         chain_steps x sy_steps Suzuki-Yoshida sub-steps; each
                         sub-step updates the chain momenta backwards, rescales
                         the particle momenta, moves the chain positions and
                         updates the chain momenta forwards)
* ``nvt_nose_hoover_step``  <- torch_sim/integrators/nvt.py:381-488
                         (NHC(dt/2) . velocity Verlet . NHC(dt/2))
* ``nose_hoover_invariant`` <- nvt.py:491-562
* ``vrescale_factor``  <- nvt.py:594-654 (Bussi-Donadio-Parrinello 2007, Eq. A7)
* ``nvt_vrescale_step``<- nvt.py:715-741 (rescale, then velocity Verlet)

Degrees of freedom are 3N - 3 per system (nvt.py:287-290, 355-357).
"""

from __future__ import annotations

import numpy as np

from . import md as omd

# Suzuki-Yoshida composition weights (Yoshida 1990; Suzuki 1993), as tabulated in
# the reference (md.py:308-335)
SY_WEIGHTS = {
    1: (1.0,),
    3: (0.828981543588751, -0.657963087177502, 0.828981543588751),
    5: (0.2967324292201065, 0.2967324292201065, -0.186929716880426, 0.2967324292201065,
        0.2967324292201065),
    7: (0.784513610477560, 0.235573213359357, -1.17767998417887, 1.31518632068391,
        -1.17767998417887, 0.235573213359357, 0.784513610477560),
}


def chain_masses(dof, kT, tau, chain_length):
    dof = np.asarray(dof, dtype=np.float64)
    q = np.ones((len(dof), chain_length)) * (np.asarray(kT) * np.asarray(tau) ** 2)[..., None]
    q[:, 0] *= dof
    return q


def _substep(delta, p, xi, p_xi, q, ke, dof, kT, system_idx):
    """One chain sub-step of length delta; returns (p, xi, p_xi, ke)."""
    xi, p_xi, ke = xi.copy(), p_xi.copy(), ke.copy()
    m = p_xi.shape[1] - 1
    d2, d4, d8 = delta / 2.0, delta / 4.0, delta / 8.0
    if m > 0:
        p_xi[:, m] += d4 * (p_xi[:, m - 1] ** 2 / q[:, m - 1] - kT)
    for j in range(m - 1, 0, -1):
        g = p_xi[:, j - 1] ** 2 / q[:, j - 1] - kT
        s = np.exp(-d8 * p_xi[:, j + 1] / q[:, j + 1])
        p_xi[:, j] = s * (s * p_xi[:, j] + d4 * g)
    g = 2.0 * ke - dof * kT
    s = np.exp(-d8 * p_xi[:, 1] / q[:, 1]) if m > 0 else 1.0
    p_xi[:, 0] = s * (s * p_xi[:, 0] + d4 * g)
    scale = np.exp(-d2 * p_xi[:, 0] / q[:, 0])
    ke = ke * scale ** 2
    p = p * scale[system_idx][:, None]
    xi = xi + d2 * p_xi / q
    g = 2.0 * ke - dof * kT
    for j in range(m):
        s = np.exp(-d8 * p_xi[:, j + 1] / q[:, j + 1])
        p_xi[:, j] = s * (s * p_xi[:, j] + d4 * g)
        g = p_xi[:, j] ** 2 / q[:, j] - kT
    p_xi[:, m] += d4 * g
    return p, xi, p_xi, ke


def nhc_half_step(p, xi, p_xi, q, ke, dof, kT, dt, chain_steps, sy_steps, system_idx):
    dof = np.asarray(dof, dtype=np.float64)
    if chain_steps == 1 and sy_steps == 1:
        return _substep(dt, p, xi, p_xi, q, ke, dof, kT, system_idx)
    w = SY_WEIGHTS[sy_steps]
    for k in range(chain_steps * sy_steps):
        p, xi, p_xi, ke = _substep(dt / chain_steps * w[k % sy_steps], p, xi, p_xi, q, ke,
                                   dof, kT, system_idx)
    return p, xi, p_xi, ke


def nvt_nose_hoover_step(st, chain, force_fn, dt, kT, chain_steps, sy_steps, system_idx):
    """st: dict positions/momenta/masses/forces/energy; chain: dict xi/p_xi/ke/dof/tau."""
    q = chain_masses(chain["dof"], kT, chain["tau"], chain["xi"].shape[1])
    p, xi, p_xi, ke = nhc_half_step(st["momenta"], chain["xi"], chain["p_xi"], q,
                                    chain["ke"], chain["dof"], kT, dt, chain_steps, sy_steps,
                                    system_idx)
    st = omd.nve_step(dict(st, momenta=p), force_fn, dt)
    ke = omd.kinetic_energy(st["masses"], st["momenta"], system_idx)
    p, xi, p_xi, ke = nhc_half_step(st["momenta"], xi, p_xi, q, ke, chain["dof"], kT, dt,
                                    chain_steps, sy_steps, system_idx)
    return dict(st, momenta=p), dict(chain, xi=xi, p_xi=p_xi, q=q, ke=ke)


def nose_hoover_invariant(energy, masses, momenta, system_idx, xi, p_xi, q, dof, kT):
    e = energy + omd.kinetic_energy(masses, momenta, system_idx)
    e = e + p_xi[:, 0] ** 2 / (2 * q[:, 0]) + dof * kT * xi[:, 0]
    for j in range(1, xi.shape[1]):
        e = e + p_xi[:, j] ** 2 / (2 * q[:, j]) + kT * xi[:, j]
    return e


def vrescale_factor(ke, dof, kT, tau, dt, r1, gamma_sample):
    """lambda = sqrt(c1 + c2 (r1^2 + 2 g) + 2 r1 sqrt(c1 c2)),
    c1 = exp(-dt/tau), c2 = (1 - c1) (dof kT / 2) / (ke) / dof, g ~ Gamma((dof-1)/2)."""
    dof = np.asarray(dof, dtype=np.float64)
    c1 = np.exp(-dt / tau)
    c2 = (1.0 - c1) * (dof * kT / 2.0) / ke / dof
    r2 = 2.0 * gamma_sample
    return np.sqrt(c1 + c2 * (r1 ** 2 + r2) + 2.0 * r1 * np.sqrt(c1 * c2))


def nvt_vrescale_step(st, force_fn, dt, kT, tau, r1, gamma_sample, system_idx):
    n_sys = int(system_idx.max()) + 1
    dof = 3 * np.bincount(system_idx, minlength=n_sys) - 3
    kt_now = omd.calc_kT(st["masses"], st["momenta"], system_idx, dof)
    lam = vrescale_factor(dof * kt_now / 2.0, dof, kT, tau, dt, r1, gamma_sample)
    p = st["momenta"] * lam[system_idx][:, None]
    return omd.nve_step(dict(st, momenta=p), force_fn, dt)
