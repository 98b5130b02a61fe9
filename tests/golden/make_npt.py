"""Golden fixtures for the isotropic NPT Langevin step, generated by running the
reference TorchSim itself.

Run in a container where the reference source tree is present::

    python tests/golden/make_npt.py /path/to/torch-sim

Writes ``npt.npz`` beside this script: 8 steps of ``npt_langevin_isotropic_step``
(group ``npt``) on three Morse Cu systems (compute_stress=True) at 1000 K and
1 GPa (internal units), and 8 steps of ``npt_langevin_anisotropic_step`` (group
``npt_aniso``) at (1.0, 1.3, 0.7) GPa per axis, with the reference's random
numbers recorded (per step: the cell noise [S] or [S, 3], then the particle
noise [N, 3]); and 8 deterministic steps of ``npt_nose_hoover_isotropic_step``
(group ``npt_nh``, MTK barostat with Nose-Hoover chains) with both chains and the
conserved quantity recorded.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)

from make_golden import _install_shims  # noqa: E402


def main(ref_root):
    _install_shims(ref_root)
    sys.path.insert(0, os.path.join(REPO, "torch-sim_b200"))
    import torch

    torch.set_default_dtype(torch.float64)
    import torch_sim as ts
    from torch_sim.integrators import npt as ref_npt
    from torch_sim.models.morse import MorseModel

    from tsb import workloads as W

    cu3 = W.copper_batch(3, 8, 40, seed=23, jitter=0.03)
    T = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt)  # noqa: E731
    st = ts.SimState(positions=T(cu3["positions"]), masses=T(cu3["masses"]),
                     cell=T(cu3["cell"]), pbc=True,
                     atomic_numbers=T(cu3["atomic_numbers"], torch.int64),
                     system_idx=T(cu3["system_idx"], torch.int64))
    st.rng = 31
    morse = MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                       compute_stress=True)
    kT = 1000.0 * W.KB_EV
    dt = 0.002 * W.METAL_TIME
    p_ext = 1.0 * 0.006241509074460764  # 1 GPa in eV/A^3
    md = ref_npt.npt_langevin_isotropic_init(st, morse, kT=torch.tensor(kT),
                                             dt=torch.tensor(dt))
    noises = []
    real_randn = torch.randn

    def rec(*a, **k):
        x = real_randn(*a, **k)
        noises.append(x.clone())
        return x

    keys = ("positions", "momenta", "energy", "forces", "stress", "cell", "cell_positions",
            "cell_velocities", "cell_masses")
    traj = [[getattr(md, k).clone().numpy() for k in keys]]
    torch.randn = rec
    try:
        for _ in range(8):
            md = ref_npt.npt_langevin_isotropic_step(md, morse, dt=torch.tensor(dt),
                                                     kT=torch.tensor(kT),
                                                     external_pressure=torch.tensor(p_ext))
            traj.append([getattr(md, k).clone().numpy() for k in keys])
    finally:
        torch.randn = real_randn
    out = {f"sys/{k}": cu3[k] for k in ("masses", "cell", "system_idx", "atomic_numbers")}
    for i, k in enumerate(keys):
        out[f"npt/{k}"] = np.stack([t[i] for t in traj])
    out["npt/cell_noise"] = np.stack([n.numpy() for n in noises[0::2]])
    out["npt/particle_noise"] = np.stack([n.numpy() for n in noises[1::2]])
    for k in ("alpha", "cell_alpha", "b_tau", "reference_cell"):
        out[f"npt/{k}"] = getattr(md, k).clone().numpy()
    out["npt/dt"], out["npt/kT"], out["npt/p_ext"] = np.array(dt), np.array(kT), np.array(p_ext)

    # per-axis strains with a different target pressure on each axis
    p3 = torch.tensor([1.0, 1.3, 0.7]) * p_ext
    st.rng = 31
    md = ref_npt.npt_langevin_anisotropic_init(st, morse, kT=torch.tensor(kT),
                                               dt=torch.tensor(dt))
    noises = []
    traj = [[getattr(md, k).clone().numpy() for k in keys]]
    torch.randn = rec
    try:
        for _ in range(8):
            md = ref_npt.npt_langevin_anisotropic_step(md, morse, dt=torch.tensor(dt),
                                                       kT=torch.tensor(kT), external_pressure=p3)
            traj.append([getattr(md, k).clone().numpy() for k in keys])
    finally:
        torch.randn = real_randn
    for i, k in enumerate(keys):
        out[f"npt_aniso/{k}"] = np.stack([t[i] for t in traj])
    out["npt_aniso/cell_noise"] = np.stack([n.numpy() for n in noises[0::2]])
    out["npt_aniso/particle_noise"] = np.stack([n.numpy() for n in noises[1::2]])
    for k in ("alpha", "cell_alpha", "b_tau", "reference_cell"):
        out[f"npt_aniso/{k}"] = getattr(md, k).clone().numpy()
    out["npt_aniso/dt"], out["npt_aniso/kT"] = np.array(dt), np.array(kT)
    out["npt_aniso/p_ext"] = p3.numpy()

    # MTK isotropic NPT with Nose-Hoover chains (deterministic)
    st.rng = 31
    md = ref_npt.npt_nose_hoover_isotropic_init(st, morse, kT=torch.tensor(kT),
                                                dt=torch.tensor(dt))
    nh_keys = ("positions", "momenta", "energy", "forces", "stress", "cell", "cell_position",
               "cell_momentum", "cell_mass")

    def snap(md):
        row = [getattr(md, k).clone().numpy() for k in nh_keys]
        for ch in (md.thermostat, md.barostat):
            row += [ch.positions.clone().numpy(), ch.momenta.clone().numpy(),
                    ch.masses.clone().numpy(), ch.kinetic_energy.clone().numpy()]
        row.append(ref_npt.npt_nose_hoover_isotropic_invariant(
            md, torch.tensor(kT), torch.tensor(p_ext)).clone().numpy())
        return row

    traj = [snap(md)]
    for _ in range(8):
        md = ref_npt.npt_nose_hoover_isotropic_step(md, morse, dt=torch.tensor(dt),
                                                    kT=torch.tensor(kT),
                                                    external_pressure=torch.tensor(p_ext))
        traj.append(snap(md))
    names = list(nh_keys) + [f"{c}_{v}" for c in ("thermostat", "barostat")
                             for v in ("positions", "momenta", "masses", "kinetic_energy")]
    names.append("invariant")
    for i, k in enumerate(names):
        out[f"npt_nh/{k}"] = np.stack([t[i] for t in traj])
    out["npt_nh/dt"], out["npt_nh/kT"], out["npt_nh/p_ext"] = (np.array(dt), np.array(kT),
                                                               np.array(p_ext))
    np.savez_compressed(os.path.join(HERE, "npt.npz"), **out)
    print("NPT fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TORCH_SIM_REF", ""))
