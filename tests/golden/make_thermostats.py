"""Golden fixtures for the NVT Nose-Hoover-chain and V-rescale (CSVR) steps,
generated by running the reference TorchSim itself.

Run in a container where the reference source tree is present::

    python tests/golden/make_thermostats.py /path/to/torch-sim

Writes ``thermostats.npz`` beside this script:

* ``nhc/*``   10 steps of ``nvt_nose_hoover_step`` on three Morse Cu systems of
              different sizes (chain_length 3, chain_steps 3, sy_steps 3, tau =
              10 dt): positions, momenta, energy, chain positions / momenta /
              masses / kinetic energy per step, and ``nvt_nose_hoover_invariant``
* ``vr/*``    10 steps of ``nvt_vrescale_step`` on the same systems, with the
              reference's random numbers recorded (the standard normal r1 and
              the Gamma((dof-1)/2) sample, before the factor 2 of
              nvt.py:_vrescale_update)
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
    from torch_sim.integrators import nvt as ref_nvt
    from torch_sim.models.morse import MorseModel

    from tsb import workloads as W

    def to_state(d):
        T = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt)  # noqa: E731
        return ts.SimState(positions=T(d["positions"]), masses=T(d["masses"]),
                           cell=T(d["cell"]), pbc=True,
                           atomic_numbers=T(d["atomic_numbers"], torch.int64),
                           system_idx=T(d["system_idx"], torch.int64))

    out = {}
    cu3 = W.copper_batch(3, 8, 40, seed=21, jitter=0.03)
    morse = MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0)
    kT = 1000.0 * W.KB_EV
    dt = 0.002 * W.METAL_TIME
    for k in ("masses", "cell", "system_idx", "positions"):
        out[f"sys/{k}"] = cu3[k]
    out["sys/dt"] = np.array(dt)
    out["sys/kT"] = np.array(kT)

    # ------------------------------------------------------------ Nose-Hoover
    st = to_state(cu3)
    st.rng = 11
    md = ts.nvt_nose_hoover_init(st, morse, kT=torch.tensor(kT), dt=torch.tensor(dt),
                                 chain_length=3, chain_steps=3, sy_steps=3)
    rec = {k: [] for k in ("positions", "momenta", "energy", "xi", "p_xi", "Q", "KE",
                           "invariant")}

    def snap(m):
        rec["positions"].append(m.positions.clone().numpy())
        rec["momenta"].append(m.momenta.clone().numpy())
        rec["energy"].append(m.energy.clone().numpy())
        rec["xi"].append(m.chain.positions.clone().numpy())
        rec["p_xi"].append(m.chain.momenta.clone().numpy())
        rec["Q"].append(m.chain.masses.clone().numpy())
        rec["KE"].append(m.chain.kinetic_energy.clone().numpy())
        rec["invariant"].append(
            ref_nvt.nvt_nose_hoover_invariant(m, torch.tensor(kT)).clone().numpy())

    snap(md)
    out["nhc/dof"] = md.chain.degrees_of_freedom.clone().numpy()
    out["nhc/tau"] = md.chain.tau.clone().numpy()
    for _ in range(10):
        md = ts.nvt_nose_hoover_step(md, morse, dt=torch.tensor(dt), kT=torch.tensor(kT))
        snap(md)
    for k, v in rec.items():
        out[f"nhc/{k}"] = np.stack(v)

    # ------------------------------------------------------------- V-rescale
    st = to_state(cu3)
    st.rng = 12
    md = ts.nvt_vrescale_init(st, morse, kT=torch.tensor(kT))
    r1s, gs = [], []
    real_randn, real_gamma = torch.randn, torch._standard_gamma

    def rec_randn(*a, **k):
        x = real_randn(*a, **k)
        r1s.append(x.clone())
        return x

    def rec_gamma(*a, **k):
        x = real_gamma(*a, **k)
        gs.append(x.clone())
        return x

    traj = [(md.positions.clone(), md.momenta.clone(), md.energy.clone())]
    torch.randn, torch._standard_gamma = rec_randn, rec_gamma
    try:
        for _ in range(10):
            md = ts.nvt_vrescale_step(morse, md, dt=torch.tensor(dt), kT=torch.tensor(kT))
            traj.append((md.positions.clone(), md.momenta.clone(), md.energy.clone()))
    finally:
        torch.randn, torch._standard_gamma = real_randn, real_gamma
    for k, name in enumerate(("positions", "momenta", "energy")):
        out[f"vr/{name}"] = np.stack([t[k].numpy() for t in traj])
    out["vr/r1"] = np.stack([x.numpy() for x in r1s])
    out["vr/gamma"] = np.stack([x.numpy() for x in gs])
    out["vr/tau"] = np.array(10 * dt)
    np.savez_compressed(os.path.join(HERE, "thermostats.npz"), **out)
    print("thermostat fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TORCH_SIM_REF", ""))
