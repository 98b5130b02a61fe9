"""Generate ``config1.npz`` by running the reference TorchSim itself on the
256-atom Lennard-Jones argon NVE case.

Run in a container where the reference source tree is present::

    python tests/golden/make_config1.py /path/to/torch-sim

The case: argon fcc 4x4x4 conventional cells (256 atoms, a = 5.26 A, cubic
periodic cell), positions jittered by N(0, 0.05 A) from a seeded generator,
LJ sigma = 3.405 A, epsilon = 0.0104 eV, cutoff 2.5 sigma; Maxwell-Boltzmann
momenta at 50 K from the reference's own ``initialize_momenta`` with
``state.rng = 2024`` (zero net momentum), float64; 100 NVE velocity-Verlet
steps of 2 fs.  Two potentials:

* ``lj``       the reference's ``LennardJonesModel`` (truncated, unshifted);
* ``lj_shift`` ``PairPotentialModel`` with the LJ pair function minus its
               value at the cutoff (energy continuous at rc).

Recorded (float64): positions and momenta every 10 steps, potential energy,
kinetic energy and stress at every step, forces at the start and the end, and
the initial full pair set (i, j as int32; shifts as int8).
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)

from make_golden import _install_shims  # noqa: E402

SIGMA, EPS, RC = 3.405, 0.0104, 2.5 * 3.405
N_STEPS, EVERY = 100, 10


def main(ref_root):
    _install_shims(ref_root)
    sys.path.insert(0, os.path.join(REPO, "torch-sim_b200"))
    import torch

    torch.set_default_dtype(torch.float64)
    import torch_sim as ts
    from torch_sim.models.lennard_jones import LennardJonesModel, lennard_jones_pair
    from torch_sim.models.pair_potential import PairPotentialModel
    from torch_sim.neighbors import torch_nl_linked_cell

    from tsb import workloads as W

    d = W.argon_fcc((4, 4, 4), jitter=0.05, seed=1)
    T = lambda x, dt=torch.float64: torch.as_tensor(np.asarray(x), dtype=dt)  # noqa: E731

    def state():
        st = ts.SimState(positions=T(d["positions"]), masses=T(d["masses"]),
                         cell=T(d["cell"]), pbc=T(d["pbc"], torch.bool),
                         atomic_numbers=T(d["atomic_numbers"], torch.long),
                         system_idx=T(d["system_idx"], torch.long))
        st.rng = 2024
        return st

    shift = float(lennard_jones_pair(torch.tensor([RC]), 18, 18, SIGMA, EPS)[0])

    def shifted_pair(r, zi, zj):
        return lennard_jones_pair(r, zi, zj, SIGMA, EPS) - shift

    models = {
        "lj": LennardJonesModel(sigma=SIGMA, epsilon=EPS, cutoff=RC, compute_stress=True),
        "lj_shift": PairPotentialModel(pair_fn=shifted_pair, cutoff=RC, compute_stress=True),
    }
    out = {k: d[k] for k in ("positions", "masses", "cell", "pbc", "atomic_numbers",
                             "system_idx")}
    out = {f"init/{k}": v for k, v in out.items()}
    kT = 50.0 * W.KB_EV
    dt = 0.002 * W.METAL_TIME
    for name, model in models.items():
        md = ts.nve_init(state(), model, kT=torch.tensor(kT))
        frames_x, frames_p, epot, ekin, stress = [], [], [], [], []
        f0 = md.forces.clone()
        for step in range(N_STEPS + 1):
            if step:
                md = ts.nve_step(md, model, dt=torch.tensor(dt))
            if step % EVERY == 0:
                frames_x.append(md.positions.clone())
                frames_p.append(md.momenta.clone())
            epot.append(float(md.energy[0]))
            ekin.append(float(ts.calc_kinetic_energy(masses=md.masses, momenta=md.momenta,
                                                     system_idx=md.system_idx)[0]))
            stress.append(model(md)["stress"][0].clone())
        out[f"{name}/positions"] = torch.stack(frames_x).numpy()
        out[f"{name}/momenta"] = torch.stack(frames_p).numpy()
        out[f"{name}/epot"] = np.array(epot)
        out[f"{name}/ekin"] = np.array(ekin)
        out[f"{name}/stress"] = torch.stack(stress).numpy()
        out[f"{name}/forces0"] = f0.numpy()
        out[f"{name}/forces_end"] = md.forces.numpy()
    out["dt"] = np.array(dt)
    out["kT"] = np.array(kT)
    out["every"] = np.array(EVERY)
    out["shift"] = np.array(shift)
    st = state()
    mapping, sysm, shifts = torch_nl_linked_cell(st.positions, st.row_vector_cell, st.pbc,
                                                 torch.tensor(RC), st.system_idx)
    out["pairs/ij"] = mapping.numpy().astype(np.int32)
    out["pairs/shifts"] = np.rint(shifts.numpy()).astype(np.int8)
    np.savez_compressed(os.path.join(HERE, "config1.npz"), **out)
    print("pairs:", mapping.shape[1], "E drift lj:", max(np.abs(
        np.array(out["lj/epot"]) + out["lj/ekin"] - out["lj/epot"][0] - out["lj/ekin"][0])))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
