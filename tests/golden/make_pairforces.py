"""Golden fixtures for force-defined pair models (PairForcesModel, particle life),
generated by running the reference TorchSim itself.

Run in a container where the reference source tree is present::

    python tests/golden/make_pairforces.py /path/to/torch-sim

Writes ``pairforces.npz`` beside this script:

* ``sys/*``    two periodic systems of seeded random points (species 1/2)
* ``plife/*``  ParticleLifeModel(sigma=1, epsilon=1, beta=0.3, cutoff=1.2):
               energy, forces, stress, per-atom stresses
* ``asym/*``   PairForcesModel with an asymmetric species-dependent force
               f(r, zi, zj) = (1 + zi - 0.5 zj) (1.1 - r) on a full list, cutoff 1.1
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)

from make_golden import _install_shims  # noqa: E402


def asym_force(dr, zi, zj):
    return (1.0 + zi.to(dr.dtype) - 0.5 * zj.to(dr.dtype)) * (1.1 - dr)


def main(ref_root):
    _install_shims(ref_root)
    import torch

    torch.set_default_dtype(torch.float64)
    import torch_sim as ts
    from torch_sim.models.pair_potential import PairForcesModel
    from torch_sim.models.particle_life import ParticleLifeModel

    rng = np.random.default_rng(5)
    pos, sysi, z, cells = [], [], [], []
    for s, (n, L) in enumerate(((48, 3.6), (30, 3.1))):
        cell = np.diag([L, L * 1.1, L * 0.95])
        cell[1, 0] = 0.2  # triclinic (row-vector cell, lower triangle)
        pos.append(rng.uniform(0, 1, (n, 3)) @ cell)
        sysi.append(np.full(n, s))
        z.append(rng.integers(1, 3, n))
        cells.append(cell.T)  # column-vector convention of SimState
    d = {"positions": np.concatenate(pos), "system_idx": np.concatenate(sysi),
         "atomic_numbers": np.concatenate(z), "cell": np.stack(cells),
         "masses": np.ones(sum(len(p) for p in pos))}
    T = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt)  # noqa: E731
    st = ts.SimState(positions=T(d["positions"]), masses=T(d["masses"]), cell=T(d["cell"]),
                     pbc=True, atomic_numbers=T(d["atomic_numbers"], torch.int64),
                     system_idx=T(d["system_idx"], torch.int64))
    out = {f"sys/{k}": v for k, v in d.items()}

    m = ParticleLifeModel(sigma=1.0, epsilon=1.0, beta=0.3, cutoff=1.2, compute_stress=True,
                          per_atom_stresses=True)
    o = m(st)
    for k in ("energy", "forces", "stress", "stresses"):
        out[f"plife/{k}"] = o[k].detach().numpy()

    m2 = PairForcesModel(force_fn=asym_force, cutoff=1.1, compute_stress=True,
                         per_atom_stresses=True)
    o = m2(st)
    for k in ("energy", "forces", "stress", "stresses"):
        out[f"asym/{k}"] = o[k].detach().numpy()
    np.savez_compressed(os.path.join(HERE, "pairforces.npz"), **out)
    print("pair-force fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TORCH_SIM_REF", ""))
