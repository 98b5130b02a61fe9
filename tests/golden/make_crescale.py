"""Golden fixtures for the isotropic C-rescale NPT step, generated by running the
reference TorchSim itself.

Run in a container where the reference source tree is present::

    python tests/golden/make_crescale.py /path/to/torch-sim

Writes ``crescale.npz`` beside this script: 8 steps each of
``npt_crescale_isotropic_step`` (group ``crescale``),
``npt_crescale_anisotropic_step`` (``crescale_aniso``),
``npt_crescale_triclinic_step`` with a scalar and with a non-hydrostatic tensor
pressure (``crescale_tri``, ``crescale_tri_dev``) and
``npt_crescale_triclinic_average_step`` (``crescale_tri_avg``) on three Morse Cu
systems (compute_stress=True) at 600 K and 1 GPa (internal units), tau = 5 dt,
tau_p = 50 dt, compressibility 1e-4 bar^-1, with the reference's random numbers
recorded per step in the order drawn: V-rescale (r1, Gamma deviate), the
barostat normals (isotropic: one [S]; anisotropic: [S], [S, 3], [S]; triclinic:
[S], [S, 3, 3], [S]), V-rescale (r1, Gamma deviate).
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
    from torch_sim.units import MetalUnits

    from tsb import workloads as W

    cu3 = W.copper_batch(3, 8, 40, seed=29, jitter=0.03)
    T = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt)  # noqa: E731
    st = ts.SimState(positions=T(cu3["positions"]), masses=T(cu3["masses"]),
                     cell=T(cu3["cell"]), pbc=True,
                     atomic_numbers=T(cu3["atomic_numbers"], torch.int64),
                     system_idx=T(cu3["system_idx"], torch.int64))
    st.rng = 37
    morse = MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                       compute_stress=True)
    kT = 600.0 * W.KB_EV
    dt = 0.002 * W.METAL_TIME
    p_ext = 1.0 * 0.006241509074460764  # 1 GPa in eV/A^3
    beta = 1e-4 / float(MetalUnits.pressure)
    out = {f"sys/{k}": cu3[k] for k in ("masses", "cell", "system_idx", "atomic_numbers")}
    real_randn, real_gamma = torch.randn, torch._standard_gamma
    keys = ("positions", "momenta", "energy", "forces", "stress", "cell")
    # a non-hydrostatic external pressure for the deviatoric correction
    p_tensor = torch.tensor([[1.2, 0.1, 0.0], [0.1, 0.9, -0.05], [0.0, -0.05, 1.0]]) * p_ext
    runs = (("crescale", ref_npt.npt_crescale_isotropic_step, 3, p_ext),
            ("crescale_aniso", ref_npt.npt_crescale_anisotropic_step, 5, p_ext),
            ("crescale_tri", ref_npt.npt_crescale_triclinic_step, 5, p_ext),
            ("crescale_tri_dev", ref_npt.npt_crescale_triclinic_step, 5, p_tensor),
            ("crescale_tri_avg", ref_npt.npt_crescale_triclinic_average_step, 5, p_ext))
    for grp, step_fn, n_normal, pe in runs:
        st.rng = 37
        md = ref_npt.npt_crescale_init(st, morse, kT=torch.tensor(kT), dt=torch.tensor(dt),
                                       tau_p=torch.tensor(50 * dt),
                                       isothermal_compressibility=torch.tensor(beta))
        normals, gammas = [], []

        def rec_randn(*a, **k):
            x = real_randn(*a, **k)
            normals.append(x.clone())
            return x

        def rec_gamma(*a, **k):
            x = real_gamma(*a, **k)
            gammas.append(x.clone())
            return x

        traj = [[getattr(md, k).clone().numpy() for k in keys]]
        torch.randn, torch._standard_gamma = rec_randn, rec_gamma
        try:
            for _ in range(8):
                md = step_fn(md, morse, dt=torch.tensor(dt), kT=torch.tensor(kT),
                             external_pressure=torch.as_tensor(pe), tau=torch.tensor(5 * dt))
                traj.append([getattr(md, k).clone().numpy() for k in keys])
        finally:
            torch.randn, torch._standard_gamma = real_randn, real_gamma
        assert len(normals) == 8 * n_normal and len(gammas) == 16, (len(normals), len(gammas))
        for i, k in enumerate(keys):
            out[f"{grp}/{k}"] = np.stack([t[i] for t in traj])
        per = [normals[j::n_normal] for j in range(n_normal)]
        out[f"{grp}/r1_a"] = np.stack([n.numpy() for n in per[0]])
        out[f"{grp}/r1_b"] = np.stack([n.numpy() for n in per[-1]])
        if n_normal == 3:
            out[f"{grp}/cell_noise"] = np.stack([n.numpy() for n in per[1]])
        else:  # (volume normal, z [S, 3] or Z [S, 3, 3], volume normal) -> [S, 5 | 11]
            out[f"{grp}/cell_noise"] = np.stack([
                np.concatenate([a.numpy()[:, None], b.numpy().reshape(len(a), -1),
                                c.numpy()[:, None]], axis=1)
                for a, b, c in zip(per[1], per[2], per[3])])
        out[f"{grp}/gamma_a"] = np.stack([g.numpy() for g in gammas[0::2]])
        out[f"{grp}/gamma_b"] = np.stack([g.numpy() for g in gammas[1::2]])
        for k in ("isothermal_compressibility", "tau_p"):
            out[f"{grp}/{k}"] = getattr(md, k).clone().numpy()
        out[f"{grp}/dt"], out[f"{grp}/kT"] = np.array(dt), np.array(kT)
        out[f"{grp}/p_ext"], out[f"{grp}/tau"] = np.asarray(pe), np.array(5 * dt)
    np.savez_compressed(os.path.join(HERE, "crescale.npz"), **out)
    print("C-rescale fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TORCH_SIM_REF", ""))
