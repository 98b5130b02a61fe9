"""Generate the golden fixtures by running the reference TorchSim itself.

Run in a container where the reference source tree is present::

    python tests/golden/make_golden.py /path/to/torch-sim

The reference package imports ``tables`` (PyTables) at module level and reads
its own dist metadata; neither is needed on the hot path, so this script puts a
stub ``tables`` module and a dist-info directory on ``sys.path`` first.

Outputs (small ``.npz`` files beside this script):

* ``nl.npz``        neighbour pair sets from ``torch_nl_linked_cell`` (and a
                    cross-check against ``torch_nl_n2``) on cubic, triclinic,
                    partial-PBC, non-periodic and self-image cases
* ``models.npz``    energy / forces / stress / per-atom energies and stresses of
                    LennardJonesModel, MorseModel, SoftSphereModel,
                    SoftSphereMultiModel and harness PairPotentialModels (energy-
                    shifted LJ, Kob-Andersen species-matrix LJ)
* ``md.npz``        NVE (velocity Verlet) and NVT-Langevin (BAOAB) trajectories,
                    with the Langevin noise recorded
* ``fire.npz``      ASE-FIRE + Frechet cell filter and VV-FIRE trajectories
* ``adjoint.npz``   gradients of a 20-step NVE histogram loss w.r.t. sigma,
                    epsilon, q0, p0 by FP64 autograd with create_graph=True (the
                    exact trajectory derivative), and the reference's own
                    retain_graph=True route for comparison
* ``math.npz``      expm / Frechet derivative / matrix log of 3x3 batches
"""

from __future__ import annotations

import functools
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _install_shims(ref_root):
    d = tempfile.mkdtemp(prefix="tsref_")
    with open(os.path.join(d, "tables.py"), "w") as f:
        f.write("class _Dummy:\n    def __init__(self, *a, **k):\n        pass\n"
                "def __getattr__(name):\n    return _Dummy\n")
    meta = os.path.join(d, "torch_sim_atomistic-0.6.1.dist-info")
    os.makedirs(meta)
    with open(os.path.join(meta, "METADATA"), "w") as f:
        f.write("Metadata-Version: 2.1\nName: torch-sim-atomistic\nVersion: 0.6.1\n")
    sys.path[:0] = [d, ref_root]


def main(ref_root):
    _install_shims(ref_root)
    sys.path.insert(0, os.path.join(REPO, "torch-sim_b200"))
    import torch

    torch.set_default_dtype(torch.float64)
    import torch_sim as ts
    from torch_sim.models.lennard_jones import LennardJonesModel, lennard_jones_pair
    from torch_sim.models.morse import MorseModel
    from torch_sim.models.pair_potential import PairPotentialModel
    from torch_sim.models.soft_sphere import SoftSphereModel, SoftSphereMultiModel
    from torch_sim.neighbors import torch_nl_linked_cell, torch_nl_n2

    from tsb import workloads as W

    def T(x, dt=torch.float64):
        return torch.as_tensor(np.asarray(x), dtype=dt)

    def to_state(d):
        return ts.SimState(positions=T(d["positions"]), masses=T(d["masses"]),
                           cell=T(d["cell"]), pbc=T(d["pbc"], torch.bool),
                           atomic_numbers=T(d["atomic_numbers"], torch.long),
                           system_idx=T(d["system_idx"], torch.long))

    # ------------------------------------------------------------------ NL
    rng = np.random.default_rng(1234)
    cases = {}
    cases["ar_fcc444"] = (W.argon_fcc((4, 4, 4), jitter=0.05, seed=0), 2.5 * 3.405, None)
    cases["cu_tri_batch"] = (W.copper_batch(6, 4, 120, seed=3, jitter=0.05), 6.0, None)
    slab = W.copper_batch(2, 30, 60, seed=5, jitter=0.1)
    slab["positions"] = slab["positions"] + rng.normal(0, 3.0, slab["positions"].shape)
    cases["slab_pbc_TTF"] = (slab, 5.0, np.array([True, True, False]))
    clus = W.argon_fcc((2, 2, 2), jitter=0.3, seed=7)
    clus["positions"] = clus["positions"] + 40.0 * rng.normal(size=3)
    cases["cluster_nopbc"] = (clus, 7.0, np.array([False, False, False]))
    tiny = {"positions": np.array([[0.3, 0.2, 0.1]]), "masses": np.array([1.0]),
            "cell": np.array([np.eye(3) * 2.0 + np.array([[0, 0.3, 0], [0, 0, 0],
                                                            [0.2, 0, 0]])]),
            "pbc": np.array([True] * 3), "atomic_numbers": np.array([1]),
            "system_idx": np.array([0])}
    cases["tiny_self_images"] = (tiny, 4.5, None)
    rh = W.argon_fcc((1, 1, 1), a=4.0, jitter=0.2, seed=11)
    ang = np.deg2rad(60.0)
    cell_row = 4.0 * np.array([[1, 0, 0], [np.cos(ang), np.sin(ang), 0],
                               [np.cos(ang), (np.cos(ang) - np.cos(ang) ** 2) / np.sin(ang),
                                0]])
    cell_row[2, 2] = np.sqrt(16.0 - cell_row[2, 0] ** 2 - cell_row[2, 1] ** 2)
    rh["positions"] = rng.uniform(0, 1, (4, 3)) @ cell_row + 4.0 * rng.normal(size=(4, 3))
    rh["cell"] = cell_row.T[None]
    cases["rhombohedral_unwrapped"] = (rh, 6.5, None)
    out = {}
    for name, (d, rc, pbc) in cases.items():
        st = to_state(d)
        pb = T(d["pbc"] if pbc is None else pbc, torch.bool)
        n_sys = int(d["system_idx"].max()) + 1
        pbb = pb.unsqueeze(0).expand(n_sys, 3)
        for si in (False, True):
            m, sm, sh = torch_nl_linked_cell(st.positions, st.row_vector_cell, pbb, rc,
                                             st.system_idx, self_interaction=si)
            key = f"{name}{'_self' if si else ''}"
            m2, sm2, sh2 = torch_nl_n2(st.positions, st.row_vector_cell, pbb, rc,
                                       st.system_idx, self_interaction=si)
            out[f"{key}/n2_count"] = np.array(m2.shape[1])
            out[f"{key}/mapping"] = m.numpy().astype(np.int32)
            out[f"{key}/system_mapping"] = sm.numpy().astype(np.int32)
            out[f"{key}/shifts"] = np.rint(sh.numpy()).astype(np.int16)
        out[f"{name}/positions"] = d["positions"]
        out[f"{name}/cell_row"] = np.transpose(d["cell"], (0, 2, 1))
        out[f"{name}/pbc"] = np.asarray(d["pbc"] if pbc is None else pbc)
        out[f"{name}/system_idx"] = d["system_idx"].astype(np.int32)
        out[f"{name}/cutoff"] = np.array(rc)
    np.savez_compressed(os.path.join(HERE, "nl.npz"), **out)

    # -------------------------------------------------------------- models
    out = {}

    def run_model(key, model, d, pbc=None):
        st = to_state(d)
        if pbc is not None:
            st.pbc = T(pbc, torch.bool)
        r = model(st)
        for k, v in r.items():
            out[f"{key}/{k}"] = v.detach().numpy()
        for k in ("positions", "cell", "system_idx", "atomic_numbers"):
            out[f"{key}/{k}"] = np.asarray(d[k])
        out[f"{key}/pbc"] = np.asarray(d["pbc"] if pbc is None else pbc)

    ar = cases["ar_fcc444"][0]
    kw = dict(compute_stress=True, per_atom_energies=True, per_atom_stresses=True)
    run_model("lj_ar", LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=2.5 * 3.405,
                                         **kw), ar)
    cu = cases["cu_tri_batch"][0]
    run_model("morse_cu", MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588,
                                     cutoff=6.0, **kw), cu)
    run_model("morse_slab", MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588,
                                       cutoff=5.0, **kw), slab, pbc=[True, True, False])
    box = {"positions": rng.uniform(0, 9.0, (60, 3)), "masses": np.ones(60),
           "cell": np.eye(3)[None] * 9.0, "pbc": np.array([True] * 3),
           "atomic_numbers": rng.choice([18, 36], 60), "system_idx": np.zeros(60, int)}
    run_model("soft_sphere", SoftSphereModel(sigma=2.6, epsilon=0.05, alpha=2.0, **kw),
              box)
    run_model("soft_sphere_a3", SoftSphereModel(sigma=2.6, epsilon=0.05, alpha=3.5, **kw),
              box)
    sig = torch.tensor([[2.6, 2.9], [2.9, 3.1]])
    eps = torch.tensor([[0.05, 0.07], [0.07, 0.04]])
    alp = torch.tensor([[2.0, 2.5], [2.5, 3.0]])
    run_model("soft_sphere_multi",
              SoftSphereMultiModel(atomic_numbers=torch.tensor([18, 36]), sigma_matrix=sig,
                                   epsilon_matrix=eps, alpha_matrix=alp, **kw), box)
    alp_int = torch.tensor([[2.0, 3.0], [3.0, 2.0]])
    run_model("soft_sphere_multi_int",
              SoftSphereMultiModel(atomic_numbers=torch.tensor([18, 36]), sigma_matrix=sig,
                                   epsilon_matrix=eps, alpha_matrix=alp_int, **kw), box)
    rc = 2.5 * 3.405
    e_rc = float(lennard_jones_pair(torch.tensor([rc]), None, None, 3.405, 0.0104)[0])

    def lj_shifted(dr, zi, zj):
        return lennard_jones_pair(dr, zi, zj, 3.405, 0.0104) - e_rc

    run_model("lj_shifted", PairPotentialModel(pair_fn=lj_shifted, cutoff=rc,
                                               reduce_to_half_list=True, **kw), ar)
    # Kob-Andersen species-matrix LJ, truncated and shifted at 2.5 sigma_ab
    ka = W.kob_andersen_batch(2, 64, 90, seed=9)
    s_aa, e_aa = 3.4, 0.0104
    sigm = torch.tensor([[1.0, 0.8], [0.8, 0.88]]) * s_aa
    epsm = torch.tensor([[1.0, 1.5], [1.5, 0.5]]) * e_aa
    rcm = 2.5 * sigm
    shiftm = 4 * epsm * ((sigm / rcm) ** 12 - (sigm / rcm) ** 6)

    def ka_pair(dr, zi, zj):
        a, b = zi - 1, zj - 1
        s, e, r_c, sh = sigm[a, b], epsm[a, b], rcm[a, b], shiftm[a, b]
        v = 4 * e * ((s / dr) ** 12 - (s / dr) ** 6) - sh
        return torch.where((dr > 0) & (dr < r_c), v, torch.zeros_like(v))

    run_model("ka_lj", PairPotentialModel(pair_fn=ka_pair, cutoff=2.5 * s_aa,
                                          reduce_to_half_list=True, **kw), ka)
    np.savez_compressed(os.path.join(HERE, "models.npz"), **out)

    # ------------------------------------------------------------------ MD
    out = {}
    small = W.argon_fcc((2, 2, 2), jitter=0.05, seed=2)
    st = to_state(small)
    lj = LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=2.5 * 3.405)
    kT = 50.0 * W.KB_EV
    st.rng = 42
    md = ts.nve_init(st, lj, kT=torch.tensor(kT))
    dt = 0.002 * W.METAL_TIME
    traj = [(md.positions.clone(), md.momenta.clone(), md.energy.clone(),
             md.forces.clone())]
    for _ in range(10):
        md = ts.nve_step(md, lj, dt=torch.tensor(dt))
        traj.append((md.positions.clone(), md.momenta.clone(), md.energy.clone(),
                     md.forces.clone()))
    for k, name in enumerate(("positions", "momenta", "energy", "forces")):
        out[f"nve/{name}"] = np.stack([t[k].numpy() for t in traj])
    for k in ("masses", "cell", "system_idx"):
        out[f"nve/{k}"] = small[k]
    out["nve/dt"] = np.array(dt)

    cu3 = W.copper_batch(3, 8, 40, seed=21, jitter=0.03)
    st = to_state(cu3)
    morse = MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0)
    kT = 1000.0 * W.KB_EV
    st.rng = 7
    md = ts.nvt_langevin_init(st, morse, kT=torch.tensor(kT))
    gamma = 10.0 / W.METAL_TIME  # 10 ps^-1 in internal units
    noises = []
    real_randn = torch.randn

    def rec_randn(*a, **k):
        x = real_randn(*a, **k)
        noises.append(x.clone())
        return x

    traj = [(md.positions.clone(), md.momenta.clone(), md.energy.clone(),
             md.forces.clone())]
    torch.randn = rec_randn
    try:
        for _ in range(5):
            md = ts.nvt_langevin_step(md, morse, dt=torch.tensor(dt), kT=torch.tensor(kT),
                                      gamma=torch.tensor(gamma))
            traj.append((md.positions.clone(), md.momenta.clone(), md.energy.clone(),
                         md.forces.clone()))
    finally:
        torch.randn = real_randn
    for k, name in enumerate(("positions", "momenta", "energy", "forces")):
        out[f"nvt/{name}"] = np.stack([t[k].numpy() for t in traj])
    out["nvt/noise"] = np.stack([n.numpy() for n in noises])
    for k in ("masses", "cell", "system_idx"):
        out[f"nvt/{k}"] = cu3[k]
    out["nvt/dt"] = np.array(dt)
    out["nvt/kT"] = np.array(kT)
    out["nvt/gamma"] = np.array(gamma)
    np.savez_compressed(os.path.join(HERE, "md.npz"), **out)

    # ---------------------------------------------------------------- FIRE
    out = {}
    ka2 = W.kob_andersen_batch(2, 40, 60, seed=33)
    model = PairPotentialModel(pair_fn=ka_pair, cutoff=2.5 * s_aa, reduce_to_half_list=True,
                               compute_stress=True)
    st = to_state(ka2)
    fs = ts.fire_init(st, model, cell_filter=ts.CellFilter.frechet)
    keys = ("positions", "cell", "velocities", "forces", "energy", "stress", "dt",
            "alpha", "n_pos", "cell_positions", "cell_velocities", "cell_forces")
    traj = [{k: getattr(fs, k).clone() for k in keys}]
    for _ in range(12):
        fs = ts.fire_step(fs, model)
        traj.append({k: getattr(fs, k).clone() for k in keys})
    for k in keys:
        out[f"ase_frechet/{k}"] = np.stack([t[k].numpy() for t in traj])
    for k in ("masses", "system_idx", "atomic_numbers"):
        out[f"ase_frechet/{k}"] = ka2[k]
    # VV-FIRE has no step clamp, so start from a jittered lattice (random overlapping
    # starts make it chaotic at the rounding level)
    vv = W.argon_fcc((2, 2, 2), a=5.4, jitter=0.15, seed=17, n_systems=2)
    vv["atomic_numbers"] = np.where(rng.uniform(size=len(vv["masses"])) < 0.8, 1, 2)
    ka2 = vv
    st = to_state(ka2)
    fs = ts.fire_init(st, model, fire_flavor="vv_fire")
    keys = ("positions", "velocities", "forces", "energy", "dt", "alpha", "n_pos")
    traj = [{k: getattr(fs, k).clone() for k in keys}]
    for _ in range(8):
        fs = ts.fire_step(fs, model, fire_flavor="vv_fire")
        traj.append({k: getattr(fs, k).clone() for k in keys})
    for k in keys:
        out[f"vv/{k}"] = np.stack([t[k].numpy() for t in traj])
    for k in ("masses", "system_idx", "atomic_numbers", "cell"):
        out[f"vv/{k}"] = ka2[k]
    np.savez_compressed(os.path.join(HERE, "fire.npz"), **out)

    # ------------------------------------------------------------- adjoint
    # FP64 restatement of an NVE trajectory with autograd through the forces
    # (create_graph=True keeps the Hessian terms), on the reference's own LJ
    # pair function and neighbour list; plus the reference's retain_graph route.
    from torch_sim.models.pair_potential import full_to_half_list
    from torch_sim.transforms import compute_cell_shifts

    out = {}
    ad = W.argon_species_batch(2, (2, 2, 2), jitter=0.05, seed=5)
    n_steps, dt_ad, rc_ad = 20, 0.002 * W.METAL_TIME, 2.5 * 3.405
    sp = T(ad["atomic_numbers"] - 1, torch.long)
    row_cell = T(np.transpose(ad["cell"], (0, 2, 1)))
    pbc2 = torch.ones((2, 3), dtype=torch.bool)
    sysi = T(ad["system_idx"], torch.long)
    masses = T(ad["masses"])
    gen = torch.Generator().manual_seed(11)
    p0 = torch.randn((len(masses), 3), generator=gen, dtype=torch.float64) * torch.sqrt(
        masses * 80.0 * W.KB_EV).unsqueeze(-1)
    q0 = T(ad["positions"])
    rng_ad = np.random.default_rng(4)
    sig0 = torch.full((2, 2), 3.405, dtype=torch.float64)
    eps0 = torch.full((2, 2), 0.0104, dtype=torch.float64)
    sig = sig0.clone()
    eps_ = eps0.clone()
    for a_ in range(2):
        for b_ in range(a_, 2):
            fs, fe = 1 + rng_ad.uniform(-0.05, 0.05, 2)
            sig[a_, b_] = sig[b_, a_] = 3.405 * fs
            eps_[a_, b_] = eps_[b_, a_] = 0.0104 * fe

    def pairs_of(q, cut):
        m, sm, sh = torch_nl_linked_cell(q.detach(), row_cell, pbc2, cut, sysi)
        m, sm, sh = full_to_half_list(m, sm, sh)
        cs = compute_cell_shifts(row_cell, sh, sm)
        return m, sm, q[m[1]] - q[m[0]] + cs

    def energy(q, sg, ep):
        m, _, dr = pairs_of(q, rc_ad)
        r = dr.norm(dim=1)
        a_, b_ = sp[m[0]], sp[m[1]]
        v = lennard_jones_pair(r, None, None, sg[a_, b_], ep[a_, b_])
        return torch.where(r < rc_ad, v, torch.zeros_like(v)).sum()

    def force(q, sg, ep, graph=True):
        (g_,) = torch.autograd.grad(energy(q, sg, ep), q, create_graph=graph)
        return -g_

    centers = (torch.arange(64, dtype=torch.float64) + 0.5) * (8.0 / 64)

    def hist(q):
        m, sm, dr = pairs_of(q, 8.0)
        r = dr.norm(dim=1)
        w_ = torch.exp(-((r[:, None] - centers[None]) ** 2) / (2 * 0.05 ** 2))
        w_ = torch.where((r < 8.0)[:, None], w_, torch.zeros_like(w_))
        return torch.zeros((2, 64), dtype=torch.float64).index_add(0, sm, w_)

    def run(q, p, sg, ep, graph=True):
        f = force(q, sg, ep, graph)
        for _ in range(n_steps):
            p = p + f * (dt_ad / 2)
            q = q + p / masses.unsqueeze(-1) * dt_ad
            f = force(q, sg, ep, graph)
            p = p + f * (dt_ad / 2)
        return q

    q_t = run(q0.clone().requires_grad_(True), p0, sig0, eps0, graph=False).detach()
    target = hist(q_t).detach()
    sg_ = sig.clone().requires_grad_(True)
    ep_ = eps_.clone().requires_grad_(True)
    qq = q0.clone().requires_grad_(True)
    pp = p0.clone().requires_grad_(True)
    loss = ((hist(run(qq, pp, sg_, ep_)) - target) ** 2).sum()
    gs_, ge_, gq_, gp_ = torch.autograd.grad(loss, [sg_, ep_, qq, pp])
    out["adj/positions"] = ad["positions"]
    out["adj/cell"] = ad["cell"]
    out["adj/masses"] = ad["masses"]
    out["adj/system_idx"] = ad["system_idx"]
    out["adj/atomic_numbers"] = ad["atomic_numbers"]
    out["adj/p0"] = p0.numpy()
    out["adj/sigma"] = sig.numpy()
    out["adj/epsilon"] = eps_.numpy()
    out["adj/target"] = target.numpy()
    out["adj/loss"] = np.array(float(loss))
    out["adj/n_steps"] = np.array(n_steps)
    out["adj/dt"] = np.array(dt_ad)
    sym = lambda g_: (g_ + g_.T - torch.diag(torch.diagonal(g_))).numpy()  # noqa: E731
    out["adj/grad_sigma"] = sym(gs_)
    out["adj/grad_epsilon"] = sym(ge_)
    out["adj/grad_q0"] = gq_.numpy()
    out["adj/grad_p0"] = gp_.numpy()
    # the reference's route: PairPotentialModel(retain_graph=True) inside nve_step
    def ka2(dr, zi, zj, sg=sg_, ep=ep_):
        return lennard_jones_pair(dr, zi, zj, sg[zi - 1, zj - 1], ep[zi - 1, zj - 1])

    model_rg = PairPotentialModel(pair_fn=ka2, cutoff=rc_ad, reduce_to_half_list=True,
                                  retain_graph=True)
    st = to_state(ad)
    st.positions = q0.clone().requires_grad_(True)
    q_leaf = st.positions
    md = ts.nve_init(st, model_rg, kT=torch.tensor(80.0 * W.KB_EV))
    md.momenta = p0.clone()
    md.forces = model_rg(md)["forces"]
    for _ in range(n_steps):
        md = ts.nve_step(md, model_rg, dt=torch.tensor(dt_ad))
    loss_rg = ((hist(md.positions) - target) ** 2).sum()
    (gq_rg,) = torch.autograd.grad(loss_rg, [q_leaf], allow_unused=True)
    out["adj/ref_retain_graph_grad_q0"] = gq_rg.numpy()
    out["adj/ref_retain_graph_loss"] = np.array(float(loss_rg))
    np.savez_compressed(os.path.join(HERE, "adjoint.npz"), **out)

    # ---------------------------------------------------------------- math
    import torch_sim.math as tsm

    A = torch.tensor(rng.normal(0, 0.3, (16, 3, 3)))
    E = torch.tensor(rng.normal(0, 1.0, (16, 3, 3)))
    R, L = tsm.expm_frechet(A, E)
    Tm = torch.eye(3) + torch.tensor(rng.normal(0, 0.05, (16, 3, 3)))
    logT = tsm.matrix_log_33(Tm)
    np.savez_compressed(os.path.join(HERE, "math.npz"), A=A.numpy(), E=E.numpy(),
                        expA=R.numpy(), L=L.numpy(), T=Tm.numpy(), logT=logT.numpy(),
                        expm_torch=torch.matrix_exp(A).numpy())
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TORCH_SIM_REF", ""))
