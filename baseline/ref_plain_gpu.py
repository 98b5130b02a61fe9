"""The reference's own torch path on the GPU: the metric's "plain GPU path".

Runs, from the reference installed in ``baseline/_ref`` (``install_ref.py``),
``torch_sim.models.morse.MorseModel`` + ``torch_sim.nvt_langevin_step`` (its
default neighbour list, ``torch_nl_linked_cell``, rebuilt every call: the
reference has no Verlet list for pair models) on the batched Cu Morse NVT
workload, and prints one JSON line with the atom-steps/s it reaches and the
force error of the chosen dtype against a float64 evaluation by the same
reference model.

The reference's batched cell list pads every system to the largest one and to
the batch-wide shift superset, so its memory grows with systems x 512 x 125;
the batch is a seeded random sample of the workload's systems (the same mix),
halved until it fits the device.

Usage (from bench.py, in a child process so that its device memory is freed):
``python baseline/ref_plain_gpu.py --systems 1024 --steps 5 --warmup 2``.
Nothing here is part of the tsb product; it measures the reference only.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF = os.path.join(HERE, "_ref")


def _import_reference():
    """Put the installed reference on sys.path with a stub ``tables`` module
    (PyTables is absent; the reference imports it at module level for its HDF5
    trajectory writer, which this measurement does not use)."""
    if not os.path.isdir(os.path.join(REF, "torch_sim")):
        raise ImportError("baseline/_ref holds no reference install")
    d = tempfile.mkdtemp(prefix="tsref_stub_")
    with open(os.path.join(d, "tables.py"), "w") as f:
        f.write("class _Dummy:\n    def __init__(self, *a, **k):\n        pass\n"
                "def __getattr__(name):\n    return _Dummy\n")
    sys.path[:0] = [d, REF]
    import torch_sim  # noqa: F401

    return torch_sim


def _subset(d, sel):
    import numpy as np

    counts = np.bincount(d["system_idx"])
    off = np.concatenate([[0], np.cumsum(counts)])
    return {
        "positions": np.concatenate([d["positions"][off[s]:off[s + 1]] for s in sel]),
        "masses": np.concatenate([d["masses"][off[s]:off[s + 1]] for s in sel]),
        "atomic_numbers": np.concatenate([d["atomic_numbers"][off[s]:off[s + 1]] for s in sel]),
        "system_idx": np.concatenate([np.full(counts[s], k) for k, s in enumerate(sel)]),
        "cell": d["cell"][sel], "pbc": d["pbc"],
    }


def run(n_systems=2048, systems=1024, steps=5, warmup=2, dtype="float32", device="cuda"):
    import numpy as np
    import torch

    ts = _import_reference()
    from torch_sim.models.morse import MorseModel

    sys.path.insert(0, os.path.join(REPO, "torch-sim_b200"))
    from tsb import workloads as W

    dev = torch.device(device)
    if dev.type == "cpu":
        torch.set_num_threads(os.cpu_count() or 1)
    dt_ = getattr(torch, dtype)
    d = W.copper_batch(n_systems, 8, 512, seed=0)
    perm = np.random.default_rng(0).permutation(n_systems)
    dt = torch.tensor(0.002 * W.METAL_TIME, dtype=dt_, device=dev)
    kT = torch.tensor(1000.0 * W.KB_EV, dtype=dt_, device=dev)
    gamma = torch.tensor(10.0 / W.METAL_TIME, dtype=dt_, device=dev)

    def state(sub, dtype_):
        T = lambda x, t: torch.as_tensor(np.asarray(x), dtype=t, device=dev)  # noqa: E731
        return ts.SimState(positions=T(sub["positions"], dtype_), masses=T(sub["masses"], dtype_),
                           cell=T(sub["cell"], dtype_), pbc=T(sub["pbc"], torch.bool),
                           atomic_numbers=T(sub["atomic_numbers"], torch.long),
                           system_idx=T(sub["system_idx"], torch.long))

    def model(dtype_):
        return MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0, device=dev,
                          dtype=dtype_)

    take = min(systems, n_systems)
    while True:
        sub = _subset(d, perm[:take])
        try:
            st = state(sub, dt_)
            st.rng = 1
            m = model(dt_)
            md = ts.nvt_langevin_init(st, m, kT=kT)
            for _ in range(warmup):
                md = ts.nvt_langevin_step(md, m, dt=dt, kT=kT, gamma=gamma)
            if dev.type == "cuda":
                torch.cuda.synchronize(dev)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                for _ in range(steps):
                    md = ts.nvt_langevin_step(md, m, dt=dt, kT=kT, gamma=gamma)
                b.record()
                torch.cuda.synchronize(dev)
                sec = a.elapsed_time(b) / 1e3
            else:
                import time

                t0 = time.perf_counter()
                for _ in range(steps):
                    md = ts.nvt_langevin_step(md, m, dt=dt, kT=kT, gamma=gamma)
                sec = time.perf_counter() - t0
            break
        except torch.OutOfMemoryError:
            md = st = m = None
            if dev.type == "cuda":
                torch.cuda.empty_cache()
            if take <= 16:
                raise
            take //= 2
    n_atoms = int(len(sub["masses"]))
    peak_gb = torch.cuda.max_memory_allocated(dev) / 1e9 if dev.type == "cuda" else None
    # force error of this dtype against float64, both by the reference model, on
    # the final configuration of a 64-system part of the sample
    part = _subset(d, perm[:min(64, take)])
    n_part = len(part["masses"])
    part["positions"] = md.positions[:n_part].double().cpu().numpy()
    f_lo = model(dt_)(state(part, dt_))["forces"].double()
    f_hi = model(torch.float64)(state(part, torch.float64))["forces"]
    err = float((f_lo - f_hi).abs().max() / f_hi.abs().max())
    return {
        "value": n_atoms * steps / sec, "unit": "atom-steps/s", "systems": take,
        "of_systems": n_systems, "atoms": n_atoms, "md_steps": steps, "warmup": warmup,
        "ms_per_md_step": 1e3 * sec / steps, "dtype": dtype, "device": str(dev),
        "threads": torch.get_num_threads() if dev.type == "cpu" else None,
        "peak_device_gb": peak_gb, "force_err_vs_fp64": err,
        "what": "reference torch_sim MorseModel + nvt_langevin_step (torch_nl_linked_cell "
                "rebuilt every call), imported from baseline/_ref",
    }


def _timed(fn, steps, dev):
    import time

    import torch

    if dev.type == "cuda":
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            fn()
        b.record()
        torch.cuda.synchronize(dev)
        return a.elapsed_time(b) / 1e3
    t0 = time.perf_counter()
    for _ in range(steps):
        fn()
    return time.perf_counter() - t0


def run_other(config, systems=1024, steps=3, warmup=1, dtype="float64", device="cuda"):
    """The reference on the other workloads, same seeded inputs as tsb's bench:
    c1 LJ argon 256 atoms NVE (100 steps), c2 one 500,000-atom LJ force
    evaluation (linked cell rebuilt per call), c4 Kob-Andersen FIRE + Frechet
    cell filter on a sample of the 1024 boxes."""
    import numpy as np
    import torch

    ts = _import_reference()
    from torch_sim.models.lennard_jones import LennardJonesModel, lennard_jones_pair
    from torch_sim.models.pair_potential import PairPotentialModel

    sys.path.insert(0, os.path.join(REPO, "torch-sim_b200"))
    from tsb import workloads as W

    dev = torch.device(device)
    dt_ = getattr(torch, dtype)
    T = lambda x, t: torch.as_tensor(np.asarray(x), dtype=t, device=dev)  # noqa: E731

    def state(d):
        return ts.SimState(positions=T(d["positions"], dt_), masses=T(d["masses"], dt_),
                           cell=T(d["cell"], dt_), pbc=T(d["pbc"], torch.bool),
                           atomic_numbers=T(d["atomic_numbers"], torch.long),
                           system_idx=T(d["system_idx"], torch.long))

    res = {"config": config, "dtype": dtype, "device": str(dev)}
    if config == "c1":
        d = W.argon_fcc((4, 4, 4), jitter=0.05, seed=1)
        st = state(d)
        st.rng = 2024
        m = LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=2.5 * 3.405, device=dev,
                              dtype=dt_)
        dt = torch.tensor(0.002 * W.METAL_TIME, dtype=dt_, device=dev)
        box = [ts.nve_init(st, m, kT=torch.tensor(50 * W.KB_EV, dtype=dt_, device=dev))]

        def step():
            box[0] = ts.nve_step(box[0], m, dt=dt)

        for _ in range(warmup):
            step()
        sec = _timed(step, 100, dev)
        res.update(atoms=256, md_steps=100, ms_per_md_step=10.0 * sec,
                   value=256 * 100 / sec, unit="atom-steps/s",
                   what="reference nve_step + LennardJonesModel (cell list per call)")
    elif config == "c2":
        d = W.argon_fcc((50, 50, 50), jitter=0.1, seed=0)
        st = state(d)
        m = LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=8.5, device=dev, dtype=dt_)
        for _ in range(warmup):
            m(st)
        sec = _timed(lambda: m(st), steps, dev)
        res.update(atoms=len(d["masses"]), evals=steps, ms_per_eval=1e3 * sec / steps,
                   value=len(d["masses"]) * steps / sec, unit="atom-evals/s",
                   what="reference LennardJonesModel forward (linked cell rebuilt per call)")
    elif config == "c4":
        full = W.kob_andersen_batch(1024, 64, 1000, seed=0)
        take = min(systems, 1024)
        sig = torch.tensor([[1.0, 0.8], [0.8, 0.88]], dtype=dt_, device=dev) * 3.4
        eps = torch.tensor([[1.0, 1.5], [1.5, 0.5]], dtype=dt_, device=dev) * 0.0104

        def pf(r, zi, zj):
            a, b = zi - 1, zj - 1
            s_, e_ = sig[a, b], eps[a, b]
            v = lennard_jones_pair(r, zi, zj, s_, e_) - lennard_jones_pair(2.5 * s_, zi, zj,
                                                                          s_, e_)
            return torch.where(r < 2.5 * s_, v, torch.zeros_like(v))

        while True:
            sub = _subset(full, np.arange(take))
            try:
                m = PairPotentialModel(pair_fn=pf, cutoff=8.5, compute_stress=True, device=dev,
                                       dtype=dt_)
                box = [ts.fire_init(state(sub), m, cell_filter=ts.CellFilter.frechet)]

                def step():
                    box[0] = ts.fire_step(box[0], m)

                for _ in range(warmup):
                    step()
                sec = _timed(step, steps, dev)
                break
            except torch.OutOfMemoryError:
                box = m = None
                if dev.type == "cuda":
                    torch.cuda.empty_cache()
                if take <= 8:
                    raise
                take //= 2
        n = len(sub["masses"])
        res.update(systems=take, of_systems=1024, atoms=n, fire_steps=steps,
                   ms_per_fire_step=1e3 * sec / steps, value=n * steps / sec,
                   unit="atom-steps/s",
                   what="reference fire_step (ase_fire) + CellFilter.frechet, Kob-Andersen "
                        "PairPotentialModel (cell list per call)")
    if dev.type == "cuda":
        res["peak_device_gb"] = torch.cuda.max_memory_allocated(dev) / 1e9
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c3", choices=["c1", "c2", "c3", "c4"])
    ap.add_argument("--n-systems", type=int, default=2048)
    ap.add_argument("--systems", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--dtype", default="float32", choices=["float32", "float64"])
    ap.add_argument("--device", default="cuda")
    a = ap.parse_args()
    if a.config == "c3":
        out = run(a.n_systems, a.systems, a.steps, a.warmup, a.dtype, a.device)
    else:
        out = run_other(a.config, a.systems, a.steps, a.warmup, a.dtype, a.device)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
