"""Time the reference's own torch CPU path (float64) on the workload configs
(BASELINE ONLY; never the product path, never run on the GPU box).

Run in a container where the reference source tree is present::

    python oracle/ref_cpu_timing.py c1|c2 <cells>|c3 <systems>|c4 <systems> [/path/to/torch-sim]

It imports the reference through the same shims as tests/golden/make_golden.py
(stub ``tables`` module, dist metadata), uses every host core, and prints one
JSON line: the rate per atom-step (or atom-evaluation), the thread count and
the peak resident memory.
"""
import json
import os
import resource
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "tests", "golden"))
sys.path.insert(0, os.path.join(REPO, "torch-sim_b200"))
from make_golden import _install_shims  # noqa: E402

_install_shims(sys.argv[3] if len(sys.argv) > 3 else "/root/reference")
import numpy as np  # noqa: E402
import torch  # noqa: E402
torch.set_default_dtype(torch.float64)
torch.set_num_threads(os.cpu_count())
import torch_sim as ts
from torch_sim.models.lennard_jones import LennardJonesModel
from torch_sim.models.morse import MorseModel
from tsb import workloads as W
T = lambda x, dt=torch.float64: torch.as_tensor(np.asarray(x), dtype=dt)
def state(d):
    return ts.SimState(positions=T(d["positions"]), masses=T(d["masses"]), cell=T(d["cell"]),
                       pbc=T(d["pbc"], torch.bool), atomic_numbers=T(d["atomic_numbers"], torch.long),
                       system_idx=T(d["system_idx"], torch.long))
which = sys.argv[1]
res = {"threads": torch.get_num_threads()}
dt = 0.002 * W.METAL_TIME
if which == "c1":
    d = W.argon_fcc((4, 4, 4), jitter=0.05, seed=1); st = state(d); st.rng = 2024
    m = LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=2.5 * 3.405)
    md = ts.nve_init(st, m, kT=torch.tensor(50 * W.KB_EV))
    md = ts.nve_step(md, m, dt=torch.tensor(dt))
    t = time.perf_counter()
    for _ in range(100):
        md = ts.nve_step(md, m, dt=torch.tensor(dt))
    el = time.perf_counter() - t
    res.update(per_step_s=el / 100, atom_steps_per_s=256 * 100 / el)
elif which == "c3":
    ns = int(sys.argv[2])
    d = W.copper_batch(2048, 8, 512, seed=0)
    counts = np.bincount(d["system_idx"]); off = np.concatenate([[0], np.cumsum(counts)])
    sel = np.random.default_rng(0).permutation(2048)[:ns]
    sub = {"positions": np.concatenate([d["positions"][off[s]:off[s+1]] for s in sel]),
           "masses": np.concatenate([d["masses"][off[s]:off[s+1]] for s in sel]),
           "atomic_numbers": np.concatenate([d["atomic_numbers"][off[s]:off[s+1]] for s in sel]),
           "system_idx": np.concatenate([np.full(counts[s], k) for k, s in enumerate(sel)]),
           "cell": d["cell"][sel], "pbc": d["pbc"]}
    st = state(sub); st.rng = 1
    m = MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0)
    kT = torch.tensor(1000 * W.KB_EV); g = torch.tensor(10.0 / W.METAL_TIME)
    md = ts.nvt_langevin_init(st, m, kT=kT)
    md = ts.nvt_langevin_step(md, m, dt=torch.tensor(dt), kT=kT, gamma=g)
    ts_ = []
    for _ in range(5):
        t = time.perf_counter(); md = ts.nvt_langevin_step(md, m, dt=torch.tensor(dt), kT=kT, gamma=g)
        ts_.append(time.perf_counter() - t)
    med = float(np.median(ts_))
    res.update(systems=ns, atoms=int(len(sub["masses"])), median_step_s=med,
               atom_steps_per_s=len(sub["masses"]) / med)
elif which == "c4":
    ns = int(sys.argv[2])
    d = W.kob_andersen_batch(ns, 64, 1000, seed=0)
    st = state(d)
    from torch_sim.models.pair_potential import PairPotentialModel
    from torch_sim.models.lennard_jones import lennard_jones_pair
    sig = torch.tensor([[1.0, 0.8], [0.8, 0.88]]) * 3.4
    eps = torch.tensor([[1.0, 1.5], [1.5, 0.5]]) * 0.0104
    def pf(r, zi, zj):
        a, b = zi - 1, zj - 1
        s, e = sig[a, b], eps[a, b]
        v = lennard_jones_pair(r, zi, zj, s, e) - lennard_jones_pair(2.5 * s, zi, zj, s, e)
        return torch.where(r < 2.5 * s, v, torch.zeros_like(v))
    m = PairPotentialModel(pair_fn=pf, cutoff=8.5, compute_stress=True)
    fs = ts.fire_init(st, m, cell_filter=ts.CellFilter.frechet)
    fs = ts.fire_step(fs, m)
    ts_ = []
    for _ in range(5):
        t = time.perf_counter(); fs = ts.fire_step(fs, m); ts_.append(time.perf_counter() - t)
    med = float(np.median(ts_))
    res.update(systems=ns, atoms=int(len(d["masses"])), median_step_s=med,
               atom_steps_per_s=len(d["masses"]) / med)
if which == "c2":
    nc = int(sys.argv[2])
    d = W.argon_fcc((nc, nc, nc), jitter=0.1, seed=0); st = state(d)
    m = LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=8.5)
    m(st)
    ts_ = []
    for _ in range(3):
        t = time.perf_counter(); m(st); ts_.append(time.perf_counter() - t)
    med = float(np.median(ts_))
    res.update(atoms=int(len(d["masses"])), median_eval_s=med, atom_evals_per_s=len(d["masses"]) / med)
res["peak_rss_gb"] = resource.getrusage(resource.RUSAGE_SELF).ru_maxrss / 1e6
res["which"] = which
print(json.dumps(res))
