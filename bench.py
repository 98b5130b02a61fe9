#!/usr/bin/env python
"""Benchmark: batched uneven Morse NVT-Langevin MD on B200.

Workload (seeded synthetic, no dataset): 2048 Cu fcc supercells (a = 3.61 A)
with atom counts uniform in [8, 512] rounded to 4*n1*n2*n3, random diagonal
strain +-2 % and triclinic shear +-3 deg; Morse D = 0.3429 eV,
alpha = 1.3588 1/A, r0 = 2.866 A, cutoff 6.0 A; NVT Langevin (BAOAB) at
1000 K, dt = 2 fs, gamma = 0.01 1/fs; FP32 pair arithmetic with FP64
positions, momenta and per-system energy.

One bench "step" is one launch of the persistent fused kernel that advances
every system by --md-steps MD steps (default 500; 10 timed steps = the 5,000
MD steps of the workload).  Metric: atom-steps/s = atoms x MD steps / time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tsb|reference]

N > 1 runs under torchrun, one rank per GPU, each rank advancing its own
2048-system batch (independent systems, no collective in the step: weak
scaling).  --impl reference times the reference algorithm's CPU restatement
(the oracle port) on the host cores.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "torch-sim_b200"))

METRIC = "atom-steps/s on 1 B200 (batched fused vs plain path) at force err ≤1e-5 vs FP64"
UNIT = "atom-steps/s"
WORKLOAD = ("2048 Cu fcc systems (8-512 atoms, strain +-2%, shear +-3deg), Morse "
            "(D=0.3429 eV, alpha=1.3588/A, r0=2.866 A, rc=6.0 A), NVT-Langevin BAOAB "
            "1000 K, dt=2 fs, gamma=0.01/fs")
INTEGRATOR_NAMES = {"nvt_nose_hoover": "NVT Nose-Hoover chain (3 x 3 x 3)",
                    "nvt_vrescale": "NVT V-rescale (tau 10 dt)", "nve": "NVE velocity Verlet"}
ALG_BYTES_PER_ATOM_STEP = 76  # streaming state r/w: 48 B FP64 pos + 24 B mom + 4 B type/mass
# algorithmic compute per half-list pair of the Morse workload: ~45 FP32 flops and
# one exp (the half pairs within the cutoff are counted on the workload itself)
FLOPS_PER_PAIR = 45


def sm_peaks(device):
    """Nominal FP32 (FMA = 2 flops, 128 lanes/SM) and MUFU (16 lanes/SM) peaks at
    the maximum SM clock (the measured-peaks file has no FP32 or MUFU figure)."""
    import torch

    props = torch.cuda.get_device_properties(device)
    ghz = ClockSampler.max_sm_mhz(device.index or 0) / 1e3
    fp32 = props.multi_processor_count * 128 * 2 * ghz / 1e3  # TFLOP/s
    sfu = props.multi_processor_count * 16 * ghz  # G ops/s
    return fp32, sfu


def pair_counts(x, cell_row, system_idx, cutoff, skin, n_systems):
    """(half-list pairs within the cutoff, full-list entries within cutoff + skin,
    both per atom) of one configuration, from the neighbour-list drop-in: the
    algorithmic pairs of a step and the size of the lists the fused kernel
    evaluates every step at that skin."""
    import torch

    from tsb import neighbors

    pbc = torch.ones((n_systems, 3), dtype=torch.bool, device=x.device)
    n = x.shape[0]
    p_rc = neighbors.torchsim_nl(x, cell_row, pbc, cutoff, system_idx,
                                 n_systems=n_systems)[0].shape[1]
    p_list = neighbors.torchsim_nl(x, cell_row, pbc, cutoff + skin, system_idx,
                                   n_systems=n_systems)[0].shape[1]
    return p_rc / 2 / n, p_list / n


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tsb", choices=["tsb", "reference"])
    ap.add_argument("--md-steps", type=int, default=500)
    ap.add_argument("--n-systems", type=int, default=2048)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skin", default="auto",
                    help="Verlet skin in A, or 'auto' (project autotuner, cached per workload)")
    ap.add_argument("--lanes", default=None,
                    help="most threads per atom of small systems (power of two <= 32), or "
                         "'auto'; default: 'auto' with --skin auto, else 32")
    ap.add_argument("--prune", default=None,
                    help="pruning skin of the list's shell in A (0: off), or 'auto'; default: "
                         "'auto' with --skin auto, else a fixed fraction of the skin")
    ap.add_argument("--plain-steps", type=int, default=20,
                    help="MD steps of the plain per-call path timed beside the fused kernel")
    ap.add_argument("--integrator", default="nvt_langevin",
                    choices=["nvt_langevin", "nvt_nose_hoover", "nvt_vrescale", "nve"],
                    help="batched_md: integrator inside the fused kernel and the plain path")
    ap.add_argument("--list-skin", type=float, default=1.5,
                    help="relax workload: Verlet-list skin in A (0 = cell-list search per call)")
    ap.add_argument("--list-prune", type=float, default=None,
                    help="relax workload: pruning skin of the Verlet lists in A (default "
                         "0: off)")
    ap.add_argument("--graph-steps", type=int, default=50,
                    help="relax workload: FIRE steps per CUDA-graph replay (0 = eager loop)")
    ap.add_argument("--ref-plain-systems", type=int, default=2048,
                    help="batched_md: systems of the reference's own torch path timed on the "
                         "GPU (baseline/_ref; halved until it fits; 0: skip)")
    ap.add_argument("--no-other-workloads", action="store_true",
                    help="batched_md: skip the single_large / relax / adjoint runs whose "
                         "lines the default run attaches (child processes, run first)")
    ap.add_argument("--workload", default="batched_md",
                    choices=["batched_md", "single_large", "relax", "adjoint"])
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms in a thread."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                     "--format=csv,noheader,nounits"], capture_output=True, text=True,
                    timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:  # noqa: BLE001
                pass
            self._stop.wait(0.2)

    @staticmethod
    def max_sm_mhz(index: int) -> float:
        """clocks.max.sm of GPU `index` (B200 specification value if unreadable)."""
        try:
            out = subprocess.run(["nvidia-smi", f"--id={index}", "--query-gpu=clocks.max.sm",
                                  "--format=csv,noheader,nounits"], capture_output=True,
                                 text=True, timeout=5).stdout.strip()
            return float(out.splitlines()[0])
        except Exception:  # noqa: BLE001
            return 1965.0

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 5 + k and r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def measured_peak_hbm():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


def build_workload(n_systems, seed, device):
    import torch

    from tsb import integrators, models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(n_systems, 8, 512, seed=seed)
    st = state_from_arrays(d, device=device)
    st.rng = 1000 + seed
    model = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                              device=device)
    kT = 1000.0 * workloads.KB_EV
    md = integrators.nvt_langevin_init(st, model, kT=kT)
    torch.cuda.synchronize(device)
    return d, md, model


def cpu_baseline(d, budget_s=20.0, processes=None, n_steps=2, seed=0):
    """Oracle port on the host: a bounded sample of systems (see oracle/cpu_md.py)."""
    import numpy as np

    sys.path.insert(0, REPO)
    from oracle import cpu_md
    from tsb import workloads as W

    if processes is None:  # all host cores, as the --impl reference arm uses
        processes = cpu_md.cpu_count()
    rng = np.random.default_rng(seed)
    n_sys = int(d["system_idx"].max()) + 1
    systems = rng.permutation(n_sys)
    dt, kT, g = 0.002 * W.METAL_TIME, 1000 * W.KB_EV, 10.0 / W.METAL_TIME
    take = 4 * processes
    a, t = cpu_md.time_sample(d, systems[:take], n_steps, dt, kT, g, 6.0, processes)
    # grow the sample toward the time budget, keeping the same per-system mix
    if t < budget_s / 4:
        take = int(min(n_sys, max(take, take * budget_s / 2 / max(t, 1e-3))))
        a, t = cpu_md.time_sample(d, systems[:take], n_steps, dt, kT, g, 6.0, processes)
    atoms = int(np.bincount(d["system_idx"])[systems[:take]].sum())
    return {"value": a / t, "unit": UNIT, "cores": processes, "kind": "port",
            "sample": f"{take} of {n_sys} systems ({atoms} atoms) x {n_steps} BAOAB steps, "
                      f"numpy oracle (NL + Morse + BAOAB), {t:.1f} s"}


def reference_plain_path(n_systems, systems, device="cuda:0", steps=3, timeout_s=900):
    """The reference's own torch path (MorseModel + nvt_langevin_step, float64:
    its float32 misses the 1e-5 force bar) timed in a child process
    (baseline/ref_plain_gpu.py) on this GPU, or on the host cores with
    device="cpu"; or why it could not be."""
    import subprocess

    script = os.path.join(REPO, "baseline", "ref_plain_gpu.py")
    if not os.path.isdir(os.path.join(REPO, "baseline", "_ref", "torch_sim")):
        return {"unavailable": "reference not installed in baseline/_ref "
                               "(python baseline/install_ref.py)"}
    cmd = [sys.executable, script, "--n-systems", str(n_systems), "--systems", str(systems),
           "--steps", str(steps), "--warmup", "1", "--dtype", "float64", "--device", device]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s)
    except subprocess.TimeoutExpired:
        return {"unavailable": f"reference path did not finish in {timeout_s} s"}
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    if r.returncode != 0 or not lines:
        tail = (r.stderr or r.stdout).strip().splitlines()[-1:] or ["no output"]
        return {"unavailable": f"reference path failed (rc {r.returncode}): {tail[0][:200]}"}
    return json.loads(lines[-1])


def other_workloads(timeout_s=600):
    """The other workloads' bench lines (configs 2, 4 and 5), each run by this
    script in a child process before the main measurement, so that one default
    run records all of them."""
    import subprocess

    out = {}
    for w in ("single_large", "relax", "adjoint"):
        cmd = [sys.executable, os.path.abspath(__file__), "--workload", w]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s)
        except subprocess.TimeoutExpired:
            out[w] = {"unavailable": f"did not finish in {timeout_s} s"}
            continue
        lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
        if r.returncode != 0 or not lines:
            tail = (r.stderr or r.stdout).strip().splitlines()[-1:] or ["no output"]
            out[w] = {"unavailable": f"rc {r.returncode}: {tail[0][:200]}"}
            continue
        d = json.loads(lines[-1])
        out[w] = {k: d[k] for k in ("metric", "value", "unit", "ms_per_step", "steps", "config",
                                    "roofline", "force_err_vs_fp64", "clocks") if k in d}
    return out


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, REPO)
    from oracle import cpu_md
    from tsb import workloads as W

    import numpy as np

    d = W.copper_batch(args.n_systems, 8, 512, seed=0)
    procs = cpu_md.cpu_count()
    n_sys = args.n_systems
    rng = np.random.default_rng(0)
    perm = rng.permutation(n_sys)
    dt, kT, g = 0.002 * W.METAL_TIME, 1000 * W.KB_EV, 10.0 / W.METAL_TIME
    per = 2 * procs  # systems per step: a bounded sample of the workload
    times, work = [], []
    for k in range(args.warmup + args.steps):
        systems = perm[(k * per) % n_sys:][:per]
        a, t = cpu_md.time_sample(d, systems, 1, dt, kT, g, 6.0, procs)
        if k >= args.warmup:
            times.append(t)
            work.append(a)
    value = sum(work) / sum(times)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "n_systems": n_sys,
                       "sample_systems_per_step": per, "md_steps_per_step": 1},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                             "sample": f"{per} systems x 1 BAOAB step per bench step, "
                                       "numpy oracle of the reference path"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_single_large(args):
    """500,000-atom LJ argon (fp32 positions), NVE at 50 K with a reused Verlet list
    (cutoff 8.5 A + skin 1.0 A, rebuilt when an atom moved > 0.5 A): one bench step
    = --md-steps force evaluations."""
    import torch

    from tsb import integrators, models, workloads
    from tsb.state import state_from_arrays

    dev = torch.device("cuda", 0)
    d = workloads.argon_fcc((50, 50, 50), jitter=0.1, seed=0)
    st = state_from_arrays(d, device=dev, dtype=torch.float32)
    st.rng = 7
    base = models.LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=8.5,
                                    dtype=torch.float32, compute_stress=True, device=dev)
    vm = models.VerletListModel(base, skin=1.0)
    md = integrators.nve_init(st, vm, kT=50.0 * workloads.KB_EV)
    dt = 0.002 * workloads.METAL_TIME
    n_steps = args.md_steps
    for _ in range(args.warmup):
        for _ in range(n_steps):
            md = integrators.nve_step(md, vm, dt=dt)
    torch.cuda.synchronize()
    builds0 = vm.n_builds
    stream = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(0) as clocks:
        for k in range(args.steps):
            ev[k][0].record(stream)
            for _ in range(n_steps):
                md = integrators.nve_step(md, vm, dt=dt)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    t = sum(a.elapsed_time(b) for a, b in ev) / 1e3
    evals = n_steps * args.steps
    n = md.n_atoms
    entries = int(vm.list_counts.sum())
    # algorithmic bytes per evaluation: list (4 B/entry) + build-frame positions
    # (32 B) + forces (12 B) + per-atom energy/virial scratch (56 B)
    alg = 4 * entries + n * (32 + 12 + 56)
    peak, kind = measured_peak_hbm()
    achieved = alg * evals / t / 1e9
    # FP32 list forces of the final configuration vs an FP64 evaluation of it
    f32 = vm(md)["forces"].double()
    ref = models.LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=8.5, precision="fp64",
                                   dtype=torch.float64, device=dev)(md.to(dtype=torch.float64))
    df = (f32 - ref["forces"]).abs()
    force_err = {"max_abs_over_max_abs": float(df.max() / ref["forces"].abs().max()),
                 "rms_rel": float(df.pow(2).mean().sqrt() / ref["forces"].pow(2).mean().sqrt())}
    line = {"metric": "force evaluations x atoms / s (single 500k-atom system, Verlet list)",
            "value": n * evals / t, "unit": "atom-evals/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (LJ argon fcc 50x50x50, N(0,0.1 A) jitter)",
            "config": {"workload": "single_large", "atoms": n,
                       "force_evals": evals, "list_builds": vm.n_builds - builds0,
                       "mean_list_entries_per_atom": entries / n, "cutoff_A": 8.5,
                       "skin_A": 1.0, "integrator": "NVE 50 K, dt 2 fs"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_source": kind,
                         "kernel": "k_verlet_forces (+ integrator kernels)"},
            "force_err_vs_fp64": force_err,
            "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)
    return 0


def run_relax(args):
    """1024 Kob-Andersen boxes (64-1000 atoms), FIRE (ASE) + Frechet cell filter until
    max|F| < 1e-3 eV/A and cell-force rows < 1e-3; converged systems frozen on the
    device.  Timed once (the whole relaxation)."""
    import torch

    from tsb import models, optimizers, workloads
    from tsb.state import state_from_arrays

    dev = torch.device("cuda", 0)
    d = workloads.kob_andersen_batch(args.n_systems if args.n_systems != 2048 else 1024,
                                     64, 1000, seed=0)
    st = state_from_arrays(d, device=dev)
    m = models.kob_andersen_model(compute_stress=True, device=dev)
    if args.list_skin > 0:
        m = models.VerletListModel(m, skin=args.list_skin, prune=args.list_prune)
    st = optimizers.fire_init(st, m, cell_filter="frechet")
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clocks:
        a.record()
        st, steps, conv = optimizers.optimize(st, m, fmax=1e-3, max_steps=args.md_steps * 20,
                                              cell_filter="frechet", check_every=50,
                                              graph_steps=args.graph_steps)
        b.record()
        torch.cuda.synchronize()
    t = a.elapsed_time(b) / 1e3
    n = st.n_atoms
    # forces of the relaxed states: FP32 pair math vs FP64, against the fmax criterion
    ref = models.kob_andersen_model(compute_stress=True, device=dev, precision="fp64")(st)
    err = float((m(st)["forces"] - ref["forces"]).abs().max())
    line = {"metric": "FIRE+Frechet relaxation: atom-steps/s (all systems, until converged)",
            "value": n * steps / t, "unit": "atom-steps/s", "n_gpus": 1, "steps": steps,
            "warmup": 0, "ms_per_step": 1e3 * t / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair / f64 state",
            "data": "synthetic (Kob-Andersen 80:20, rho = 1.2 sigma^-3, uniform random)",
            "config": {"workload": "relax", "systems": st.n_systems, "atoms": n,
                       "fire_steps": steps, "converged": int(conv.sum()),
                       "graph_steps_per_replay": args.graph_steps,
                       "time_to_all_converged_s": t, "fmax": 1e-3,
                       "neighbour_lists": (
                           f"Verlet, skin {args.list_skin} A, "
                           + (f"pruned to cutoff + {m.prune:.3g} A, "
                              if getattr(m, "prune", 0.0) > 0 else "not pruned, ")
                           + "expired systems rebuilt "
                           + ("on the device inside the graph (not counted on the host)"
                              if args.graph_steps > 0
                              else f"by host decision ({m.n_builds} builds)")
                           if args.list_skin > 0 else "cell-list search per call")},
            "force_err_vs_fp64": {"max_abs_eV_per_A": err, "over_fmax": err / 1e-3},
            "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)
    return 0


def run_adjoint(args):
    """256 two-species LJ systems of 108 atoms, 200 NVE steps (2 fs) from 80 K;
    loss = squared error of the final-frame smeared pair-distance histogram;
    one bench step = loss + adjoint gradients (sigma, epsilon, q0, p0), 20-step
    checkpoints."""
    import torch

    from tsb import adjoint, integrators, workloads
    from tsb.state import state_from_arrays

    dev = torch.device("cuda", 0)
    d = workloads.argon_species_batch(256, (3, 3, 3), seed=0)
    st = state_from_arrays(d, device=dev)
    g = torch.Generator(device=dev).manual_seed(5)
    p0 = integrators.initialize_momenta(st.positions, st.masses, st.system_idx,
                                        torch.tensor(80.0 * workloads.KB_EV, device=dev), g)
    P = adjoint.make_problem(st, 200, 0.002 * workloads.METAL_TIME)
    s0, e0 = adjoint.argon_pair_params(device=dev)
    qT, _, _ = adjoint.integrate(st.positions, p0, adjoint.lj_table(s0, e0), P, False)
    P.target = adjoint.histogram(qT, P)
    s, e = adjoint.argon_pair_params(perturb=0.05, seed=1, device=dev)
    for _ in range(max(1, args.warmup)):
        adjoint.loss_and_grad(s, e, st.positions, p0, P)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(0) as clocks:
        for a, b in evs:
            a.record()
            loss, gs, ge, gq, gp = adjoint.loss_and_grad(s, e, st.positions, p0, P)
            b.record()
        torch.cuda.synchronize()
    t = sum(a.elapsed_time(b) for a, b in evs) / 1e3 / args.steps
    n = st.n_atoms
    line = {"metric": "gradient evaluations/s (200-step NVE trajectory loss, adjoint)",
            "value": 1.0 / t, "unit": "grad-evals/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (256 x fcc 3x3x3 argon, two species 50:50)",
            "config": {"workload": "adjoint", "systems": 256, "atoms": n, "md_steps": 200,
                       "checkpoint_every": 20, "atom_steps_per_s_incl_adjoint": n * 200 / t,
                       "loss": float(loss)},
            "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.workload == "adjoint" and args.impl != "reference":
        return run_adjoint(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "single_large":
        return run_single_large(args)
    if args.workload == "relax":
        return run_relax(args)
    import torch

    ws, rank, local = dist_env()
    # the other workloads run first, in child processes, before this process
    # holds a CUDA context (their launch-bound loops run slower beside one)
    others = None
    if (not args.no_other_workloads and ws == 1 and args.integrator == "nvt_langevin"
            and args.n_systems == 2048):
        others = other_workloads()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = torch.device("cuda", local if ws > 1 else 0)
    torch.cuda.set_device(device)
    from tsb import integrators

    d, md, model = build_workload(args.n_systems, seed=rank, device=device)
    n_atoms = md.n_atoms
    from tsb import workloads as W

    dt_md, kT_md = 0.002 * W.METAL_TIME, 1000 * W.KB_EV
    if args.integrator == "nvt_nose_hoover":
        md = integrators.nvt_nose_hoover_init(md, model, kT=kT_md, dt=dt_md)
    runner = integrators.FusedMD(md, model, integrator=args.integrator,
                                 dt=dt_md, kT=kT_md if args.integrator != "nve" else None,
                                 gamma=10.0 / W.METAL_TIME if args.integrator == "nvt_langevin"
                                 else None,
                                 skin=args.skin if args.skin == "auto" else float(args.skin),
                                 seed=1234 + rank,
                                 prune=(None if args.prune is None else
                                        args.prune if args.prune == "auto" else
                                        float(args.prune)),
                                 lanes=(None if args.lanes is None else
                                        args.lanes if args.lanes == "auto" else
                                        int(args.lanes)))
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    for _ in range(args.warmup):
        runner.launch(args.md_steps)
    torch.cuda.synchronize(device)
    runner.check()

    from tsb import replicas

    barrier = replicas.barrier

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize(device)
    with ClockSampler(device.index) as clocks:
        for k in range(args.steps):
            flush.fill_(float(k))  # 256 MB write: evicts L2 between timed launches
            starts[k].record(stream)
            runner.launch(args.md_steps)
            ends[k].record(stream)
        torch.cuda.synchronize(device)
    barrier()
    runner.check()
    rebuilds = runner.rebuilds.double()
    rebuild_interval = args.md_steps / max(float(rebuilds.mean()), 1e-9)
    per_launch_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    t_rank = sum(per_launch_ms) / 1e3
    t_max = replicas.max_over_ranks(t_rank, device)
    value = replicas.weak_scaling_value(n_atoms * args.md_steps * args.steps, t_max, ws)
    avg_launch_s = statistics.mean(per_launch_ms) / 1e3

    # ---- end to end through the C ABI with host buffers (pinned), copies timed;
    # every e2e step starts from the state reached after the timed launches (a
    # hot, equilibrating trajectory like the timed ones, not the initial lattice)
    f64 = torch.float64
    hx = runner.x.cpu().pin_memory()
    hp = runner.p.cpu().pin_memory()
    hf = runner.f.cpu().pin_memory()
    ox = torch.empty_like(hx).pin_memory()
    op = torch.empty_like(hp).pin_memory()
    oe = torch.empty(md.n_systems, dtype=f64).pin_memory()
    e2e_steps = max(2, min(args.steps, 5))
    es = [torch.cuda.Event(enable_timing=True) for _ in range(e2e_steps)]
    ee = [torch.cuda.Event(enable_timing=True) for _ in range(e2e_steps)]
    barrier()
    torch.cuda.synchronize(device)
    for k in range(e2e_steps):
        flush.fill_(float(k))
        es[k].record(stream)
        runner.x.copy_(hx, non_blocking=True)
        runner.p.copy_(hp, non_blocking=True)
        runner.f.copy_(hf, non_blocking=True)
        runner.launch(args.md_steps)
        ox.copy_(runner.x, non_blocking=True)
        op.copy_(runner.p, non_blocking=True)
        oe.copy_(runner.energy, non_blocking=True)
        ee[k].record(stream)
    torch.cuda.synchronize(device)
    barrier()
    runner.check()
    te = replicas.max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(es, ee)) / 1e3, device)
    e2e_value = replicas.weak_scaling_value(n_atoms * args.md_steps * e2e_steps, te, ws)
    h2d = 3 * hx.numel() * 8
    d2h = 2 * hx.numel() * 8 + oe.numel() * 8

    # force error of the fused kernel's FP32 pair arithmetic vs an FP64 evaluation
    # of the same final configuration (the metric's "force err <= 1e-5 vs FP64")
    from tsb import models as _models

    md.positions, md.forces = runner.x, runner.f
    ref64 = _models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                               precision="fp64", device=device)(md)["forces"]
    df = (runner.f - ref64).abs()
    force_err = {"max_abs_over_max_abs": float(df.max() / ref64.abs().max()),
                 "rms_rel": float(df.pow(2).mean().sqrt() / ref64.pow(2).mean().sqrt())}

    # the plain per-call GPU path on the same systems: one nvt_langevin_step per MD
    # step (cell list rebuilt, pair forces, BAOAB kernels, launched from Python)
    ps = md.clone()
    ps.momenta = runner.p.clone()
    if args.integrator == "nvt_langevin":
        def plain_step(st):
            return integrators.nvt_langevin_step(st, model, dt=dt_md, kT=kT_md,
                                                 gamma=10.0 / W.METAL_TIME)
    elif args.integrator == "nvt_nose_hoover":
        def plain_step(st):
            return integrators.nvt_nose_hoover_step(st, model, dt=dt_md, kT=kT_md)
    elif args.integrator == "nvt_vrescale":
        def plain_step(st):
            return integrators.nvt_vrescale_step(model, st, dt=dt_md, kT=kT_md)
    else:
        def plain_step(st):
            return integrators.nve_step(st, model, dt=dt_md)
    for _ in range(3):
        ps = plain_step(ps)
    pa, pb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize(device)
    pa.record(stream)
    for _ in range(args.plain_steps):
        ps = plain_step(ps)
    pb.record(stream)
    torch.cuda.synchronize(device)
    t_plain = replicas.max_over_ranks(pa.elapsed_time(pb) / 1e3, device)
    plain_value = replicas.weak_scaling_value(n_atoms * args.plain_steps, t_plain, ws)

    # pair counts of the final configuration: algorithmic half pairs within the
    # cutoff, the list entries each atom holds, and those it evaluates per fused
    # step (within cutoff + pruning skin, when the shell is pruned)
    half_pairs, evals = pair_counts(runner.x, runner.cell_row, md.system_idx, model.cutoff,
                                    runner.skin, md.n_systems)
    evaluated = evals
    if 0.0 < runner.prune < runner.skin:
        evaluated = pair_counts(runner.x, runner.cell_row, md.system_idx, model.cutoff,
                                runner.prune, md.n_systems)[1]

    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        fp32_peak, sfu_peak = sm_peaks(device)
        alg_bytes = n_atoms * args.md_steps * ALG_BYTES_PER_ATOM_STEP
        achieved = alg_bytes / avg_launch_s / 1e9
        # per-launch rate of the dominant kernel (CUDA events around each launch)
        rate = n_atoms * args.md_steps / avg_launch_s
        fp32_achieved = rate * half_pairs * FLOPS_PER_PAIR / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Cu supercells)",
            "config": {"workload": WORKLOAD if args.integrator == "nvt_langevin" else
                       WORKLOAD.replace("NVT-Langevin BAOAB", INTEGRATOR_NAMES[args.integrator]),
                       "n_systems": args.n_systems,
                       "atoms_per_gpu": n_atoms, "md_steps_per_step": args.md_steps,
                       "verlet_skin_A": runner.skin, "prune_skin_A": runner.prune,
                       "lanes_per_atom_max": runner.lanes,
                       "skin_source": "autotuner" if args.skin == "auto" else "argument",
                       "precision": "FP32 pair math, FP64 state",
                       "mean_steps_between_list_rebuilds": rebuild_interval,
                       "l2": "256 MB buffer written between timed launches",
                       "parallelism": f"replicas x{ws} (independent systems per rank)"},
            # the binding bound of this shared-memory-resident kernel is FP32 and
            # MUFU issue inside the SM: algorithmic flops = half pairs within the
            # cutoff x 45 FP32 flops; one exp per half pair
            "roofline": {"bound": "fp32", "kernel": "k_fused_md", "achieved": fp32_achieved,
                         "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": fp32_achieved / fp32_peak, "traffic": None,
                         "peak_source": "nominal: SMs x 128 FP32 lanes x 2 x max SM clock "
                                        "(no measured FP32 peak)",
                         "half_pairs_per_atom_step": half_pairs,
                         # full-list entries within cutoff + skin (each atom holds its
                         # own list; systems whose shared-memory tables overflow at this
                         # skin run at a halved one, with fewer), and the entries it
                         # evaluates per step: those within cutoff + pruning skin
                         "list_entries_per_atom_at_skin": evals,
                         "list_entries_per_atom_evaluated": evaluated,
                         "flops_per_half_pair": FLOPS_PER_PAIR,
                         "exp_per_s": rate * half_pairs,
                         "sfu_peak_per_s": sfu_peak * 1e9,
                         "sfu_frac": rate * half_pairs / (sfu_peak * 1e9)},
            # the streaming-design HBM bound, for comparison: this kernel keeps the
            # per-step state in shared memory and registers
            "roofline_hbm": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                             "algorithmic_bytes_per_atom_step": ALG_BYTES_PER_ATOM_STEP,
                             "kernel": "k_fused_md"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "force_err_vs_fp64": force_err,
            "plain_path": {"value": plain_value, "unit": UNIT, "md_steps": args.plain_steps,
                           "what": f"tsb.integrators step function ({args.integrator}) per MD "
                                   "step (cell list + FP32 pair forces + integrator kernels "
                                   "each call)",
                           "fused_over_plain": value / plain_value},
            # k_bounds_fused, k_fused_md (one launch per block shape), k_advance_counter
            "gpu_launches": (3 + (0 < runner.n_wide < md.n_systems)) * args.steps,
            "clocks": clocks.summary(),
            "per_launch_ms": per_launch_ms,
        }
        if args.ref_plain_systems > 0 and ws == 1 and args.integrator == "nvt_langevin":
            # the metric's plain GPU path as the reference itself runs it
            ref = reference_plain_path(args.n_systems, args.ref_plain_systems,
                                       f"cuda:{device.index or 0}")
            if "value" in ref:
                ref["fused_over_reference_plain"] = value / ref["value"]
            line["plain_path_reference"] = ref
        if others is not None:
            line["other_workloads"] = others
        if not args.no_cpu_baseline and ws == 1:
            line["cpu_baseline"] = cpu_baseline(d)
            if args.integrator == "nvt_langevin":
                # the reference's own torch path on the host cores (a random
                # sample of the systems; reported baseline only)
                cref = reference_plain_path(args.n_systems, 64, "cpu", steps=2)
                if "value" in cref:
                    cref = {"value": cref["value"], "unit": UNIT, "cores": cref["threads"],
                            "kind": "reference",
                            "sample": f"{cref['systems']} of {cref['of_systems']} systems "
                                      f"({cref['atoms']} atoms) x {cref['md_steps']} steps, "
                                      "float64, torch threads = host cores",
                            "what": cref["what"]}
                line["cpu_reference"] = cref
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
