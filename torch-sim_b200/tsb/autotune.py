"""Project-written autotuner for launch parameters that depend on the workload.

The persistent fused MD kernel has three tunable parameters: the Verlet skin
and the pruning skin of the list's shell (physics), and the launch shape of
small systems, i.e. how many threads share
one atom's neighbour list (``lanes``: 4, 8, 16 or 32 at most; more lanes split
each list finer, but every lane repeats the atom's integration step).  First
the skin.  A wider skin puts
more pairs in the list (more pair evaluations every step); a narrower one makes
atoms leave it sooner (more list rebuilds).  Where the balance lies depends on
temperature, density, cutoff, time step and system sizes, so
:func:`tune_fused_skin` times candidate skins on a sample of the batch's own
systems and keeps the fastest, cached per device and workload signature in a
JSON file (``TSB_AUTOTUNE_CACHE``, default ``~/.cache/tsb/autotune.json``).
Results do not depend on the skin (only the rebuild rate does), so any choice
is safe.  Skins are timed with the shell pruned at a fixed fraction of the
skin; then, at the chosen skin, :func:`tune_fused_prune` times pruning skins
(0 = every list pair evaluated every step; a narrower pruning skin evaluates
fewer pairs but prunes the shell more often), and :func:`tune_fused_lanes` the
lane caps, the same way.  ``FusedMD(..., skin="auto")`` and
``run_md(..., skin="auto")`` use all three.
"""

from __future__ import annotations

import json
import math
import os
import tempfile
import threading

import torch

DEFAULT_SKINS = (0.5, 0.7, 1.0, 1.2, 1.4)
DEFAULT_LANES = (4, 8, 16, 32)
DEFAULT_PRUNE_FRACTIONS = (0.0, 0.25, 0.375, 0.5)


def cache_path() -> str:
    return os.environ.get("TSB_AUTOTUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "tsb", "autotune.json")


class TuneCache:
    """JSON file of ``{key: record}``; writes replace the file atomically."""

    _lock = threading.Lock()

    def __init__(self, path: str | None = None):
        self.path = path or cache_path()

    def load(self) -> dict:
        try:
            with open(self.path) as fh:
                d = json.load(fh)
            return d if isinstance(d, dict) else {}
        except (OSError, ValueError):
            return {}

    def get(self, key: str):
        return self.load().get(key)

    def put(self, key: str, record: dict) -> None:
        with self._lock:
            d = self.load()
            d[key] = record
            os.makedirs(os.path.dirname(os.path.abspath(self.path)), exist_ok=True)
            fd, tmp = tempfile.mkstemp(dir=os.path.dirname(os.path.abspath(self.path)),
                                       suffix=".tmp")
            with os.fdopen(fd, "w") as fh:
                json.dump(d, fh, indent=1, sort_keys=True)
            os.replace(tmp, self.path)


def _sig(x: float, digits: int = 2) -> str:
    """x to `digits` significant digits (stable text for cache keys)."""
    x = float(x)
    if x == 0.0 or not math.isfinite(x):
        return repr(x)
    return f"{x:.{digits - 1}e}"


def fused_signature(state, model, integrator: str, dt, kT, device_name: str) -> str:
    """Workload key: device, potential, species, cutoff, integrator, dt, kT,
    number density and the atoms-per-system scale (log2 buckets)."""
    counts = torch.bincount(state.system_idx, minlength=state.n_systems).double()
    vol = torch.linalg.det(state.cell.double()).abs().sum()
    density = float(state.n_atoms / vol)
    mean_t = lambda v: float(torch.as_tensor(v, dtype=torch.float64).mean())  # noqa: E731
    parts = [device_name, f"pot{model.kind}", f"ns{model.n_species}", _sig(model.cutoff, 4),
             integrator, "dt" + _sig(mean_t(dt)),
             "kT" + (_sig(mean_t(kT)) if kT is not None else "-"), "rho" + _sig(density),
             f"mean2^{round(math.log2(max(float(counts.mean()), 1.0)))}",
             f"max2^{round(math.log2(max(float(counts.max()), 1.0)))}",
             f"S2^{round(math.log2(max(state.n_systems, 1)))}"]
    return "|".join(parts)


def select_best(timings: dict) -> float:
    """Fastest candidate; ties go to the smaller skin (fewer pairs per step)."""
    return min(timings, key=lambda s: (timings[s], s))


def spread_sample(n_systems: int, k: int) -> list[int]:
    """k system indices spread evenly over the batch (all if k >= n_systems)."""
    if k >= n_systems:
        return list(range(n_systems))
    return sorted({int(i * n_systems / k) for i in range(k)})


def _time_launch(runner, n_steps: int) -> float:
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    runner.launch(n_steps)
    b.record()
    torch.cuda.synchronize(runner.dev)
    return a.elapsed_time(b)


def tune_fused_skin(state, model, *, integrator: str = "nvt_langevin", dt, kT=None,
                    gamma=None, candidates=DEFAULT_SKINS, n_steps: int = 200,
                    sample_systems: int | None = None, cache: TuneCache | None = None,
                    force: bool = False, timer=_time_launch) -> float:
    """Verlet skin for ``FusedMD`` on this workload (cached; see module doc).

    Each candidate runs the fused kernel on a sample of the batch (sixteen
    systems per SM by default, spread over the batch: the whole batch up to
    2,368 systems on a B200; with only a few systems per SM the launch time is
    that of the SMs holding the largest systems and the ranking is noisy) from
    the same starting point:
    ``n_steps`` steps of warm-up (the atoms leave their starting positions and
    the list rebuild rate settles), then ``n_steps`` timed steps.
    """
    from .integrators import FusedMD

    cache = cache or TuneCache()
    dev = state.device
    name = torch.cuda.get_device_name(dev) if dev.type == "cuda" else str(dev)
    key = "fused_skin|" + fused_signature(state, model, integrator, dt, kT, name)
    if not force:
        rec = cache.get(key)
        if rec is not None and float(rec.get("skin", -1)) in [float(c) for c in candidates]:
            return float(rec["skin"])
    from .state import select_systems

    if sample_systems is None:
        n_sm = (torch.cuda.get_device_properties(dev).multi_processor_count
                if dev.type == "cuda" else 1)
        sample_systems = 16 * n_sm
    idx = spread_sample(state.n_systems, sample_systems)
    sample = select_systems(state, idx) if len(idx) < state.n_systems else state

    def per_sys(v):
        if v is None or not torch.is_tensor(v) or v.ndim == 0:
            return v
        return v.to(dev)[torch.as_tensor(idx, device=dev)]

    timings = {}
    for skin in candidates:
        r = FusedMD(sample.clone(), model, integrator=integrator, dt=per_sys(dt),
                    kT=per_sys(kT), gamma=per_sys(gamma), skin=float(skin), seed=0,
                    prune=None)
        r.launch(n_steps)
        timings[float(skin)] = float(timer(r, n_steps))
        r.check()
    best = select_best(timings)
    cache.put(key, {"skin": best, "timings_ms": {str(k): v for k, v in timings.items()},
                    "n_steps": n_steps, "sample_systems": len(idx)})
    return best


def _sample(state, sample_systems):
    from .state import select_systems

    dev = state.device
    if sample_systems is None:
        n_sm = (torch.cuda.get_device_properties(dev).multi_processor_count
                if dev.type == "cuda" else 1)
        sample_systems = 16 * n_sm
    idx = spread_sample(state.n_systems, sample_systems)
    sample = select_systems(state, idx) if len(idx) < state.n_systems else state

    def per_sys(v):
        if v is None or not torch.is_tensor(v) or v.ndim == 0:
            return v
        return v.to(dev)[torch.as_tensor(idx, device=dev)]

    return sample, per_sys, len(idx)


def tune_fused_prune(state, model, *, skin: float, integrator: str = "nvt_langevin", dt,
                     kT=None, gamma=None, fractions=DEFAULT_PRUNE_FRACTIONS, n_steps: int = 200,
                     sample_systems: int | None = None, cache: TuneCache | None = None,
                     force: bool = False, timer=_time_launch) -> float:
    """Pruning skin (Angstrom) for ``FusedMD`` at a given skin: candidates are
    ``fractions`` of the skin, timed like :func:`tune_fused_skin` and cached under
    the same workload signature; ties go to the smaller pruning skin."""
    from .integrators import FusedMD

    cache = cache or TuneCache()
    dev = state.device
    name = torch.cuda.get_device_name(dev) if dev.type == "cuda" else str(dev)
    key = (f"fused_prune|skin{_sig(skin, 3)}|" +
           fused_signature(state, model, integrator, dt, kT, name))
    candidates = sorted({round(float(f) * float(skin), 6) for f in fractions})
    if not force:
        rec = cache.get(key)
        if rec is not None and float(rec.get("prune", -1)) in candidates:
            return float(rec["prune"])
    sample, per_sys, n_sample = _sample(state, sample_systems)
    timings = {}
    for prune in candidates:
        r = FusedMD(sample.clone(), model, integrator=integrator, dt=per_sys(dt),
                    kT=per_sys(kT), gamma=per_sys(gamma), skin=float(skin), seed=0,
                    prune=float(prune))
        r.launch(n_steps)
        timings[float(prune)] = float(timer(r, n_steps))
        r.check()
    best = select_best(timings)
    cache.put(key, {"prune": best, "timings_ms": {str(k): v for k, v in timings.items()},
                    "n_steps": n_steps, "sample_systems": n_sample})
    return best


def tune_fused_lanes(state, model, *, skin: float, integrator: str = "nvt_langevin", dt,
                     kT=None, gamma=None, candidates=DEFAULT_LANES, n_steps: int = 200,
                     sample_systems: int | None = None, cache: TuneCache | None = None,
                     force: bool = False, timer=_time_launch, prune: float | None = None) -> int:
    """Lane cap (threads per atom) for ``FusedMD`` at a given skin (and pruning
    skin), timed like :func:`tune_fused_skin` and cached under the same workload
    signature; ties go to fewer lanes."""
    from .integrators import FusedMD

    cache = cache or TuneCache()
    dev = state.device
    name = torch.cuda.get_device_name(dev) if dev.type == "cuda" else str(dev)
    key = (f"fused_lanes|skin{_sig(skin, 3)}|" +
           (f"prune{_sig(prune, 3)}|" if prune is not None else "") +
           fused_signature(state, model, integrator, dt, kT, name))
    if not force:
        rec = cache.get(key)
        if rec is not None and int(rec.get("lanes", -1)) in [int(c) for c in candidates]:
            return int(rec["lanes"])
    sample, per_sys, n_sample = _sample(state, sample_systems)
    timings = {}
    for lanes in candidates:
        r = FusedMD(sample.clone(), model, integrator=integrator, dt=per_sys(dt),
                    kT=per_sys(kT), gamma=per_sys(gamma), skin=float(skin), seed=0,
                    lanes=int(lanes), prune=prune)
        r.launch(n_steps)
        timings[int(lanes)] = float(timer(r, n_steps))
        r.check()
    best = min(timings, key=lambda k: (timings[k], k))
    cache.put(key, {"lanes": best, "timings_ms": {str(k): v for k, v in timings.items()},
                    "n_steps": n_steps, "sample_systems": n_sample})
    return best
