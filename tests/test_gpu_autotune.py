"""Autotuned Verlet skin of the fused MD kernel on the GPU: the tuner times
every candidate, picks one, caches it, and FusedMD(skin="auto") runs with it
(same trajectory physics: positions agree with a fixed-skin run to FP32
rounding)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup(n_sys=24, seed=5):
    from tsb import integrators, models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(n_sys, 8, 256, seed=seed)
    st = state_from_arrays(d, device="cuda")
    st.rng = seed
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0)
    md = integrators.nvt_langevin_init(st, m, kT=1000.0 * workloads.KB_EV)
    return md, m


def test_tuner_times_candidates_and_caches(tmp_path):
    from tsb import autotune, workloads

    md, m = _setup()
    cache = autotune.TuneCache(str(tmp_path / "t.json"))
    calls = []

    def timer(runner, n):
        calls.append(runner.skin)
        return autotune._time_launch(runner, n)

    kw = dict(integrator="nve", dt=0.002 * workloads.METAL_TIME)
    best = autotune.tune_fused_skin(md, m, candidates=(0.3, 0.7), n_steps=30,
                                    sample_systems=8, cache=cache, timer=timer, **kw)
    assert best in (0.3, 0.7) and sorted(calls) == [0.3, 0.7]
    rec = list(cache.load().values())[0]
    assert rec["skin"] == best and set(rec["timings_ms"]) == {"0.3", "0.7"}
    assert all(v > 0 for v in rec["timings_ms"].values())
    calls.clear()
    assert autotune.tune_fused_skin(md, m, candidates=(0.3, 0.7), cache=cache,
                                    timer=timer, **kw) == best
    assert calls == []  # served from the cache


def test_fused_md_with_auto_skin(tmp_path, monkeypatch):
    from tsb import integrators, workloads

    monkeypatch.setenv("TSB_AUTOTUNE_CACHE", str(tmp_path / "t.json"))
    md, m = _setup(12, seed=6)
    kw = dict(integrator="nve", dt=0.002 * workloads.METAL_TIME)
    r = integrators.FusedMD(md.clone(), m, skin="auto", **kw)
    assert r.skin in (0.5, 0.7, 1.0, 1.2, 1.4)
    r.launch(40)
    torch.cuda.synchronize()
    r.check()
    b = integrators.run_md(md.clone(), m, 40, skin=0.3, **kw)
    np.testing.assert_allclose(r.x.cpu(), b.positions.cpu(), atol=1e-5)


def test_lane_tuner_and_lane_invariance(tmp_path):
    """The lane cap is timed and cached like the skin; trajectories with 4 and 32
    lanes per atom agree to FP32 rounding (only the split of each list over
    threads, and so the summation order, changes)."""
    from tsb import autotune, integrators, workloads

    md, m = _setup(16, seed=8)
    kw = dict(integrator="nve", dt=0.002 * workloads.METAL_TIME)
    cache = autotune.TuneCache(str(tmp_path / "t.json"))
    calls = []

    def timer(runner, n):
        calls.append(runner.lanes)
        return autotune._time_launch(runner, n)

    best = autotune.tune_fused_lanes(md, m, skin=0.5, candidates=(4, 32), n_steps=30,
                                     sample_systems=8, cache=cache, timer=timer, **kw)
    assert best in (4, 32) and sorted(calls) == [4, 32]
    calls.clear()
    assert autotune.tune_fused_lanes(md, m, skin=0.5, candidates=(4, 32), cache=cache,
                                     timer=timer, **kw) == best and calls == []
    out = []
    for lanes in (4, 32):
        r = integrators.FusedMD(md.clone(), m, skin=0.5, lanes=lanes, **kw)
        r.launch(40)
        torch.cuda.synchronize()
        r.check()
        out.append((r.x.cpu().numpy(), r.energy.cpu().numpy()))
    np.testing.assert_allclose(out[0][0], out[1][0], atol=1e-5)
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=1e-5)


def test_prune_tuner_times_fractions_and_caches(tmp_path):
    """The pruning skin is timed over fractions of the skin and cached; a
    FusedMD with skin="auto" carries a pruning skin below its skin."""
    from tsb import autotune, integrators, workloads

    md, m = _setup(16, seed=9)
    kw = dict(integrator="nve", dt=0.002 * workloads.METAL_TIME)
    cache = autotune.TuneCache(str(tmp_path / "t.json"))
    calls = []

    def timer(runner, n):
        calls.append(runner.prune)
        return autotune._time_launch(runner, n)

    best = autotune.tune_fused_prune(md, m, skin=1.0, fractions=(0.0, 0.3), n_steps=30,
                                     sample_systems=8, cache=cache, timer=timer, **kw)
    assert best in (0.0, 0.3) and sorted(calls) == [0.0, 0.3]
    calls.clear()
    assert autotune.tune_fused_prune(md, m, skin=1.0, fractions=(0.0, 0.3), cache=cache,
                                     timer=timer, **kw) == best and calls == []
    r = integrators.FusedMD(md.clone(), m, skin=1.0, prune=best, **kw)
    r.launch(20)
    torch.cuda.synchronize()
    r.check()
    assert 0.0 <= r.prune < r.skin
