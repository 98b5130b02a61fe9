"""Autotuner host logic (CPU): cache file, workload key, sampling, selection,
and the system subset used for tuning."""

import json

import pytest
import torch


def _md_cpu(n_sys=6, seed=0):
    from tsb import workloads
    from tsb.state import MDState, state_from_arrays

    d = workloads.copper_batch(n_sys, 8, 64, seed=seed)
    st = state_from_arrays(d, device="cpu")
    n, s = st.n_atoms, st.n_systems
    return MDState.from_state(st, momenta=torch.randn(n, 3, dtype=torch.float64),
                              forces=torch.randn(n, 3, dtype=torch.float64),
                              energy=torch.arange(s, dtype=torch.float64))


def test_select_systems_masks_atoms_and_renumbers():
    from tsb.state import select_systems

    md = _md_cpu()
    sub = select_systems(md, [4, 1])
    counts = torch.bincount(md.system_idx)
    assert sub.n_systems == 2
    assert sub.n_atoms == int(counts[1] + counts[4])
    assert torch.equal(sub.system_idx, torch.repeat_interleave(
        torch.arange(2), torch.stack([counts[1], counts[4]])))
    assert torch.equal(sub.cell, md.cell[[1, 4]])
    assert torch.equal(sub.energy, md.energy[[1, 4]])
    m1 = md.system_idx == 1
    assert torch.equal(sub.positions[: int(counts[1])], md.positions[m1])
    assert torch.equal(sub.momenta[: int(counts[1])], md.momenta[m1])
    with pytest.raises(IndexError):
        select_systems(md, [6])


def test_cache_roundtrip(tmp_path):
    from tsb.autotune import TuneCache

    c = TuneCache(str(tmp_path / "sub" / "t.json"))
    assert c.get("k") is None
    c.put("k", {"skin": 0.5})
    c.put("k2", {"skin": 0.7})
    assert c.get("k") == {"skin": 0.5}
    assert json.load(open(tmp_path / "sub" / "t.json"))["k2"]["skin"] == 0.7
    (tmp_path / "bad.json").write_text("not json")
    assert TuneCache(str(tmp_path / "bad.json")).get("k") is None


def test_selection_and_sampling():
    from tsb.autotune import select_best, spread_sample

    assert select_best({0.3: 2.0, 0.5: 1.0, 0.7: 1.0}) == 0.5
    assert spread_sample(10, 20) == list(range(10))
    s = spread_sample(2048, 296)
    assert len(s) == 296 and s[0] == 0 and s[-1] < 2048 and s == sorted(set(s))


def test_signature_separates_workloads():
    from tsb import models
    from tsb.autotune import fused_signature

    md = _md_cpu()
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0, device="cpu")
    a = fused_signature(md, m, "nvt_langevin", 0.2, 0.086, "dev")
    assert a == fused_signature(md, m, "nvt_langevin", 0.2, 0.0861, "dev")  # 2 digits
    assert a != fused_signature(md, m, "nvt_langevin", 0.2, 0.05, "dev")
    assert a != fused_signature(md, m, "nve", 0.2, None, "dev")


def test_cached_skin_is_returned_without_running(tmp_path):
    from tsb import autotune, models

    md = _md_cpu()
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0, device="cpu")
    cache = autotune.TuneCache(str(tmp_path / "t.json"))
    key = "fused_skin|" + autotune.fused_signature(md, m, "nve", 0.2, None, "cpu")
    cache.put(key, {"skin": 0.5})

    def boom(*_a):
        raise AssertionError("must not time anything")

    assert autotune.tune_fused_skin(md, m, integrator="nve", dt=0.2, cache=cache,
                                    timer=boom) == 0.5


def test_cached_prune_is_returned_without_running(tmp_path):
    """The pruning skin is cached per (skin, workload) like the skin; candidates are
    fractions of the skin, so a cached value outside them is ignored."""
    from tsb import autotune, models

    md = _md_cpu()
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0, device="cpu")
    cache = autotune.TuneCache(str(tmp_path / "t.json"))
    key = ("fused_prune|skin" + autotune._sig(1.2, 3) + "|" +
           autotune.fused_signature(md, m, "nve", 0.2, None, "cpu"))
    cache.put(key, {"prune": 0.3})

    def boom(*_a):
        raise AssertionError("must not time anything")

    assert autotune.tune_fused_prune(md, m, skin=1.2, integrator="nve", dt=0.2, cache=cache,
                                     timer=boom) == 0.3
    cache.put(key, {"prune": 0.31})  # not a candidate fraction of 1.2: would be re-tuned
    assert 0.31 not in sorted({round(f * 1.2, 6) for f in autotune.DEFAULT_PRUNE_FRACTIONS})
