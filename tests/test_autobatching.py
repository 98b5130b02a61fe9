"""The admission policy (tsb.autobatching) against the reference's own bins and
memory scalers (tests/golden/autobatch.npz, made by make_autobatch.py from
torch_sim/autobatching.py:46-144, 305-420)."""

import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN


@pytest.fixture(scope="module")
def ab():
    return np.load(os.path.join(GOLDEN, "autobatch.npz"))


@pytest.mark.parametrize("k", range(6))
def test_bins_match_reference(ab, k):
    from tsb.autobatching import to_constant_volume_bins

    w = ab[f"case{k}/weights"]
    cap = float(ab[f"case{k}/max_volume"])
    bins = to_constant_volume_bins(dict(enumerate(w.tolist())), cap)
    bid = np.full(len(w), -1)
    for b, d in enumerate(bins):
        assert sum(d.values()) <= cap + 1e-12
        for key in d:
            bid[key] = b
    assert np.array_equal(bid, ab[f"case{k}/bin_of_item"])
    lst = to_constant_volume_bins(w.tolist(), cap)
    np.testing.assert_allclose([sum(b) for b in lst], ab[f"case{k}/list_bin_sums"])


def test_bin_options():
    from tsb.autobatching import to_constant_volume_bins

    items = [("a", 3.0), ("b", 5.0), ("c", 1.0), ("d", 4.0)]
    bins = to_constant_volume_bins(items, 6.0, weight_pos=1)
    assert bins == [[("b", 5.0), ("c", 1.0)], [("d", 4.0)], [("a", 3.0)]] or \
        sorted(sum(x[1] for x in b) for b in bins) == [3.0, 4.0, 6.0]
    assert to_constant_volume_bins(items, 6.0, key=lambda x: x[1], lower_bound=1.0,
                                   upper_bound=5.0) == [[("d", 4.0)], [("a", 3.0)]]
    with pytest.raises(ValueError):
        to_constant_volume_bins(items, 6.0)
    with pytest.raises(ValueError):
        to_constant_volume_bins([1.0], 6.0, lower_bound=2.0, upper_bound=1.0)
    assert to_constant_volume_bins([], 1.0) == []


def test_memory_scalers_match_reference(ab):
    from tsb import workloads
    from tsb.autobatching import calculate_memory_scalers
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(12, 8, 512, seed=3)
    st = state_from_arrays(d, device="cpu")
    np.testing.assert_allclose(calculate_memory_scalers(st, "n_atoms_x_density"),
                               ab["cu/scalers_density"], rtol=1e-12)
    np.testing.assert_allclose(calculate_memory_scalers(st, "n_atoms"), ab["cu/scalers_atoms"])


def test_binning_batcher_round_trip():
    from tsb import workloads
    from tsb.autobatching import BinningAutoBatcher, calculate_memory_scalers
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(10, 8, 300, seed=9)
    st = state_from_arrays(d, device="cpu")
    cap = 2.5 * max(calculate_memory_scalers(st))
    bat = BinningAutoBatcher(max_memory_scaler=cap)
    bat.load_states(st)
    seen = []
    for sub, idx in bat:
        assert sub.n_systems == len(idx)
        seen.append(idx)
        sc = calculate_memory_scalers(sub)
        assert sum(sc) <= cap + 1e-9
    flat = sorted(i for b in seen for i in b)
    assert flat == list(range(10))
    res = bat.restore_original_order([i for b in seen for i in b])
    assert res == list(range(10))
    with pytest.raises(ValueError):
        BinningAutoBatcher()
