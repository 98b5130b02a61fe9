"""GPU neighbour list vs the reference's pair sets (bit-exact) and the oracle."""

import os

import numpy as np
import pytest
import torch

from oracle import neighbors as onl

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

NL_CASES = ["ar_fcc444", "cu_tri_batch", "slab_pbc_TTF", "cluster_nopbc",
            "tiny_self_images", "rhombohedral_unwrapped"]


def _run(c, self_interaction=False, dtype=torch.float64, half=False):
    from tsb import neighbors

    dev = torch.device("cuda")
    pos = torch.as_tensor(c["positions"], dtype=dtype, device=dev)
    cell = torch.as_tensor(c["cell_row"], dtype=dtype, device=dev)
    pbc = torch.as_tensor(c["pbc"], dtype=torch.bool, device=dev)
    sysi = torch.as_tensor(c["system_idx"], dtype=torch.int64, device=dev)
    m, sm, sh = neighbors.torchsim_nl(pos, cell, pbc, float(c["cutoff"]), sysi,
                                      self_interaction, half=half)
    assert m.dtype == torch.int64 and sm.dtype == torch.int64 and sh.dtype == dtype
    return m.cpu().numpy(), sm.cpu().numpy(), sh.cpu().numpy()


@pytest.mark.parametrize("case", NL_CASES)
@pytest.mark.parametrize("self_interaction", [False, True])
def test_nl_matches_reference_pair_set(golden, case, self_interaction):
    g = golden["nl"]
    c = g[case]
    key = case + ("_self" if self_interaction else "")
    ref = onl.sort_pairs(g[key]["mapping"], g[key]["system_mapping"], g[key]["shifts"])
    got = onl.sort_pairs(*_run(c, self_interaction))
    assert got[0].shape == ref[0].shape
    np.testing.assert_array_equal(got[0], ref[0])
    np.testing.assert_array_equal(got[1], ref[1])
    np.testing.assert_array_equal(np.rint(got[2]).astype(int), ref[2].astype(int))
    # shifts are exact integers stored as floats
    assert np.all(got[2] == np.rint(got[2]))


@pytest.mark.parametrize("case", NL_CASES)
def test_nl_half_list_matches_full_to_half(golden, case):
    c = golden["nl"][case]
    full = _run(c)
    ref = onl.sort_pairs(*onl.full_to_half_list(*full))
    got = onl.sort_pairs(*_run(c, half=True))
    np.testing.assert_array_equal(got[0], ref[0])
    np.testing.assert_array_equal(got[2], ref[2])


def test_nl_float32_positions(golden):
    c = golden["nl"]["cu_tri_batch"]
    got = onl.sort_pairs(*_run(c, dtype=torch.float32))
    ref = onl.neighbor_list(c["positions"].astype(np.float32).astype(np.float64),
                            c["cell_row"].astype(np.float32).astype(np.float64), c["pbc"],
                            float(c["cutoff"]), c["system_idx"].astype(np.int64))
    np.testing.assert_array_equal(got[0], ref[0])
    np.testing.assert_array_equal(np.rint(got[2]), ref[2])


def test_nl_output_grouped_by_i_and_deterministic(golden):
    c = golden["nl"]["cu_tri_batch"]
    a = _run(c)
    b = _run(c)
    assert np.all(np.diff(a[0][0]) >= 0)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_nl_empty_and_isolated():
    from tsb import neighbors

    dev = torch.device("cuda")
    # two atoms far apart in a big non-periodic box: no pairs
    pos = torch.tensor([[0.0, 0.0, 0.0], [50.0, 0.0, 0.0]], dtype=torch.float64, device=dev)
    cell = torch.eye(3, dtype=torch.float64, device=dev) * 100
    pbc = torch.zeros(3, dtype=torch.bool, device=dev)
    sysi = torch.zeros(2, dtype=torch.int64, device=dev)
    m, sm, sh = neighbors.torchsim_nl(pos, cell, pbc, 5.0, sysi)
    assert m.shape == (2, 0) and sm.shape == (0,) and sh.shape == (0, 3)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_nl_random_triclinic_batches_vs_oracle(seed):
    from tsb import workloads

    d = workloads.copper_batch(12, 8, 300, seed=100 + seed, jitter=0.3)
    c = {"positions": d["positions"] + np.random.default_rng(seed).normal(0, 4.0, (1, 3)),
         "cell_row": np.transpose(d["cell"], (0, 2, 1)), "pbc": d["pbc"],
         "system_idx": d["system_idx"], "cutoff": 6.0 + seed}
    got = onl.sort_pairs(*_run(c))
    ref = onl.neighbor_list(c["positions"], c["cell_row"], c["pbc"], c["cutoff"],
                            c["system_idx"])
    np.testing.assert_array_equal(got[0], ref[0])
    np.testing.assert_array_equal(got[1], ref[1])
    np.testing.assert_array_equal(np.rint(got[2]), ref[2])


def test_nl_large_system_properties():
    """500k-atom-class single system at reduced size: symmetry and counts."""
    from tsb import neighbors, workloads

    d = workloads.argon_fcc((20, 20, 20), jitter=0.1, seed=5)
    dev = torch.device("cuda")
    pos = torch.as_tensor(d["positions"], dtype=torch.float32, device=dev)
    cell = torch.as_tensor(np.transpose(d["cell"], (0, 2, 1)), dtype=torch.float32,
                           device=dev)
    sysi = torch.zeros(len(pos), dtype=torch.int64, device=dev)
    m, sm, sh = neighbors.torchsim_nl(pos, cell, torch.ones(3, dtype=torch.bool, device=dev),
                                      8.5, sysi)
    n = len(pos)
    # every (i, j, S) has its mirror (j, i, -S)
    key = lambda a, b, s: ((a * n + b) * 1000 + (s[:, 0] + 5) * 100 + (s[:, 1] + 5) * 10
                           + (s[:, 2] + 5))
    si = sh.round().long()
    fwd = torch.sort(key(m[0], m[1], si)).values
    bwd = torch.sort(key(m[1], m[0], -si)).values
    assert torch.equal(fwd, bwd)
    # fcc shells within 8.5 A at a = 5.26: 12 + 6 + 24 + 12 + 24 = 78 neighbours;
    # the 0.1 A jitter moves a few across the cutoff
    assert abs(m.shape[1] / n - 78.0) < 4.0


@pytest.mark.parametrize("rc", [8.5, 9.5])
def test_nl_32k_atom_pair_set_is_exact(rc):
    """Config-2 geometry at 32,000 atoms (argon fcc 20x20x20, N(0, 0.1 A)
    jitter, slightly sheared cell): the full pair set at the cutoff and at
    cutoff + skin equals the oracle's integer-exactly (torch_nl.py:156-215)."""
    from oracle import neighbors as onl
    from tsb import neighbors, workloads

    d = workloads.argon_fcc((20, 20, 20), jitter=0.1, seed=2)
    rng = np.random.default_rng(4)
    F = np.eye(3) + rng.normal(0, 0.01, (3, 3))
    pos = d["positions"] @ F.T
    C = d["cell"][0].T @ F.T
    ref = onl.neighbor_list_cells(pos, C, rc)
    dev = torch.device("cuda")
    m, sm, sh = neighbors.torchsim_nl(torch.as_tensor(pos, device=dev),
                                      torch.as_tensor(C, device=dev),
                                      torch.ones(3, dtype=torch.bool, device=dev), rc,
                                      torch.zeros(len(pos), dtype=torch.int64, device=dev))
    got = onl.sort_pairs(m.cpu().numpy(), sm.cpu().numpy(), sh.cpu().numpy())
    assert got[0].shape == ref[0].shape, (got[0].shape, ref[0].shape)
    assert np.array_equal(got[0], ref[0])
    assert np.array_equal(np.rint(got[2]).astype(np.int64), np.rint(ref[2]).astype(np.int64))


@pytest.mark.parametrize("rc", [8.5, 9.5])
def test_nl_500k_atom_pair_set_matches_reference_digest(rc):
    """Config 2 at full size (argon fcc 50x50x50, 500,000 atoms, N(0, 0.1 A)):
    the full pair set at the cutoff and at cutoff + skin hashes to the digest of
    the reference's own torch_nl_linked_cell on the same input
    (tests/golden/nl500k.json, made by make_nl500k.py; torch_nl.py:156-215).
    Pairs are packed into int64 keys and sorted on the GPU, then hashed."""
    import hashlib
    import json

    from tsb import neighbors, workloads

    with open(os.path.join(GOLDEN, "nl500k.json")) as f:
        want = json.load(f)["cutoffs"][str(rc)]
    d = workloads.argon_fcc((50, 50, 50), jitter=0.1, seed=0)
    dev = torch.device("cuda")
    pos = torch.as_tensor(d["positions"], dtype=torch.float64, device=dev)
    cell_row = torch.as_tensor(d["cell"][0].T.copy(), dtype=torch.float64, device=dev)
    m, _, sh = neighbors.torchsim_nl(pos, cell_row, torch.ones(3, dtype=torch.bool, device=dev),
                                     rc, torch.zeros(len(pos), dtype=torch.int64, device=dev))
    assert m.shape[1] == want["n_pairs"]
    si = torch.round(sh).to(torch.int64)
    assert int(m.min()) >= 0 and int(m.max()) < (1 << 19) and int(si.abs().max()) <= 3
    key = (((m[0] << 19) | m[1]) << 9) | ((si[:, 0] + 4) << 6) | ((si[:, 1] + 4) << 3) | (
        si[:, 2] + 4)
    key = torch.sort(key).values.cpu().numpy().astype("<i8")
    assert hashlib.sha256(key.tobytes()).hexdigest() == want["sha256"]
