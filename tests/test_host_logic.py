"""Host-side logic that needs no GPU: workloads, state mirror, half-list rule."""

import numpy as np
import torch

from oracle import neighbors as onl


def test_copper_batch_shapes_and_sizes():
    from tsb import workloads

    d = workloads.copper_batch(64, 8, 512, seed=0)
    counts = np.bincount(d["system_idx"])
    assert len(counts) == 64 and counts.min() >= 4 and counts.max() <= 512
    assert np.all(counts % 4 == 0)
    assert d["cell"].shape == (64, 3, 3)
    # triclinic: off-diagonal shear present, small strain on the diagonal
    cr = np.transpose(d["cell"], (0, 2, 1))
    assert np.abs(cr[:, 0, 1]).max() > 0


def test_nearest_fcc_shape():
    from tsb import workloads

    for t in (8, 32, 100, 256, 500, 512):
        n1, n2, n3 = workloads.nearest_fcc_shape(t)
        assert abs(4 * n1 * n2 * n3 - t) <= max(4, 0.2 * t)


def test_kob_andersen_density_and_ratio():
    from tsb import workloads

    d = workloads.kob_andersen_batch(8, 64, 1000, seed=1)
    for s in range(8):
        sel = d["system_idx"] == s
        n = sel.sum()
        L = d["cell"][s, 0, 0]
        assert abs(n / L ** 3 - 1.2 / 3.4 ** 3) < 1e-9
        assert abs((d["atomic_numbers"][sel] == 2).sum() - round(0.2 * n)) == 0


def test_state_mirror_properties():
    from tsb.state import MDState, SimState

    st = SimState(positions=torch.zeros((4, 3)), masses=torch.ones(4),
                  cell=torch.eye(3) * 5, pbc=True, atomic_numbers=torch.ones(4, dtype=int),
                  system_idx=torch.tensor([0, 0, 1, 1]))
    assert st.cell.shape == (1, 3, 3) and st.pbc.tolist() == [True] * 3
    md = MDState.from_state(st, momenta=torch.ones((4, 3)), energy=torch.zeros(1),
                            forces=torch.zeros((4, 3)))
    assert torch.equal(md.velocities, torch.ones((4, 3)))
    assert torch.equal(md.row_vector_cell, st.cell.mT)


def test_torch_full_to_half_matches_oracle(golden):
    from tsb import neighbors

    g = golden["nl"]["tiny_self_images"]
    m, sm, sh = g["mapping"].astype(np.int64), g["system_mapping"].astype(np.int64), g["shifts"]
    ref = onl.sort_pairs(*onl.full_to_half_list(m, sm, sh.astype(float)))
    got = neighbors.full_to_half_list(torch.as_tensor(m), torch.as_tensor(sm),
                                      torch.as_tensor(sh.astype(float)))
    got = onl.sort_pairs(*(t.numpy() for t in got))
    np.testing.assert_array_equal(got[0], ref[0])
    np.testing.assert_array_equal(got[2], ref[2])


def test_units_match_reference_constants():
    from tsb import workloads

    assert abs(workloads.METAL_TIME - 98.22694788464062) < 1e-9
    assert abs(workloads.KB_EV - 8.617330337217213e-05) < 1e-18


def test_pbc_rows_accepts_every_reference_form():
    """SimState.pbc may be a bool, a 0-d or [3] tensor, or per-system rows."""
    import pytest
    import torch

    from tsb import _lib as L

    want = torch.tensor([[1, 0, 1]] * 4, dtype=torch.uint8)
    assert torch.equal(L.pbc_rows(torch.tensor([True, False, True]), 4, "cpu"), want)
    assert torch.equal(L.pbc_rows(want.bool(), 4, "cpu"), want)
    assert torch.equal(L.pbc_rows(want.reshape(-1), 4, "cpu"), want)
    assert torch.equal(L.pbc_rows(True, 4, "cpu"), torch.ones(4, 3, dtype=torch.uint8))
    assert torch.equal(L.pbc_rows(torch.tensor(False), 2, "cpu"),
                       torch.zeros(2, 3, dtype=torch.uint8))
    assert L.pbc_rows(True, 4, "cpu").is_contiguous()
    with pytest.raises(ValueError):
        L.pbc_rows(torch.ones(5, dtype=torch.bool), 4, "cpu")


def test_max_system_atoms_hint_is_cached_per_system_idx_version():
    from tsb import _lib as L

    sysi = torch.tensor([0, 0, 0, 1, 1, 2, 2, 2, 2], dtype=torch.int64)
    assert L.max_system_atoms(sysi, 3) == 4
    assert L.max_system_atoms(sysi, 4) == 4  # an empty trailing system
    sysi[4] = 0  # in place: a new version, a new count
    assert L.max_system_atoms(sysi, 3) == 4
    sysi[:] = 1
    assert L.max_system_atoms(sysi, 3) == 9
    assert L.max_system_atoms(torch.zeros(0, dtype=torch.int64), 1) == 0


def test_adjoint_list_width_rule():
    """Verlet lists inside the adjoint graphs need every periodic plane spacing
    >= cutoff + skin; an open axis does not count."""
    from tsb import adjoint

    class P:
        cutoff = 8.5

    c = torch.eye(3, dtype=torch.float64)
    hexa = torch.tensor([[10.0, 0, 0], [5.0, 8.66, 0], [0, 0, 10.0]], dtype=torch.float64)
    P.cell_row = torch.stack([15.78 * c, hexa])
    P.pbc = torch.ones((2, 3), dtype=torch.uint8)
    assert not adjoint._lists_fit(P, 1.0)  # the hexagonal cell's a-b planes are 8.66 A apart
    P.pbc[1, :2] = 0
    assert adjoint._lists_fit(P, 1.0)
    P.cell_row = torch.stack([15.78 * c, 15.78 * c])
    P.pbc = torch.ones((2, 3), dtype=torch.uint8)
    assert adjoint._lists_fit(P, 1.0) and not adjoint._lists_fit(P, 7.5)


def test_adjoint_overflow_retry_regrows_and_gives_up():
    from tsb import adjoint

    made = []

    class FakeGraphs:
        def __init__(self, P, table, cap=0):
            made.append(cap)

    class P:
        pass

    P = P()
    calls = {"n": 0}

    def flaky():
        calls["n"] += 1
        if calls["n"] < 3:
            raise adjoint._ListOverflow(100 * calls["n"])
        return "ok"

    orig = adjoint._Graphs
    adjoint._Graphs = FakeGraphs
    try:
        assert adjoint._retry_on_overflow(flaky, P, None) == "ok"
        assert made == [128, 248]  # 1.2 x the reported count + 8
        made.clear()

        def always():
            raise adjoint._ListOverflow(64)

        try:
            adjoint._retry_on_overflow(always, P, None)
            raise AssertionError("no error")
        except RuntimeError as e:
            assert "overflowing" in str(e)
        assert len(made) == 4
    finally:
        adjoint._Graphs = orig


def test_fp32_distance_band_bounds_the_rounding():
    """The mixed-precision Verlet-list path decides a pair from FP32 positions
    unless its FP32 r^2 lies within a band of the cutoff.  The band rests on the
    bound |r2_f32 - r2| <= 2^-24 (17.3 B r + 6.5 r^2) for coordinates and shifts
    of magnitude <= B and r near the cutoff; check it on random pairs laid out as
    the kernel forms them ((x_j - x_i) + shift, then the sum of squares)."""
    rng = np.random.default_rng(0)
    u = 2.0 ** -24
    worst = 0.0
    for B, rc in ((20.0, 2.5), (60.0, 8.5), (800.0, 8.5), (300.0, 6.0)):
        m = 200_000
        xi = rng.uniform(-B / 2, B / 2, (m, 3))
        d = rng.normal(size=(m, 3))
        d *= (rc * rng.uniform(0.98, 1.02, m) / np.linalg.norm(d, axis=1))[:, None]
        shift = rng.choice([-1.0, 0.0, 1.0], (m, 3)) * (B / 2)
        xj = xi + d - shift  # so that (xj - xi) + shift = d exactly in real arithmetic
        ok = np.all(np.abs(xj) <= B, axis=1)
        xi, xj, shift, d = xi[ok], xj[ok], shift[ok], d[ok]
        r2 = np.sum(((xj - xi) + shift) ** 2, axis=1)  # FP64 reference
        f = np.float32
        a = (xj.astype(f) - xi.astype(f)) + shift.astype(f)
        r2f = (a[:, 0] * a[:, 0] + a[:, 1] * a[:, 1]) + a[:, 2] * a[:, 2]
        bound = u * (17.3 * B * rc + 6.5 * rc * rc)
        ratio = np.abs(r2f.astype(np.float64) - r2).max() / bound
        worst = max(worst, ratio)
        assert ratio <= 1.0, (B, rc, ratio)
    assert worst > 0.01  # the test exercises rounding at all


def test_histogram_window_drops_only_negligible_terms():
    """The loss histogram adds a pair only to the bins within 12 widths of its
    distance; every dropped term is below exp(-72) of the pair's peak term, far
    under the FP64 rounding of the bins it does reach."""
    rng = np.random.default_rng(1)
    r_max, nb, w = 8.0, 64, 0.05
    bw = r_max / nb
    c = (np.arange(nb) + 0.5) * bw
    r = rng.uniform(0.5, r_max, 20000)
    g = np.exp(-((r[:, None] - c[None, :]) ** 2) / (2 * w * w))
    full = g.sum(0)
    k0 = np.maximum(0, np.ceil((r - 12 * w) / bw - 0.5)).astype(int)
    k1 = np.minimum(nb - 1, np.floor((r + 12 * w) / bw - 0.5)).astype(int)
    kk = np.arange(nb)[None, :]
    win = np.where((kk >= k0[:, None]) & (kk <= k1[:, None]), g, 0.0).sum(0)
    dropped = np.where((kk < k0[:, None]) | (kk > k1[:, None]), g, 0.0)
    assert dropped.max() <= np.exp(-72.0)
    np.testing.assert_allclose(win, full, rtol=1e-15, atol=1e-28)


def test_verlet_list_prune_argument():
    """VerletListModel's list pruning: off unless asked for, and a pruning skin
    at or above the list skin (the whole list is within reach) turns it off."""
    import pytest

    from tsb import models

    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0, device="cpu")
    assert models.VerletListModel(m, skin=1.5).prune == 0.0
    assert models.VerletListModel(m, skin=1.5, prune=0.3).prune == 0.3
    assert models.VerletListModel(m, skin=1.0, prune=1.2).prune == 0.0
    with pytest.raises(ValueError):
        models.VerletListModel(m, skin=1.0, prune=-0.1)


def test_narrow_routing_uses_image_estimate():
    """Systems of at most 256 atoms whose estimated atoms + images fit 95 % of
    the narrow table take the two-per-SM blocks, largest first after the wide
    ones; a thin cell (many images) stays wide."""
    from tsb import integrators, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(64, 8, 512, seed=3)
    st = state_from_arrays(d, device="cpu")
    order, n_wide = integrators._split_order(st, 6.0, 1.2)
    counts = np.bincount(d["system_idx"])
    order = order.numpy()
    wide, narrow = order[:n_wide], order[n_wide:]
    assert (counts[narrow] <= integrators.NARROW_MAX_ATOMS).all()
    assert (counts[wide] > integrators.NARROW_MAX_ATOMS).sum() == \
        (counts > integrators.NARROW_MAX_ATOMS).sum()
    # each group largest first
    assert (np.diff(counts[narrow]) <= 0).all() and (np.diff(counts[wide]) <= 0).all()
    # the estimate: n * prod(1 + 2 R |b_k|) <= 0.95 * table for every narrow system
    R = 7.2
    for s in narrow:
        cr = np.asarray(d["cell"][s]).T
        h = R * np.linalg.norm(np.linalg.inv(cr).T, axis=1)
        assert counts[s] * np.prod(1 + 2 * h) <= 0.95 * integrators.NARROW_MAX_IMAGES + 1e-9
