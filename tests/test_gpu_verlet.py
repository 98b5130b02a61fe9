"""Verlet-list force path for one large periodic system (500,000-atom workload
at reduced size).  Pair set and forces must equal the per-call neighbour-search
model's; the list is reused until an atom moved more than skin/2.

Tolerance: FP32 pair arithmetic on both paths -> max|dF|/max|F| <= 1e-5 and the
energy to 1e-6 relative; vs the FP64 model the same bound."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _argon(n=(12, 12, 12), dtype=torch.float64, jitter=0.1, seed=0):
    from tsb import workloads
    from tsb.state import state_from_arrays

    d = workloads.argon_fcc(n, jitter=jitter, seed=seed)
    return state_from_arrays(d, device="cuda", dtype=dtype)


def _models(dtype=torch.float64):
    from tsb import models

    base = models.LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=8.5,
                                    compute_stress=True, dtype=dtype)
    ref = models.LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=8.5,
                                   compute_stress=True, dtype=torch.float64, precision="fp64")
    return models.VerletListModel(base, skin=1.0), ref


def _rel(a, b):
    a, b = a.double().cpu().numpy(), b.double().cpu().numpy()
    return np.abs(a - b).max() / np.abs(b).max()


def test_verlet_matches_fused_search_and_reuses_list():
    st = _argon()
    vm, ref = _models()
    out = vm(st)
    r = ref(st)
    assert _rel(out["forces"], r["forces"]) < 1e-5
    assert abs(float(out["energy"][0] - r["energy"][0])) < 1e-6 * abs(float(r["energy"][0]))
    assert _rel(out["stress"], r["stress"]) < 1e-5
    assert vm.n_builds == 1
    # small moves (< skin/2): no rebuild, still exact pairs
    g = torch.Generator(device="cuda").manual_seed(1)
    for _ in range(3):
        st.positions = st.positions + 0.08 * torch.randn(st.positions.shape, device="cuda",
                                                         dtype=st.dtype, generator=g) / 3
        out, r = vm(st), ref(st)
        assert _rel(out["forces"], r["forces"]) < 1e-5
    assert vm.n_builds == 1
    # one atom jumps 0.7 A: list expires and is rebuilt
    st.positions[17] += torch.tensor([0.7, 0.0, 0.0], device="cuda", dtype=st.dtype)
    out, r = vm(st), ref(st)
    assert vm.n_builds == 2
    assert _rel(out["forces"], r["forces"]) < 1e-5


def test_verlet_float32_positions_across_boundary():
    """FP32 state (500k-atom setup): displacements across the periodic boundary
    are formed in FP64, so boundary pairs keep FP32-level force accuracy."""
    st32 = _argon(dtype=torch.float32, seed=3)
    vm, ref = _models(dtype=torch.float32)
    st64 = _argon(dtype=torch.float64, seed=3)
    st64.positions = st32.positions.double()
    st64.cell = st32.cell.double()
    # shift the whole crystal so many atoms sit just inside the upper boundary
    shift = torch.tensor([0.4, 0.3, 0.2], device="cuda")
    st32.positions = (st32.positions - shift.float()).contiguous()
    st64.positions = st32.positions.double()
    out = vm(st32)
    r = ref(st64)
    assert out["forces"].dtype == torch.float32
    assert _rel(out["forces"], r["forces"]) < 1e-5


def test_verlet_unwrapped_positions():
    st = _argon(seed=4)
    vm, ref = _models()
    L = st.cell[0].diagonal()
    k = torch.randint(-3, 4, st.positions.shape, device="cuda").double()
    st.positions = st.positions + k * L
    out, r = vm(st), ref(st)
    assert _rel(out["forces"], r["forces"]) < 1e-5


def test_verlet_small_cell_two_images_and_rejection():
    """A cell narrower than 2 (rc + skin) but wider than rc + skin is fine: the
    list holds both images of a neighbour.  Narrower cells need shifts beyond
    +-1 and are rejected."""
    from tsb import models, workloads
    from tsb.state import state_from_arrays

    d = workloads.argon_fcc((3, 3, 3), jitter=0.1, seed=0)  # 15.8 A: 9.5 < L < 19
    st = state_from_arrays(d, device="cuda")
    vm, ref = _models()
    out, r = vm(st), ref(st)
    assert _rel(out["forces"], r["forces"]) < 1e-5
    d1 = workloads.argon_fcc((1, 1, 1), seed=0)  # 5.26 A < rc + skin
    vm1, _ = _models()
    with pytest.raises(ValueError):
        vm1(state_from_arrays(d1, device="cuda"))
