"""The cell-list kernels come in two shapes: a group of lanes per atom for
batches of at most 65,536 atoms (enough warps to hide the search latency) and
one thread per atom above that.  The same systems computed once as a large batch and once as
two small ones must agree to FP64 rounding (max|d|/max|ref| <= 1e-10)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = a.double().cpu().numpy(), b.double().cpu().numpy()
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _split(st, k):
    from tsb.state import select_systems

    return (select_systems(st, list(range(k))),
            select_systems(st, list(range(k, st.n_systems))))


def test_pair_forces_warp_and_thread_kernels_agree():
    from tsb import models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(300, 200, 500, seed=4, jitter=0.05)
    st = state_from_arrays(d, device="cuda")
    assert st.n_atoms > 65536
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                          compute_stress=True, per_atom_energies=True, precision="fp64")
    big = m(st)  # one thread per atom
    a, b = _split(st, 150)
    assert a.n_atoms <= 65536 and b.n_atoms <= 65536
    oa, ob = m(a), m(b)  # a group of lanes per atom
    for k in ("forces", "energies"):
        assert _rel(torch.cat([oa[k], ob[k]]), big[k]) < 1e-10, k
    for k in ("energy", "stress"):
        assert _rel(torch.cat([oa[k], ob[k]]), big[k]) < 1e-10, k


def test_lj_hvp_warp_and_thread_kernels_agree():
    from tsb import adjoint, workloads
    from tsb.state import state_from_arrays

    d = workloads.argon_species_batch(700, (3, 3, 3), seed=3, jitter=0.05)
    st = state_from_arrays(d, device="cuda")
    assert st.n_atoms > 65536
    sig, eps = adjoint.argon_pair_params(perturb=0.05, seed=2)
    table = adjoint.lj_table(sig, eps)
    g = torch.Generator(device="cuda").manual_seed(1)
    v = torch.randn((st.n_atoms, 3), dtype=torch.float64, device="cuda", generator=g)

    def hvp(s, vv):
        P = adjoint.make_problem(s, 1, 1.0)
        lam = torch.zeros_like(vv)
        gp = torch.zeros((s.n_systems, 2, 2, 2), dtype=torch.float64, device="cuda")
        adjoint._hvp(s.positions.contiguous(), table, vv.contiguous(), 0.5, lam, gp, P)
        return lam, gp

    lam_big, g_big = hvp(st, v)
    a, b = _split(st, 350)
    assert a.n_atoms <= 65536 and b.n_atoms <= 65536
    la, ga = hvp(a, v[: a.n_atoms])
    lb, gb = hvp(b, v[a.n_atoms:])
    assert _rel(torch.cat([la, lb]), lam_big) < 1e-10
    assert _rel(torch.cat([ga, gb]), g_big) < 1e-10


def test_per_system_and_batch_wide_binning_agree_exactly(monkeypatch):
    """Batches of systems of at most 4096 atoms are binned one block per system
    (static bin regions); the batch-wide passes give the same bins and the same
    in-bin order (ascending atom index), so forces, energies and stresses agree
    bit for bit."""
    from tsb import _lib as L
    from tsb import adjoint, models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(64, 8, 512, seed=5, jitter=0.05)
    st = state_from_arrays(d, device="cuda")
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                          compute_stress=True, per_atom_energies=True)
    per_sys = m(st)
    assert L.max_system_atoms(st.system_idx, st.n_systems) <= 4096
    monkeypatch.setattr(L, "max_system_atoms", lambda *_: 0)
    batch = m(st)
    for k in ("energy", "forces", "stress", "energies"):
        assert torch.equal(per_sys[k], batch[k]), k
    monkeypatch.undo()

    d = workloads.argon_species_batch(40, (3, 3, 3), seed=1, jitter=0.05)
    st = state_from_arrays(d, device="cuda")
    table = adjoint.lj_table(*adjoint.argon_pair_params(perturb=0.05, seed=2))
    v = torch.randn((st.n_atoms, 3), dtype=torch.float64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(4))
    out = []
    for hint in (None, 0):
        if hint is not None:
            monkeypatch.setattr(L, "max_system_atoms", lambda *_: hint)
        P = adjoint.make_problem(st, 1, 1.0)
        lam = torch.zeros_like(v)
        gp = torch.zeros((st.n_systems, 2, 2, 2), dtype=torch.float64, device="cuda")
        adjoint._hvp(st.positions.contiguous(), table, v, 0.5, lam, gp, P)
        out.append((lam, gp, adjoint.histogram(st.positions.contiguous(), P)))
    for a, b in zip(*out):
        assert torch.equal(a, b)
