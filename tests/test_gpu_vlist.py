"""Batched Verlet lists (VerletListModel over many systems whose atoms and cells
move) against the per-call cell-list search and the reference FIRE trajectory.

Tolerances: FP64 pair arithmetic on both paths -> max|d|/max|ref| <= 1e-10 (same
pairs, different summation order); FP32 pair arithmetic -> 1e-5; the reference
FIRE + Frechet trajectory to rtol 1e-7, as for the per-call path.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ka(n_systems=12, n_min=64, n_max=400, seed=0, dtype=torch.float64):
    from tsb import workloads
    from tsb.state import state_from_arrays

    d = workloads.kob_andersen_batch(n_systems, n_min, n_max, seed=seed)
    return state_from_arrays(d, device="cuda", dtype=dtype)


def _models(precision="fp64", dtype=torch.float64, skin=1.0, **kw):
    from tsb import models

    mk = lambda: models.kob_andersen_model(compute_stress=True, precision=precision,  # noqa
                                           dtype=dtype, **kw)
    return models.VerletListModel(mk(), skin=skin), mk()


def _cmp(a, b, rtol, keys=("energy", "forces", "stress")):
    for k in keys:
        x, y = a[k].double().cpu().numpy(), b[k].double().cpu().numpy()
        err = np.abs(x - y).max() / max(np.abs(y).max(), 1e-300)
        assert err <= rtol, (k, err)


def test_vlist_matches_cell_list_per_atom_outputs():
    st = _ka()
    vm, ref = _models(per_atom_energies=True, per_atom_stresses=True)
    _cmp(vm(st), ref(st), 1e-10, ("energy", "forces", "stress", "energies", "stresses"))
    assert vm.n_builds == 1


def test_vlist_moving_atoms_and_cells_rebuild_only_when_needed():
    st = _ka(seed=3)
    vm, ref = _models()
    _cmp(vm(st), ref(st), 1e-10)
    g = torch.Generator(device="cuda").manual_seed(5)
    eye = torch.eye(3, dtype=st.dtype, device="cuda")
    # small moves and strains: lists kept, pairs still exact
    for _ in range(4):
        eps = 2e-4 * torch.randn((st.n_systems, 3, 3), device="cuda", dtype=st.dtype,
                                 generator=g)
        F = eye + 0.5 * (eps + eps.mT)
        st.positions = torch.einsum("nij,nj->ni", F[st.system_idx], st.positions) + \
            0.01 * torch.randn(st.positions.shape, device="cuda", dtype=st.dtype, generator=g)
        st.cell = torch.einsum("nij,njk->nik", F, st.cell).contiguous()
        _cmp(vm(st), ref(st), 1e-10)
    assert vm.n_builds == 1
    # a uniform 3 % strain of one system moves no atom off its affine image: the
    # list stays valid ((cutoff + skin) |F - I| < skin); a 12 % strain expires it
    shape = torch.tensor([[1.0, 0.2, 0.0], [0.2, -0.5, 0.0], [0.0, 0.0, 0.4]],
                         device="cuda", dtype=st.dtype)
    for amp, builds in ((0.03, 1), (0.12, 2)):
        F = eye.repeat(st.n_systems, 1, 1)
        F[4] += amp * shape
        st.positions = torch.einsum("nij,nj->ni", F[st.system_idx],
                                    st.positions).contiguous()
        st.cell = torch.einsum("nij,njk->nik", F, st.cell).contiguous()
        _cmp(vm(st), ref(st), 1e-10)
        assert vm.n_builds == builds
    # atoms moved by lattice vectors (unwrapped) and one atom jumping by 0.7 A
    k = torch.randint(-3, 4, st.positions.shape, device="cuda", generator=g).to(st.dtype)
    st.positions = (st.positions +
                    torch.einsum("ni,nij->nj", k, st.cell.mT[st.system_idx])).contiguous()
    st.positions[17] += torch.tensor([0.7, 0.0, 0.0], device="cuda", dtype=st.dtype)
    _cmp(vm(st), ref(st), 1e-10)


def test_vlist_triclinic_copper_and_open_axis():
    from tsb import models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(6, 256, 500, seed=0, jitter=0.02)
    # every plane spacing (10.6 A at least) exceeds cutoff + skin = 6.8 A
    widths = [1.0 / np.linalg.norm(np.linalg.inv(c.T), axis=0) for c in d["cell"]]
    assert min(w.min() for w in widths) > 6.8
    for pbc in (True, [True, False, True]):
        st = state_from_arrays(d, device="cuda")
        st.pbc = torch.as_tensor(pbc, dtype=torch.bool, device="cuda")
        mk = lambda: models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588,  # noqa
                                       cutoff=6.0, compute_stress=True, precision="fp64")
        vm, ref = models.VerletListModel(mk(), skin=0.8), mk()
        _cmp(vm(st), ref(st), 1e-10)
        st.positions = (st.positions + 0.05).contiguous()
        _cmp(vm(st), ref(st), 1e-10)


def test_vlist_float32_mixed_precision():
    st32 = _ka(seed=7, dtype=torch.float32)
    vm, _ = _models(precision="mixed", dtype=torch.float32)
    _, ref = _models()
    st64 = _ka(seed=7)
    st64.positions = st32.positions.double()
    st64.cell = st32.cell.double()
    out = vm(st32)
    assert out["forces"].dtype == torch.float32
    _cmp(out, ref(st64), 1e-5, ("forces",))


def test_vlist_list_overflow_regrows():
    st = _ka(n_systems=4, seed=9)
    vm, ref = _models()
    vm(st)
    n = st.n_atoms
    vm.cap = 8
    vm.list = torch.empty(vm.cap * n, dtype=torch.int32, device="cuda")
    vm._reset(n, st.n_systems, torch.device("cuda"))
    _cmp(vm(st), ref(st), 1e-10)
    assert vm.cap > 8


def test_vlist_narrow_cell_rejected():
    st = _ka(n_systems=2, n_min=64, n_max=64)  # 12.8 A boxes
    vm, _ = _models(skin=5.0)  # cutoff + skin = 13.5 A
    with pytest.raises(ValueError):
        vm(st)


def test_vlist_forward_into_inactive_systems_untouched():
    st = _ka(n_systems=6, seed=11)
    vm, ref = _models()
    r = ref(st)
    active = torch.tensor([1, 0, 1, 0, 0, 1], dtype=torch.uint8, device="cuda")
    e = torch.full((6,), 7.0, dtype=torch.float64, device="cuda")
    f = torch.full((st.n_atoms, 3), 7.0, dtype=torch.float64, device="cuda")
    s = torch.full((6, 3, 3), 7.0, dtype=torch.float64, device="cuda")
    vm.forward_into(st, energy=e, forces=f, stress=s, sys_active=active)
    act_atoms = active.bool()[st.system_idx]
    assert bool((f[~act_atoms] == 7.0).all()) and bool((e[~active.bool()] == 7.0).all())
    np.testing.assert_allclose(f[act_atoms].cpu(), r["forces"][act_atoms].cpu(), rtol=0,
                               atol=1e-10 * float(r["forces"].abs().max()))
    np.testing.assert_allclose(s[active.bool()].cpu(), r["stress"][active.bool()].cpu(),
                               rtol=1e-10, atol=1e-16)


def test_vlist_fire_frechet_matches_reference(golden):
    from tsb import models, optimizers
    from tsb.state import SimState

    g = golden["fire"]["ase_frechet"]
    dev = torch.device("cuda")
    T = lambda x, dt=torch.float64: torch.as_tensor(np.asarray(x), dtype=dt, device=dev)  # noqa
    st = SimState(positions=T(g["positions"][0]), masses=T(g["masses"]), cell=T(g["cell"][0]),
                  pbc=True, atomic_numbers=T(g["atomic_numbers"], torch.int64),
                  system_idx=T(g["system_idx"], torch.int64))
    m = models.VerletListModel(models.kob_andersen_model(compute_stress=True,
                                                         precision="fp64"), skin=1.0)
    st = optimizers.fire_init(st, m, cell_filter="frechet")
    for k in range(1, g["positions"].shape[0]):
        st = optimizers.fire_step(st, m)
        for key in ("positions", "cell", "energy", "forces", "cell_forces", "velocities"):
            np.testing.assert_allclose(getattr(st, key).cpu().numpy(), g[key][k], rtol=1e-7,
                                       atol=1e-10, err_msg=f"step {k} {key}")


def test_vlist_optimize_converges_like_cell_list():
    from tsb import optimizers

    st = _ka(n_systems=8, n_max=300, seed=13)
    vm, ref = _models()
    st, steps, conv = optimizers.optimize(st, vm, fmax=1e-3, max_steps=6000,
                                          cell_filter="frechet")
    assert bool(conv.all()), (steps, conv)
    out = ref(st)
    fmax = torch.zeros(st.n_systems, dtype=torch.float64, device="cuda").scatter_reduce(
        0, st.system_idx, out["forces"].norm(dim=1), reduce="amax")
    assert float(fmax.max()) < 1e-3
    assert vm.n_builds < steps


def test_single_system_engine_expires_on_cell_change():
    """One large periodic system takes the single-system kernels; a changed cell
    (or a moved atom) rebuilds its list and the forces stay exact."""
    from tsb import models, workloads
    from tsb.state import state_from_arrays

    st = state_from_arrays(workloads.argon_fcc((8, 8, 8), jitter=0.1, seed=2), device="cuda")
    mk = lambda p: models.LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=8.5,  # noqa
                                            compute_stress=True, precision=p)
    vm, ref = models.VerletListModel(mk("mixed"), skin=1.0), mk("fp64")
    _cmp(vm(st), ref(st), 1e-5, ("forces", "stress"))
    assert vm.n_builds == 1 and getattr(vm, "_s_built", False)
    F = torch.eye(3, dtype=st.dtype, device="cuda") * 1.002
    st.positions = (st.positions @ F.T).contiguous()
    st.cell = (F @ st.cell[0]).unsqueeze(0).contiguous()
    _cmp(vm(st), ref(st), 1e-5, ("forces", "stress"))
    assert vm.n_builds == 2


@pytest.mark.parametrize("rel", [1e-7, -1e-7])
def test_vlist_fp32_path_decides_near_cutoff_pairs_in_fp64(rel):
    """Perfect fcc lattices with the cutoff 1e-7 (relative) beyond or short of the
    third neighbour shell: FP32 r^2 cannot tell these pairs apart from the cutoff
    (its rounding is ~1e-6 relative here), so the mixed-precision path must
    re-decide them from the FP64 positions, as the per-call search does.  One
    wrong decision moves a system's energy by |V(r_c)| and its stress by
    r_c |V'(r_c)| / volume; the paths must agree to a tenth of that."""
    from tsb import models, workloads
    from tsb.state import state_from_arrays

    a, sig, eps = 5.26, 3.405, 0.0104
    d = workloads.argon_fcc((4, 4, 4), a=a, jitter=0.0, n_systems=3)
    st = state_from_arrays(d, device="cuda")
    g = torch.Generator(device="cuda").manual_seed(1)
    st.positions = (st.positions + 3.0 * torch.rand((st.n_systems, 3), device="cuda",
                                                    dtype=st.dtype, generator=g)
                    [st.system_idx]).contiguous()
    rc = a * np.sqrt(1.5) * (1.0 + rel)
    mk = lambda p: models.LennardJonesModel(sigma=sig, epsilon=eps, cutoff=rc,  # noqa
                                            compute_stress=True, precision=p)
    vm, ref = models.VerletListModel(mk("mixed"), skin=1.0), mk("mixed")
    s6 = (sig / rc) ** 6
    v_rc = abs(4 * eps * (s6 * s6 - s6))
    w_rc = abs(4 * eps * (-12 * s6 * s6 + 6 * s6)) / (4 * a) ** 3

    def check():
        out, r = vm(st), ref(st)
        assert not vm._last_single
        de = (out["energy"] - r["energy"]).abs().max().item()
        ds = (out["stress"] - r["stress"]).abs().max().item()
        assert de < 0.1 * v_rc and ds < 0.1 * w_rc, (de / v_rc, ds / w_rc)

    check()
    # a uniform 0.5 % strain keeps the lists (bands from the strained cells)
    F = torch.eye(3, dtype=st.dtype, device="cuda") * 1.005
    st.positions = (st.positions @ F.T).contiguous()
    st.cell = torch.einsum("ij,njk->nik", F, st.cell).contiguous()
    check()
    assert vm.n_builds == 1


def _argon_batch(shapes, jitter=0.1, seed=0):
    from tsb import workloads

    parts = [workloads.argon_fcc(n, jitter=jitter, seed=seed + k) for k, n in enumerate(shapes)]
    off = np.cumsum([0] + [len(p["positions"]) for p in parts])
    return {
        "positions": np.concatenate([p["positions"] for p in parts]),
        "masses": np.concatenate([p["masses"] for p in parts]),
        "cell": np.concatenate([p["cell"] for p in parts]),
        "pbc": parts[0]["pbc"],
        "atomic_numbers": np.concatenate([p["atomic_numbers"] for p in parts]),
        "system_idx": np.concatenate([np.full(off[k + 1] - off[k], k, dtype=np.int64)
                                      for k in range(len(parts))]),
    }


def test_vlist_batch_with_a_large_system_rebins_the_batch():
    """Systems of at most 4096 atoms are rebinned one block each; a batch with a
    larger one takes the batch-wide binning.  Both give the per-call pairs."""
    from tsb import models
    from tsb.state import state_from_arrays

    st = state_from_arrays(_argon_batch([(3, 3, 3), (11, 11, 10), (4, 3, 3)]), device="cuda")
    assert st.n_atoms - 108 - 144 > 4096
    mk = lambda: models.LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=8.5,  # noqa
                                          compute_stress=True, precision="fp64")
    vm, ref = models.VerletListModel(mk(), skin=1.0), mk()
    _cmp(vm(st), ref(st), 1e-10)
    assert vm.max_system_atoms > 4096
    g = torch.Generator(device="cuda").manual_seed(3)
    st.positions = (st.positions + 0.4 * torch.randn(st.positions.shape, device="cuda",
                                                     dtype=st.dtype, generator=g)).contiguous()
    _cmp(vm(st), ref(st), 1e-10)
    assert vm.n_builds == 2


def test_vlist_understated_max_system_atoms_still_exact():
    """The size hint only picks the binning: a system above the per-system
    kernel's shared-memory limit under a small hint is binned through global
    memory, with the same pairs."""
    from tsb import models
    from tsb.state import state_from_arrays

    st = state_from_arrays(_argon_batch([(3, 3, 3), (11, 11, 10)]), device="cuda")
    mk = lambda: models.LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=8.5,  # noqa
                                          compute_stress=True, precision="fp64")
    vm, ref = models.VerletListModel(mk(), skin=1.0), mk()
    vm._ensure(st, st.positions, st.cell.mT.contiguous())
    vm.max_system_atoms = 200
    _cmp(vm(st), ref(st), 1e-10)


@pytest.mark.parametrize("n_systems,n_max,precision",
                         [(12, 400, "fp64"), (12, 400, "mixed"), (200, 1000, "fp64"),
                          (200, 1000, "mixed")])
def test_vlist_pruned_front_parts_equal_whole_lists(n_systems, n_max, precision):
    """Pruned lists (each atom evaluates only the entries within its pair cutoff
    + prune at the system's last pruning) give the results of the whole lists
    through moves and strains that trigger re-prunings and rebuilds, to FP64
    rounding (a re-pruned list sums its entries in another order), with several
    lanes per list (12 systems) and one thread per list (200 systems, above
    65,536 atoms); in FP64 also the per-call search's results."""
    tol = 1e-12
    from tsb import models

    dtype = torch.float64
    st = _ka(n_systems=n_systems, n_max=n_max, seed=7, dtype=dtype)
    mk = lambda: models.kob_andersen_model(compute_stress=True, precision=precision,  # noqa
                                           dtype=dtype)
    pruned = models.VerletListModel(mk(), skin=1.0, prune=0.4)
    whole = models.VerletListModel(mk(), skin=1.0, prune=0.0)
    ref = mk()
    g = torch.Generator(device="cuda").manual_seed(11)
    eye = torch.eye(3, dtype=dtype, device="cuda")
    for step in range(14):
        if step:
            eps = 6e-4 * torch.randn((st.n_systems, 3, 3), device="cuda", dtype=dtype,
                                     generator=g)
            F = eye + 0.5 * (eps + eps.mT)
            st.positions = torch.einsum("nij,nj->ni", F[st.system_idx], st.positions) + \
                0.04 * torch.randn(st.positions.shape, device="cuda", dtype=dtype,
                                   generator=g)
            st.cell = torch.einsum("nij,njk->nik", F, st.cell).contiguous()
        a, b = pruned(st), whole(st)
        for k in ("energy", "forces", "stress"):
            x, y = a[k].cpu().numpy(), b[k].cpu().numpy()
            assert np.abs(x - y).max() <= tol * np.abs(y).max(), (step, k)
        # the per-call search's pairs (FP64 sums to 1e-10; in FP32 the two paths
        # form displacements differently, which on these overlapping random boxes
        # moves energies by ~1e-4, so there the whole lists are the reference)
        if precision == "fp64":
            _cmp(a, ref(st), 1e-10)
