"""The allocation-free fused-MD entry point, called through the C ABI.

``tsb_fused_md_static`` serves callers that cannot allocate device memory (hosts
that own all device memory through their own pool, code that must avoid the
implicit synchronisation of cudaMalloc/cudaFree, fixed memory budgets).  It must
give the same results as ``tsb_fused_md``, which takes a caller workspace, on
consecutive calls -- its fixed scratch keeps the previous call's contents, so
the second call checks that everything that must start at zero is cleared.

This file is collected last on purpose: a failure here leaves every other test
already run.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup(n_sys=24, seed=31):
    from tsb import integrators, models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(n_sys, 8, 512, seed=seed)
    st = state_from_arrays(d, device="cuda")
    st.rng = seed
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0)
    md = integrators.nvt_langevin_init(st, m, kT=1000.0 * workloads.KB_EV)
    return md, m


def _args(md, m, x, p, f, energy, rebuilds, status, n_steps, counter):
    from tsb import _lib as L
    from tsb import workloads

    dev = md.device
    n_sys = md.n_systems
    dt = torch.full((n_sys,), 0.002 * workloads.METAL_TIME, dtype=torch.float64, device=dev)
    kT = torch.full((n_sys,), 1000.0 * workloads.KB_EV, dtype=torch.float64, device=dev)
    gam = torch.full((n_sys,), 10.0 / workloads.METAL_TIME, dtype=torch.float64, device=dev)
    keep = [dt, kT, gam, md.cell.mT.contiguous(), md.masses.contiguous(),
            md.system_idx.contiguous()]
    args = (L.INT_LANGEVIN, m.kind, L.ptr(m.table), m.n_species, None, L.ptr(x), L.ptr(p),
            L.ptr(f), L.ptr(keep[4]), L.ptr(keep[3]), L.ptr(keep[5]), md.n_atoms, n_sys,
            None, m.cutoff, 1.0, n_steps, L.ptr(dt), L.ptr(kT), L.ptr(gam), 77, counter,
            L.ptr(energy), L.ptr(rebuilds), L.ptr(status))
    return args, keep


def test_static_entry_matches_workspace_entry_on_two_calls():
    from tsb import _lib as L

    lib = L.load()
    md, m = _setup()
    dev = md.device
    outs = {}
    for name in ("tsb_fused_md", "tsb_fused_md_static"):
        x = md.positions.clone()
        p = md.momenta.clone()
        f = md.forces.clone()
        energy = torch.zeros(md.n_systems, dtype=torch.float64, device=dev)
        rebuilds = torch.zeros(md.n_systems, dtype=torch.int32, device=dev)
        status = torch.full((4,), -7, dtype=torch.int32, device=dev)
        ws = torch.empty(lib.tsb_fused_workspace_size(md.n_atoms, md.n_systems),
                         dtype=torch.uint8, device=dev)
        stream = L.stream_ptr(dev)
        for call, counter in ((0, 0), (1, 40)):  # two calls in a row, trajectory continues
            args, keep = _args(md, m, x, p, f, energy, rebuilds, status, 40, counter)
            if name == "tsb_fused_md":
                a = list(args)
                a.insert(22, None)  # counter_dev: none, the counter is passed by value
                a.insert(24, None)  # stress: not requested
                rc = lib.tsb_fused_md(*a, L.ptr(ws), ws.numel(), stream)
            else:
                rc = lib.tsb_fused_md_static(*args, stream)
            assert rc == L.TSB_OK, (name, call, rc)
            torch.cuda.synchronize()
            assert status.tolist()[0] == 0, (name, call, status.tolist())
            outs[(name, call)] = (x.clone(), p.clone(), f.clone(), energy.clone())
    for call in (0, 1):
        a = outs[("tsb_fused_md", call)]
        b = outs[("tsb_fused_md_static", call)]
        for u, v in zip(a, b):
            # same kernel, deterministic summation order: identical results
            torch.testing.assert_close(v, u, rtol=0.0, atol=0.0)
    # the trajectory really moved between the two calls
    assert not torch.equal(outs[("tsb_fused_md_static", 0)][0],
                           outs[("tsb_fused_md_static", 1)][0])
    assert np.isfinite(outs[("tsb_fused_md_static", 1)][3].cpu().numpy()).all()


def test_static_entry_rejects_too_many_systems():
    from tsb import _lib as L

    lib = L.load()
    md, m = _setup(n_sys=4)
    dev = md.device
    status = torch.zeros(4, dtype=torch.int32, device=dev)
    energy = torch.zeros(md.n_systems, dtype=torch.float64, device=dev)
    x, p, f = md.positions.clone(), md.momenta.clone(), md.forces.clone()
    args, keep = _args(md, m, x, p, f, energy, None, status, 1, 0)
    args = list(args)
    args[12] = 16385  # n_systems beyond TSB_FUSED_STATIC_MAX_SYSTEMS (16384)
    rc = lib.tsb_fused_md_static(*args, L.stream_ptr(dev))
    assert rc == L.TSB_ERR_CAPACITY
    torch.cuda.synchronize()
    assert torch.equal(x, md.positions)  # nothing was launched


def test_static_entry_allocates_nothing():
    """After a first call on the device (which looks up the array's address),
    further calls leave the device's free memory and torch's allocator untouched."""
    from tsb import _lib as L

    lib = L.load()
    md, m = _setup(n_sys=12, seed=5)
    dev = md.device
    x, p, f = md.positions.clone(), md.momenta.clone(), md.forces.clone()
    energy = torch.zeros(md.n_systems, dtype=torch.float64, device=dev)
    status = torch.zeros(4, dtype=torch.int32, device=dev)
    args, keep = _args(md, m, x, p, f, energy, None, status, 10, 0)
    stream = L.stream_ptr(dev)
    assert lib.tsb_fused_md_static(*args, stream) == L.TSB_OK  # warm-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    alloc0, reserved0 = torch.cuda.memory_allocated(dev), torch.cuda.memory_reserved(dev)
    for _ in range(3):
        assert lib.tsb_fused_md_static(*args, stream) == L.TSB_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    assert torch.cuda.memory_allocated(dev) == alloc0
    assert torch.cuda.memory_reserved(dev) == reserved0
    assert status.tolist()[0] == 0


def test_static_entry_reports_a_bad_system_index_and_recovers():
    """A system index outside [0, n_systems) is reported in the status word and
    nothing is written outside the fixed array; the next valid call on the same
    array still equals the workspace entry."""
    from tsb import _lib as L

    lib = L.load()
    md, m = _setup(n_sys=6, seed=8)
    dev = md.device
    stream = L.stream_ptr(dev)
    bad = md.system_idx.clone()
    bad[-1] = md.n_systems  # one past the last system (still sorted)
    x, p, f = md.positions.clone(), md.momenta.clone(), md.forces.clone()
    energy = torch.zeros(md.n_systems, dtype=torch.float64, device=dev)
    status = torch.zeros(4, dtype=torch.int32, device=dev)
    args, keep = _args(md, m, x, p, f, energy, None, status, 5, 0)
    args = list(args)
    args[10] = L.ptr(bad)
    assert lib.tsb_fused_md_static(*args, stream) == L.TSB_OK
    torch.cuda.synchronize()
    st = status.tolist()
    assert st[0] == L.TSB_ERR_INVALID_ARG and st[2] == 3 and st[1] == md.n_atoms - 1, st
    # valid calls afterwards: static == workspace entry, bitwise
    outs = []
    for name in ("tsb_fused_md_static", "tsb_fused_md"):
        x, p, f = md.positions.clone(), md.momenta.clone(), md.forces.clone()
        energy = torch.zeros(md.n_systems, dtype=torch.float64, device=dev)
        status = torch.full((4,), -7, dtype=torch.int32, device=dev)
        args, keep = _args(md, m, x, p, f, energy, None, status, 20, 0)
        if name == "tsb_fused_md":
            ws = torch.empty(lib.tsb_fused_workspace_size(md.n_atoms, md.n_systems),
                             dtype=torch.uint8, device=dev)
            a = list(args)
            a.insert(22, None)
            a.insert(24, None)
            rc = lib.tsb_fused_md(*a, L.ptr(ws), ws.numel(), stream)
        else:
            rc = lib.tsb_fused_md_static(*args, stream)
        assert rc == L.TSB_OK
        torch.cuda.synchronize()
        assert status.tolist()[0] == 0
        outs.append((x, p, energy))
    for u, v in zip(*outs):
        torch.testing.assert_close(u, v, rtol=0.0, atol=0.0)
