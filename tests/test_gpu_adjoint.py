"""Hand-written adjoint of NVE trajectories vs exact autograd and finite differences.

Tolerances: vs the FP64 create_graph=True autograd gradient of the same 20-step
trajectory (golden/adjoint.npz): rtol 1e-6; vs central finite differences
(h = 1e-6) on 200-step trajectories: 1e-4 relative."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _small_problem(golden):
    from tsb import adjoint
    from tsb.state import state_from_arrays

    g = golden["adjoint"]["adj"]
    d = {"positions": g["positions"], "masses": g["masses"], "cell": g["cell"],
         "pbc": np.array([True] * 3), "atomic_numbers": g["atomic_numbers"],
         "system_idx": g["system_idx"]}
    st = state_from_arrays(d, device="cuda")
    P = adjoint.make_problem(st, int(g["n_steps"]), float(g["dt"]),
                             target=torch.as_tensor(g["target"], device="cuda"))
    T = lambda x: torch.as_tensor(x, dtype=torch.float64, device="cuda")  # noqa: E731
    return P, T(g["sigma"]), T(g["epsilon"]), st.positions.clone(), T(g["p0"]), g


@pytest.fixture(scope="module")
def golden_adj():
    from conftest import load_golden

    return {"adjoint": load_golden("adjoint.npz")}


def test_adjoint_matches_exact_autograd(golden_adj):
    from tsb import adjoint

    P, sig, eps, q0, p0, g = _small_problem(golden_adj)
    loss, gs, ge, gq, gp = adjoint.loss_and_grad(sig, eps, q0, p0, P)
    np.testing.assert_allclose(float(loss), float(g["loss"]), rtol=1e-9)
    np.testing.assert_allclose(gs.cpu(), g["grad_sigma"], rtol=1e-6)
    np.testing.assert_allclose(ge.cpu(), g["grad_epsilon"], rtol=1e-6)
    np.testing.assert_allclose(gq.cpu(), g["grad_q0"], rtol=1e-6,
                               atol=1e-6 * np.abs(g["grad_q0"]).max())
    np.testing.assert_allclose(gp.cpu(), g["grad_p0"], rtol=1e-6,
                               atol=1e-6 * np.abs(g["grad_p0"]).max())
    # the reference's retain_graph=True route misses the force-Jacobian terms
    ref = g["ref_retain_graph_grad_q0"]
    assert np.linalg.norm(ref - g["grad_q0"]) > 0.05 * np.linalg.norm(g["grad_q0"])


def test_autograd_function_and_checkpoint_invariance(golden_adj):
    from tsb import adjoint

    P, sig, eps, q0, p0, g = _small_problem(golden_adj)
    s = sig.clone().requires_grad_(True)
    e = eps.clone().requires_grad_(True)
    q = q0.clone().requires_grad_(True)
    p = p0.clone().requires_grad_(True)
    loss = adjoint.trajectory_loss(s, e, q, p, P)
    loss.backward()
    np.testing.assert_allclose(s.grad.cpu(), g["grad_sigma"], rtol=1e-6)
    P.checkpoint_every = 7
    _, gs7, _, gq7, _ = adjoint.loss_and_grad(sig, eps, q0, p0, P)
    np.testing.assert_allclose(gs7.cpu(), s.grad.cpu(), rtol=1e-12)
    np.testing.assert_allclose(gq7.cpu(), q.grad.cpu(), rtol=1e-12, atol=1e-12)


def _config5(n_sys=8, n_steps=200):
    from tsb import adjoint, integrators, workloads
    from tsb.state import state_from_arrays

    d = workloads.argon_species_batch(n_sys, (3, 3, 3), seed=3, jitter=0.02)
    st = state_from_arrays(d, device="cuda")
    sysi = st.system_idx
    g = torch.Generator(device="cuda").manual_seed(5)
    p0 = integrators.initialize_momenta(st.positions, st.masses, sysi,
                                        torch.tensor(80.0 * workloads.KB_EV, device="cuda"), g)
    dt = 0.002 * workloads.METAL_TIME
    P = adjoint.make_problem(st, n_steps, dt)
    s0, e0 = adjoint.argon_pair_params()
    qT, _, _ = adjoint.integrate(st.positions, p0, adjoint.lj_table(s0, e0), P, False)
    P.target = adjoint.histogram(qT, P)
    s, e = adjoint.argon_pair_params(perturb=0.05, seed=1)
    return P, s, e, st.positions.clone(), p0


def test_adjoint_vs_finite_differences_200_steps():
    from tsb import adjoint

    P, s, e, q0, p0 = _config5()
    loss, gs, ge, gq, _ = adjoint.loss_and_grad(s, e, q0, p0, P)

    def L(sig, eps, q):
        qT, _, _ = adjoint.integrate(q, p0, adjoint.lj_table(sig, eps), P, False)
        return float(adjoint.loss_of(qT, P)[0])

    h = 1e-6
    for (a, b) in ((0, 0), (0, 1), (1, 1)):
        for which, grad in (("sigma", gs), ("epsilon", ge)):
            dp = torch.zeros_like(s)
            dp[a, b] = dp[b, a] = h * (1.0 if which == "sigma" else 0.003)
            if which == "sigma":
                fd = (L(s + dp, e, q0) - L(s - dp, e, q0)) / (2 * dp[a, b])
            else:
                fd = (L(s, e + dp, q0) - L(s, e - dp, q0)) / (2 * dp[a, b])
            assert abs(float(grad[a, b]) - float(fd)) <= 1e-4 * abs(float(fd)) + 1e-6, \
                (which, a, b, float(grad[a, b]), float(fd))
    idx = torch.argsort(gq.abs().flatten(), descending=True)[:3]
    for k in idx.tolist():
        dq = torch.zeros_like(q0).flatten()
        dq[k] = h
        dq = dq.view_as(q0)
        fd = (L(s, e, q0 + dq) - L(s, e, q0 - dq)) / (2 * h)
        assert abs(float(gq.flatten()[k]) - fd) <= 1e-4 * abs(fd), (k, float(gq.flatten()[k]), fd)


def test_vv_kernels_round_like_the_tensor_expressions():
    """The fused velocity-Verlet and adjoint-kick launches give bitwise the
    results of the element-wise tensor expressions they replace."""
    from tsb import _lib as L

    g = torch.Generator(device="cuda").manual_seed(7)
    n = 1000
    r = lambda: torch.randn((n, 3), dtype=torch.float64, device="cuda", generator=g)  # noqa
    q, p, f, lam_q = r(), r(), r(), r()
    inv_m = 1.0 / (1.0 + torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * 40)
    dt = 0.0123456789
    st = L.stream_ptr(q.device)
    q1, p1 = torch.empty_like(q), torch.empty_like(p)
    L.call("tsb_vv_kick_drift", L.ptr(q), L.ptr(p), L.ptr(f), L.ptr(inv_m), dt / 2, dt,
           L.ptr(q1), L.ptr(p1), n, st)
    ph = p + f * (dt / 2)
    assert torch.equal(p1, ph)
    assert torch.equal(q1, q + (ph * inv_m.unsqueeze(-1)) * dt)
    p2 = torch.empty_like(p)
    L.call("tsb_vv_kick", L.ptr(p1), L.ptr(f), dt / 2, L.ptr(p2), n, st)
    assert torch.equal(p2, p1 + f * (dt / 2))
    lam_p = r()
    expect = lam_p + lam_q * (dt * inv_m.unsqueeze(-1))
    L.call("tsb_adj_kick", L.ptr(lam_p), L.ptr(lam_q), L.ptr(inv_m), dt, n, st)
    assert torch.equal(lam_p, expect)


def test_list_forces_and_hvp_match_the_per_call_search():
    """The captured segments take forces and Hessian-vector products over
    batched Verlet lists: the same pairs as the per-call search, summed in list
    order (max|d|/max|ref| <= 1e-10), also after the atoms have moved."""
    from tsb import adjoint

    P, s, e, q0, p0 = _config5(n_sys=12, n_steps=1)
    table = adjoint.lj_table(s, e)
    lf = adjoint._ListForces(P)
    g = torch.Generator(device="cuda").manual_seed(9)
    v = torch.randn(q0.shape, dtype=torch.float64, device="cuda", generator=g)

    def rel(a, b):
        return float((a - b).abs().max() / b.abs().max())

    q = q0.clone()
    for step in range(3):
        _, f_ref = adjoint.forces(q, table, P)
        _, f = lf(q, table)
        assert rel(f, f_ref) <= 1e-10, step
        lam_ref, lam = torch.zeros_like(q), torch.zeros_like(q)
        gp_ref = torch.zeros((P.n_systems, 2, 2, 2), dtype=torch.float64, device="cuda")
        gp = torch.zeros_like(gp_ref)
        adjoint._hvp(q, table, v, 0.7, lam_ref, gp_ref, P)
        lf.hvp(q, table, v, 0.7, lam, gp)
        assert rel(lam, lam_ref) <= 1e-10 and rel(gp, gp_ref) <= 1e-10, step
        q = q + 0.3 * torch.randn(q.shape, dtype=torch.float64, device="cuda", generator=g)
    lf.check()
