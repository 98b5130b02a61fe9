"""Differentiable NVE trajectories with a hand-written adjoint (FP64).

``trajectory_loss(sigma, epsilon, q0, p0, problem)`` is a ``torch.autograd.Function``:
its forward integrates velocity Verlet (torch_sim/integrators/nve.py:74-130)
for ``problem.n_steps`` steps with species-matrix Lennard-Jones forces
(lennard_jones.py:23-47; sigma/epsilon [ns, ns] symmetric) and returns the loss
``sum_s,b (h_sb(q_T) - target_sb)^2`` of the Gaussian-smeared pair-distance
histogram of the final frame; its backward runs the exact discrete adjoint:

    lam_q = dL/dq_T, lam_p = 0
    for k = T-1 .. 0:   lam_p += (dt/m) lam_q
                        lam_q += c_k J_F(q_k)^T lam_p,  g += c_k dF(q_k)/dtheta^T lam_p
    (c_k = dt, dt/2 at k = 0; J_F = -Hessian; the q_T term vanishes as lam_p = 0)

re-integrating each 20-step segment from a stored checkpoint (positions and
momenta every ``checkpoint_every`` steps), so memory is O(N * T / k + N * k).
The reference's own route (autograd through PairPotentialModel with
retain_graph=True, pair_potential.py:420-425) omits J_F and gives wrong
trajectory gradients; finite differences are the arbiter here.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import torch

from . import _lib as L


@dataclasses.dataclass
class TrajectoryProblem:
    """Everything fixed during differentiation (FP64 CUDA tensors)."""

    cell_row: torch.Tensor      # [S,3,3]
    pbc: torch.Tensor           # [S,3] uint8
    system_idx: torch.Tensor    # [N] int64
    species: torch.Tensor       # [N] int32
    masses: torch.Tensor        # [N]
    n_species: int
    n_steps: int
    dt: float
    cutoff: float = 8.5125
    target: torch.Tensor | None = None  # [S, n_bins]
    r_max: float = 8.0
    n_bins: int = 64
    width: float = 0.05
    checkpoint_every: int = 20

    @property
    def n_atoms(self):
        return self.system_idx.shape[0]

    @property
    def n_systems(self):
        return self.cell_row.shape[0]

    @property
    def max_sys(self):
        """Largest system's atom count (binning hint; cached per system_idx)."""
        return L.max_system_atoms(self.system_idx, self.n_systems)


def lj_table(sigma: torch.Tensor, epsilon: torch.Tensor) -> torch.Tensor:
    ns = sigma.shape[0]
    t = torch.zeros((ns, ns, 5), dtype=torch.float64, device=sigma.device)
    t[..., 0] = sigma
    t[..., 1] = epsilon
    t[..., 3] = float("inf")
    return t.contiguous()


def _ws(dev, n, s, per_atom):
    return L.Workspace.get(dev, L.load().tsb_adjoint_workspace_size(n, s, per_atom))


def forces(q, table, P: TrajectoryProblem, ws=None):
    """FP64 LJ energy [S] and forces [N,3] (tsb_pair_forward, FP64 pair math)."""
    dev = q.device
    n, s = P.n_atoms, P.n_systems
    e = torch.empty(s, dtype=torch.float64, device=dev)
    f = torch.empty((n, 3), dtype=torch.float64, device=dev)
    if ws is None:
        ws = L.Workspace.get(dev, L.load().tsb_pair_workspace_size(n, s))
    L.call("tsb_pair_forward", L.POT_LJ, L.ptr(table), P.n_species, L.ptr(P.species), L.ptr(q),
           L.ptr(P.cell_row), L.ptr(P.pbc), L.ptr(P.system_idx), n, s, L.F64, P.cutoff,
           L.OUT_FORCES | L.MATH_FP64, L.ptr(e), L.ptr(f), None, None, None, None, P.max_sys,
           L.ptr(ws), ws.numel(), L.stream_ptr(dev))
    return e, f


def histogram(q, P: TrajectoryProblem):
    h = torch.empty((P.n_systems, P.n_bins), dtype=torch.float64, device=q.device)
    ws = _ws(q.device, P.n_atoms, P.n_systems, P.n_bins)
    L.call("tsb_rdf_hist", L.ptr(q), L.ptr(P.cell_row), L.ptr(P.pbc), L.ptr(P.system_idx),
           P.n_atoms, P.n_systems, P.r_max, P.n_bins, P.width, L.ptr(h), P.max_sys, L.ptr(ws),
           ws.numel(), L.stream_ptr(q.device))
    return h


def _hist_grad(q, dl_dh, P):
    g = torch.empty_like(q)
    ws = _ws(q.device, P.n_atoms, P.n_systems, P.n_bins)
    L.call("tsb_rdf_hist_grad", L.ptr(q), L.ptr(P.cell_row), L.ptr(P.pbc), L.ptr(P.system_idx),
           P.n_atoms, P.n_systems, P.r_max, P.n_bins, P.width, L.ptr(dl_dh.contiguous()),
           L.ptr(g), P.max_sys, L.ptr(ws), ws.numel(), L.stream_ptr(q.device))
    return g


def _hvp(q, table, v, coef, lam_q, gparams, P, ws=None):
    if ws is None:
        ws = _ws(q.device, P.n_atoms, P.n_systems, 2 * P.n_species ** 2)
    L.call("tsb_lj_hvp", L.ptr(table), P.n_species, L.ptr(P.species), L.ptr(q),
           L.ptr(P.cell_row), L.ptr(P.pbc), L.ptr(P.system_idx), P.n_atoms, P.n_systems,
           P.cutoff, L.ptr(v), float(coef), L.ptr(lam_q), L.ptr(gparams), P.max_sys, L.ptr(ws),
           ws.numel(), L.stream_ptr(q.device))


def _vv_step(q, p, f, table, P, inv_m, ws=None, force_fn=None):
    """One velocity-Verlet step (same floating-point order as nve.py:118-130:
    p + f * (dt / 2), q + (p * inv_m) * dt, each product and sum rounded on its
    own), the kick-drift and the closing kick one launch each.  ``force_fn(q,
    table)`` replaces the per-call neighbour search when given."""
    dt, n, st = P.dt, q.shape[0], L.stream_ptr(q.device)
    q_new, p_half = torch.empty_like(q), torch.empty_like(p)
    L.call("tsb_vv_kick_drift", L.ptr(q), L.ptr(p), L.ptr(f), L.ptr(inv_m), dt / 2, dt,
           L.ptr(q_new), L.ptr(p_half), n, st)
    _, f = force_fn(q_new, table) if force_fn else forces(q_new, table, P, ws)
    p_new = torch.empty_like(p)
    L.call("tsb_vv_kick", L.ptr(p_half), L.ptr(f), dt / 2, L.ptr(p_new), n, st)
    return q_new, p_new, f


def _adj_kick(lam_p, lam_q, inv_m, P):
    """lam_p += lam_q * (dt * inv_m), in place, one launch."""
    L.call("tsb_adj_kick", L.ptr(lam_p), L.ptr(lam_q), L.ptr(inv_m), P.dt, lam_p.shape[0],
           L.stream_ptr(lam_p.device))


class _ListOverflow(RuntimeError):
    pass


def _lists_fit(P, skin):
    """Every periodic plane spacing at least cutoff + skin (the lists' limit)."""
    inv = torch.linalg.inv(P.cell_row)
    width = 1.0 / inv.norm(dim=1)  # [S, 3]: spacing of the planes of lattice vector k
    per = P.pbc.bool()
    return bool(((width >= P.cutoff + skin) | ~per).all())


class _ListForces:
    """FP64 LJ energy and forces of a trajectory through batched Verlet lists
    (``tsb_vlist_check`` / ``_build`` / ``_forces``): every call checks the
    lists and rebuilds the expired systems on the device, so a captured graph
    needs no host decision.  The pairs inside the cutoff are those of the
    per-call search; only the order of their sums follows the lists.  A list
    overflow (more neighbours than ``cap``) is kept in ``sticky`` and read by
    the host after a graph replay."""

    def __init__(self, P: "TrajectoryProblem", skin: float = 1.0, cap: int = 0):
        n, ns, dev = P.n_atoms, P.n_systems, P.cell_row.device
        self.P, self.skin = P, float(skin)
        rcs = P.cutoff + self.skin
        counts = torch.bincount(P.system_idx, minlength=ns).double()
        vol = torch.linalg.det(P.cell_row).abs().clamp_min(1e-30)
        dens = float((counts / vol).max())
        self.cap = max(cap, min(4096, int(4.19 * rcs ** 3 * dens * 1.35) + 16))
        self.list = torch.empty(self.cap * n, dtype=torch.int32, device=dev)
        self.counts = torch.empty(n, dtype=torch.int32, device=dev)
        self.flags = torch.zeros(2, dtype=torch.int32, device=dev)
        self.sticky = torch.zeros(1, dtype=torch.int32, device=dev)
        self.ws = torch.empty(L.load().tsb_vlist_workspace_size(n, ns), dtype=torch.uint8,
                              device=dev)
        self.e = torch.empty(ns, dtype=torch.float64, device=dev)
        self.scratch = torch.empty(L.load().tsb_vlist_hvp_scratch_size(n, P.n_species),
                                   dtype=torch.uint8, device=dev)
        L.call("tsb_vlist_reset", n, ns, L.ptr(self.ws), self.ws.numel(), L.stream_ptr(dev))

    def _update(self, q):
        P, st = self.P, L.stream_ptr(q.device)
        n, ns = P.n_atoms, P.n_systems
        L.call("tsb_vlist_check", L.ptr(q), L.ptr(P.cell_row), L.ptr(P.system_idx), None, n, ns,
               L.F64, P.cutoff, self.skin, 0.0, L.ptr(self.flags), L.ptr(self.ws),
               self.ws.numel(), st)
        L.call("tsb_vlist_build", L.ptr(q), L.ptr(P.cell_row), L.ptr(P.pbc),
               L.ptr(P.system_idx), L.ptr(P.species), n, ns, L.F64, P.cutoff, self.skin,
               L.ptr(self.list), L.ptr(self.counts), self.cap, P.max_sys, L.ptr(self.flags),
               L.ptr(self.ws), self.ws.numel(), st)
        torch.maximum(self.sticky, self.flags[1:], out=self.sticky)

    def __call__(self, q, table):
        P, st = self.P, L.stream_ptr(q.device)
        n, ns = P.n_atoms, P.n_systems
        self._update(q)
        f = torch.empty((n, 3), dtype=torch.float64, device=q.device)
        L.call("tsb_vlist_forces", L.POT_LJ, L.ptr(table), P.n_species, L.ptr(P.species),
               L.ptr(self.list), L.ptr(self.counts), L.ptr(q), L.ptr(P.cell_row),
               L.ptr(P.system_idx), None, n, ns, L.F64, P.cutoff, 0.0,
               L.OUT_FORCES | L.MATH_FP64, L.ptr(self.e), L.ptr(f), None, None, None,
               L.ptr(self.ws), self.ws.numel(), st)
        return self.e, f

    def hvp(self, q, table, v, coef, lam_q, gparams):
        """lam_q += coef J_F(q)^T v and the parameter gradients (as ``_hvp``)."""
        P, st = self.P, L.stream_ptr(q.device)
        self._update(q)
        L.call("tsb_vlist_lj_hvp", L.ptr(table), P.n_species, L.ptr(P.species),
               L.ptr(self.list), L.ptr(self.counts), L.ptr(q), L.ptr(P.cell_row),
               L.ptr(P.system_idx), P.n_atoms, P.n_systems, P.cutoff, L.ptr(v), float(coef),
               L.ptr(lam_q), L.ptr(gparams), L.ptr(self.scratch), self.scratch.numel(),
               L.ptr(self.ws), self.ws.numel(), st)

    def check(self):
        """Raise _ListOverflow (after growing the list) if any call overflowed."""
        st = int(self.sticky.item())
        if st == 0:
            return
        if st >= (1 << 30):
            raise ValueError("adjoint Verlet lists need every cell width >= cutoff + 1 A")
        raise _ListOverflow(st)


class _Graphs:
    """CUDA graphs of the checkpoint segments of one problem.

    A segment of ``length`` steps is (a) forces at its first positions, then
    ``length`` velocity-Verlet steps keeping the positions of each step, and (b)
    the adjoint sweep back over those positions.  Every call in them (the C-ABI
    force / HVP launches and torch element-wise ops) is stream-ordered and
    allocates nothing once its workspace exists, so each part is captured once
    and replayed: one graph launch per segment instead of some forty host calls
    per step.  The graphs read and write the static buffers below.  Forces come
    from batched Verlet lists kept across steps and segments (``_ListForces``):
    the per-call search's pairs, summed in list order, so results agree with the
    step-by-step path to rounding."""

    def __init__(self, P: TrajectoryProblem, table: torch.Tensor, cap: int = 0):
        dev = P.cell_row.device
        n, f64 = P.n_atoms, torch.float64
        self.P = P
        self.lf = _ListForces(P, cap=cap) if _lists_fit(P, 1.0) else None
        self.table = table.clone().contiguous()
        self.q0 = torch.zeros((n, 3), dtype=f64, device=dev)
        self.p0 = torch.zeros_like(self.q0)
        self.lam_q = torch.zeros_like(self.q0)
        self.lam_p = torch.zeros_like(self.q0)
        self.gpar = torch.zeros((P.n_systems, P.n_species, P.n_species, 2), dtype=f64,
                                device=dev)
        self.inv_m = (1.0 / P.masses).contiguous()
        lib = L.load()
        self.ws_pair = torch.empty(lib.tsb_pair_workspace_size(n, P.n_systems),
                                   dtype=torch.uint8, device=dev)
        self.ws_adj = torch.empty(
            lib.tsb_adjoint_workspace_size(n, P.n_systems, 2 * P.n_species ** 2),
            dtype=torch.uint8, device=dev)
        self.fwd, self.bwd, self.out = {}, {}, {}

    @staticmethod
    def _capture(body, keep=()):
        """Warm ``body`` up once, then capture it.  The warm-up really runs, so the
        buffers in ``keep`` (state that ``body`` updates in place) are restored
        after it."""
        saved = [t.clone() for t in keep]
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            body()  # warm-up outside the capture
        torch.cuda.current_stream().wait_stream(side)
        for t, v in zip(keep, saved):
            t.copy_(v)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            body()
        return g

    def forward(self, length):
        """Replay: (q0, p0) -> positions of each step and (q, p) after ``length``."""
        if length not in self.fwd:
            P = self.P

            fn = self.lf or (lambda q, t: forces(q, t, P, self.ws_pair))

            def body():
                q, p = self.q0, self.p0
                _, f = fn(q, self.table)
                seg = [q]
                for k in range(length):
                    q, p, f = _vv_step(q, p, f, self.table, P, self.inv_m, force_fn=fn)
                    if k < length - 1:
                        seg.append(q)
                self.out[length] = (seg, q, p)

            self.fwd[length] = self._capture(body)
        self.fwd[length].replay()
        if self.lf is not None:
            self.lf.check()
        return self.out[length]

    def backward(self, length, first):
        """Replay the adjoint sweep over the positions of the last ``forward(length)``
        (``first``: the segment holds step 0, whose coefficient is dt / 2)."""
        key = (length, first)
        if key not in self.bwd:
            P = self.P
            seg = self.out[length][0]

            def body():
                for k in range(length - 1, -1, -1):
                    _adj_kick(self.lam_p, self.lam_q, self.inv_m, P)
                    coef = P.dt / 2 if (first and k == 0) else P.dt
                    if self.lf is not None:
                        self.lf.hvp(seg[k], self.table, self.lam_p, coef, self.lam_q, self.gpar)
                    else:
                        _hvp(seg[k], self.table, self.lam_p, coef, self.lam_q, self.gpar, P,
                             self.ws_adj)

            self.bwd[key] = self._capture(body, keep=(self.lam_q, self.lam_p, self.gpar))
        self.bwd[key].replay()
        if self.lf is not None:
            self.lf.check()


def _graphs_for(P: TrajectoryProblem, table: torch.Tensor) -> _Graphs:
    G = P.__dict__.get("_graphs")
    if G is None:
        G = _Graphs(P, table)
        P.__dict__["_graphs"] = G
    else:
        G.table.copy_(table)
    return G


def _retry_on_overflow(fn, P, table):
    """Run ``fn``; when a Verlet list overflowed, rebuild the graphs with a larger
    list and run it again."""
    for _ in range(4):
        try:
            return fn()
        except _ListOverflow as e:
            P.__dict__["_graphs"] = _Graphs(P, table, cap=int(int(e.args[0]) * 1.2) + 8)
    raise RuntimeError("adjoint: Verlet list kept overflowing")


def _integrate_graphs(q0, p0, table, P, keep_checkpoints):
    G = _graphs_for(P, table)
    G.q0.copy_(q0)
    G.p0.copy_(p0)
    ckpt = {}
    for c in range(0, P.n_steps, P.checkpoint_every):
        if keep_checkpoints:
            ckpt[c] = (G.q0.clone(), G.p0.clone())
        _, q, p = G.forward(min(P.checkpoint_every, P.n_steps - c))
        G.q0.copy_(q)
        G.p0.copy_(p)
    return G.q0.clone(), G.p0.clone(), ckpt


def integrate(q0, p0, table, P: TrajectoryProblem, keep_checkpoints=True, use_graphs=True):
    """Velocity Verlet for ``P.n_steps`` steps from (q0, p0); returns (q_T, p_T, and
    the checkpoints {step: (q, p)} every ``P.checkpoint_every`` steps).  With
    ``use_graphs`` each checkpoint segment replays one CUDA graph."""
    if use_graphs and q0.is_cuda and P.n_steps > 0:
        return _retry_on_overflow(
            lambda: _integrate_graphs(q0, p0, table, P, keep_checkpoints), P, table)
    inv_m = (1.0 / P.masses).contiguous()
    q, p = q0.contiguous(), p0.contiguous()
    _, f = forces(q, table, P)
    ckpt = {0: (q, p)}
    for k in range(P.n_steps):
        q, p, f = _vv_step(q, p, f, table, P, inv_m)
        if keep_checkpoints and (k + 1) % P.checkpoint_every == 0 and k + 1 < P.n_steps:
            ckpt[k + 1] = (q, p)
    return q, p, ckpt


def loss_of(q_T, P):
    h = histogram(q_T, P)
    return ((h - P.target) ** 2).sum(), h


def _adjoint_graphs(table, ckpt, lam_q, P):
    """The backward sweep with one forward and one adjoint graph replay per segment."""
    G = _graphs_for(P, table)
    G.lam_q.copy_(lam_q)
    G.lam_p.zero_()
    G.gpar.zero_()
    for c in sorted(ckpt, reverse=True):
        length = min(P.checkpoint_every, P.n_steps - c)
        G.q0.copy_(ckpt[c][0])
        G.p0.copy_(ckpt[c][1])
        G.forward(length)
        G.backward(length, c == 0)
    return G.lam_q.clone(), G.lam_p.clone(), G.gpar.clone()


def loss_and_grad(sigma, epsilon, q0, p0, P: TrajectoryProblem, use_graphs=True):
    """Loss and its gradients w.r.t. sigma [ns,ns], epsilon [ns,ns], q0, p0."""
    table = lj_table(sigma, epsilon)
    qT, pT, ckpt = integrate(q0, p0, table, P, use_graphs=use_graphs)
    loss, h = loss_of(qT, P)
    lam_q = _hist_grad(qT, 2.0 * (h - P.target), P)
    if use_graphs and q0.is_cuda and P.n_steps > 0:
        lam_q, lam_p, gpar = _retry_on_overflow(
            lambda: _adjoint_graphs(table, ckpt, lam_q, P), P, table)
        g = gpar.sum(0)
        gs = g[..., 0] + g[..., 0].T - torch.diag(torch.diagonal(g[..., 0]))
        ge = g[..., 1] + g[..., 1].T - torch.diag(torch.diagonal(g[..., 1]))
        return loss, gs, ge, lam_q, lam_p
    lam_p = torch.zeros_like(lam_q)
    gpar = torch.zeros((P.n_systems, P.n_species, P.n_species, 2), dtype=torch.float64,
                       device=q0.device)
    inv_m = (1.0 / P.masses).contiguous()
    starts = sorted(ckpt)
    for c in reversed(starts):
        end = min(c + P.checkpoint_every, P.n_steps)
        q, p = ckpt[c]
        _, f = forces(q, table, P)
        seg = [q]
        for _ in range(c, end - 1):
            q, p, f = _vv_step(q, p, f, table, P, inv_m)
            seg.append(q)
        for k in range(end - 1, c - 1, -1):
            _adj_kick(lam_p, lam_q, inv_m, P)
            _hvp(seg[k - c], table, lam_p, P.dt if k > 0 else P.dt / 2, lam_q, gpar, P)
    g = gpar.sum(0)
    # sigma_ab and sigma_ba are one parameter: symmetrise the gradient
    gs = g[..., 0] + g[..., 0].T - torch.diag(torch.diagonal(g[..., 0]))
    ge = g[..., 1] + g[..., 1].T - torch.diag(torch.diagonal(g[..., 1]))
    return loss, gs, ge, lam_q, lam_p


class TrajectoryLoss(torch.autograd.Function):
    """loss = TrajectoryLoss.apply(sigma, epsilon, q0, p0, problem)."""

    @staticmethod
    def forward(ctx, sigma, epsilon, q0, p0, problem):
        ctx.problem = problem
        ctx.save_for_backward(sigma, epsilon, q0, p0)
        qT, _, _ = integrate(q0.detach(), p0.detach(), lj_table(sigma.detach(), epsilon.detach()),
                             problem, keep_checkpoints=False)
        loss, _ = loss_of(qT, problem)
        return loss

    @staticmethod
    def backward(ctx, grad_out):
        sigma, epsilon, q0, p0 = ctx.saved_tensors
        _, gs, ge, gq, gp = loss_and_grad(sigma.detach(), epsilon.detach(), q0.detach(),
                                          p0.detach(), ctx.problem)
        return grad_out * gs, grad_out * ge, grad_out * gq, grad_out * gp, None


trajectory_loss = TrajectoryLoss.apply


def make_problem(state, n_steps, dt, *, cutoff=8.5125, checkpoint_every=20, target=None,
                 species_atomic_numbers=(1, 2)):
    """TrajectoryProblem from a SimState (species = index of the atomic number)."""
    z = torch.as_tensor(species_atomic_numbers, device=state.device)
    lut = torch.full((int(z.max()) + 1,), -1, dtype=torch.int32, device=state.device)
    lut[z] = torch.arange(len(z), dtype=torch.int32, device=state.device)
    n_sys = state.n_systems
    pbc = L.pbc_rows(state.pbc, n_sys, state.positions.device).bool()
    P = TrajectoryProblem(cell_row=state.cell.mT.double().contiguous(),
                          pbc=pbc.to(torch.uint8).contiguous(),
                          system_idx=state.system_idx.contiguous(),
                          species=lut[state.atomic_numbers].contiguous(),
                          masses=state.masses.double().contiguous(), n_species=len(z),
                          n_steps=int(n_steps), dt=float(dt), cutoff=float(cutoff),
                          target=target, checkpoint_every=int(checkpoint_every))
    P.max_sys  # noqa: B018  (reads the size once, outside any graph capture)
    return P


def argon_pair_params(n_species=2, sigma=3.405, epsilon=0.0104, perturb=0.0, seed=0,
                      device="cuda"):
    """Symmetric sigma/epsilon matrices at argon values, optionally scaled by
    1 + U(-perturb, perturb) per unique species pair."""
    rng = np.random.default_rng(seed)
    s = np.full((n_species, n_species), sigma)
    e = np.full((n_species, n_species), epsilon)
    if perturb:
        for a in range(n_species):
            for b in range(a, n_species):
                fs, fe = 1 + rng.uniform(-perturb, perturb, 2)
                s[a, b] = s[b, a] = sigma * fs
                e[a, b] = e[b, a] = epsilon * fe
    return (torch.as_tensor(s, dtype=torch.float64, device=device),
            torch.as_tensor(e, dtype=torch.float64, device=device))
