"""Hand-written adjoint of the 2D solid load step, and a torch.autograd.Function
over a whole simulation (gradient of a loss w.r.t. a per-particle log-Young's
modulus field).

The reference's inverse analysis takes Warp's tape gradient of the last
residual with the state held fixed (solvers/quasi_static_coupled_solver_3d.py:
159-165, 323-325; its scalar-E "last-step partial" is reproduced by
quasi_static_coupled_solver_3d.E_grad).  Here the derivative is total: every
load step is a map s_n -> s_{n+1} = G2P(s_n, u*(s_n, E)) with R(u*; s_n, E) = 0,
and its reverse pass is

    1. rebuild the step's active set and block pattern from the checkpoint s_n,
       re-assemble the converged Jacobian K = -dR/du at u* and transpose it;
    2. adjoint G2P:  q_bar = (d out/d q)^T out_bar,  u_bar = (d out/d u)^T out_bar;
    3. transpose solve K^T lambda = u_bar (GPU GMRES);
    4. adjoint P2G:  q_bar += R_q^T lambda;

with q = (x, lp, F_old, b_old, E) per particle.  Particle states are
checkpointed per load step together with the converged nodal solution, so
the Newton iterations are not repeated (one assembly per reverse step).
"""
import ctypes as C

import torch

from . import _lib as L
from .engine import _p


def _adj_struct(d):
    a = L.Adjoint()
    a.x, a.lp, a.F, a.b, a.E = _p(d["x"]), _p(d["lp"]), _p(d["F"]), _p(d["b"]), _p(d["E"])
    return a


class LoadStepAdjoint:
    """Checkpointing forward driver + reverse load step for a 2D solid solver."""

    def __init__(self, solver, seed="displacement"):
        self.s = solver
        e = solver.engine
        if e.kind != L.KIND_SOLID2D:
            raise NotImplementedError("the hand-written adjoint covers the 2D solid solver")
        self.e = e
        dev = e.device
        N = e.N
        z = lambda *shape: torch.zeros(shape, dtype=torch.float64, device=dev)
        self.bar = dict(x=z(N, 2), lp=z(N, 2), F=z(N, 3, 3), b=z(N, 3, 3), E=z(N))
        self.q = dict(x=z(N, 2), lp=z(N, 2), F=z(N, 3, 3), b=z(N, 3, 3), E=z(N))
        self.grad_E = z(N)
        self.tape = []
        self.seed_mode = seed
        self._scratch = dict(F_new=z(N, 3, 3), b_new=z(N, 3, 3), sigma=z(N, 3, 3), pi_new=z(N))
        self._AT = None
        self._ubar = None
        self._lam = None
        self._ws = None

    # ------------------------------------------------------------------ forward with checkpoints
    def forward_step(self, k, n_steps, keep=True):
        e = self.e
        ck = dict(x=e.x.clone(), lp=e.lp.clone(), F=e.F_old.clone(), b=e.b_old.clone(), k=k, n=n_steps)
        self.s.advance_one_step(k, n_steps)
        ck["u"] = e.u_new.clone()
        if keep:
            self.tape.append(ck)
        else:
            self.tape = [ck]
        return ck

    # ------------------------------------------------------------------ reverse step
    def _swap(self, ck):
        """Point the engine at the checkpoint state (and scratch outputs)."""
        e = self.e
        saved = dict(x=e.x, lp=e.lp, F_old=e.F_old, b_old=e.b_old, F_new=e.F_new, b_new=e.b_new, sigma=e.sigma,
                     pi_new=e.pi_new, u_new=e.u_new, u_old=e.u_old)
        e.x, e.lp, e.F_old, e.b_old = ck["x"], ck["lp"], ck["F"], ck["b"]
        e.F_new, e.b_new, e.sigma, e.pi_new = (self._scratch["F_new"], self._scratch["b_new"], self._scratch["sigma"],
                                               self._scratch["pi_new"])
        e.u_new = ck["u"]
        e.u_old = torch.zeros_like(ck["u"])
        return saved

    def _restore(self, saved):
        for k, v in saved.items():
            setattr(self.e, k, v)

    def backward_step(self, k=None, n_steps=None, ck=None, rtol=None):
        """Reverse of one load step: consumes self.bar (adjoint of the state after
        the step), produces the adjoint of the state before it and accumulates
        grad_E.  Uses the most recent checkpoint unless one is given."""
        if ck is None:
            ck = self.tape.pop()
        e = self.e
        saved = self._swap(ck)
        try:
            # rebuild the step's active set and pattern from the checkpoint
            # (u_new now aliases the checkpointed converged solution: no reset)
            e.node_active.zero_()
            e.cell_span.zero_()
            e.sort_and_activate()
            e.build_system()
            e.assemble(self.s._mat, ck["k"], ck["n"], want_K=True)
            g, st, pt, A = e.grid_struct(), e.step_struct(ck["k"], ck["n"]), e.particles_struct(), e.bsr_struct()
            s = e.stream
            nv = e.nnzb * e.nf * e.nf
            vt = torch.float64 if e.prec == L.PREC_F64 else torch.float32
            if self._AT is None or self._AT.numel() < nv:
                self._AT = torch.zeros(int(nv * 1.25) + 16, dtype=vt, device=e.device)
            L.call("gw_bsr_transpose", C.byref(g), C.byref(A), e.prec, _p(self._AT), s)
            n = e.n_rows * e.nf
            if self._ubar is None or self._ubar.numel() < n:
                self._ubar = torch.zeros(int(n * 1.25) + 16, dtype=torch.float64, device=e.device)
                self._lam = torch.zeros_like(self._ubar)
            seed, q = _adj_struct(self.bar), _adj_struct(self.q)
            L.call("gw_adjoint_g2p", C.byref(g), C.byref(self.s._mat), C.byref(st), C.byref(pt), _p(e.u_new),
                   _p(e.u_old), _p(e.free_mask), C.byref(A), C.byref(seed), C.byref(q), _p(self._ubar), s)
            AT = e.bsr_struct()
            AT.vals = _p(self._AT)
            self._lam[:n].zero_()
            if rtol is None:
                rtol = max(e.krylov_rtol, e.adjoint_rtol_floor)
            it, rr, rc = e.gmres_solve(AT, self._ubar, self._lam, rtol)
            if rc not in (L.GW_OK, L.GW_ENOCONV):
                L.check(rc, "adjoint transpose solve")
            self.last_krylov = (it, rr)
            L.call("gw_adjoint_residual", C.byref(g), C.byref(self.s._mat), C.byref(st), C.byref(pt), _p(e.u_new),
                   _p(e.u_old), _p(e.free_mask), C.byref(A), _p(self._lam), C.byref(q), s)
        finally:
            self._restore(saved)
        # the adjoint of the state before the step becomes the next seed
        for key in ("x", "lp", "F", "b"):
            self.bar[key].copy_(self.q[key])
        self.grad_E += self.q["E"]
        return self.q

    def seed_displacement_misfit(self, target=None):
        """x_bar = x - x0 - target: the seed of L = 1/2 |x - x0 - target|^2."""
        e = self.e
        d = e.x - e.x0
        if target is not None:
            d = d - target
        for v in self.bar.values():
            v.zero_()
        self.bar["x"].copy_(d)
        return 0.5 * float((d * d).sum())


def simulate(solver, n_steps, adj=None, steps=None):
    """Run load steps 0..steps-1 of n_steps with checkpoints (for the adjoint)."""
    adj = adj or LoadStepAdjoint(solver)
    for k in range(steps if steps is not None else n_steps):
        adj.forward_step(k, n_steps)
    return adj


class DisplacementMisfit(torch.autograd.Function):
    """L(logE) = 1/2 sum_p |x_p - x0_p - target_p|^2 after `steps` load steps of
    `n_steps`, for a 2D solid solver whose per-particle Young's modulus is
    exp(logE).  backward() runs the hand-written adjoint in reverse over the
    checkpointed load steps."""

    @staticmethod
    def forward(ctx, logE, solver, target, n_steps, steps, reset_fn):
        reset_fn(solver)
        solver.engine.E = torch.exp(logE.detach()).contiguous()
        adj = LoadStepAdjoint(solver)
        for k in range(steps):
            adj.forward_step(k, n_steps)
        loss = adj.seed_displacement_misfit(target)
        ctx.adj = adj
        ctx.save_for_backward(logE)
        return torch.tensor(loss, dtype=torch.float64, device=logE.device)

    @staticmethod
    def backward(ctx, gout):
        adj = ctx.adj
        (logE,) = ctx.saved_tensors
        while adj.tape:
            adj.backward_step()
        g = adj.grad_E * torch.exp(logE) * gout
        return g, None, None, None, None, None
