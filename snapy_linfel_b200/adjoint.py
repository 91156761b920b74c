"""Reverse mode of the FP64 hydro step behind ``torch.autograd``.

The reference has no adjoint; this module adds one on top of the same
forward path (``snapb_stage``):

* ``Adjoint`` — the reverse entry points of include/snapb.h
  (``snapb_stage_adjoint``, ``snapb_hydro_forward_adjoint``,
  ``snapb_bc_adjoint``) with their workspace;
* ``hydro_forward(cfg, dt, u)`` — ``du`` of HydroImpl::forward
  (src/hydro/hydro_forward.cpp:14-217) as a differentiable op;
* ``bc_apply(cfg, x, kind)`` — a differentiable boundary fill
  (src/bc/bc_func.cpp:7-63);
* ``rollout(opts, u, s, dts, checkpoint_every)`` — ``len(dts)`` RK3 steps
  (MeshBlockImpl::forward, src/mesh/meshblock.cpp:577-786) as one
  differentiable op.  The forward pass keeps the state every
  ``checkpoint_every`` steps; the backward pass re-runs each segment from its
  checkpoint, keeping the three stage inputs of every step of the segment, and
  runs the stage reverses (2, 1, 0) step by step.  ``checkpoint_every=0``
  keeps the three stage inputs of every step during the forward pass instead
  (3 states per step of device memory, no re-run).

dt is a constant of the adjoint: ``dts`` holds the step sizes of the forward
run (for instance the CFL values of a first, non-differentiated run).  Every
switch of the forward path (Riemann wave selections, upwinding, clamps) is
differentiated on the branch taken at the given state.
"""
from __future__ import annotations

import ctypes

from . import _lib
from .config import CONSERVED, PRIMITIVE, SCALAR, HydroConfig, MeshBlockOptions


def _opts(options):
    if isinstance(options, HydroConfig):
        return MeshBlockOptions(options)
    return options


class Adjoint:
    """Workspace and calls of the reverse entry points for one configuration."""

    def __init__(self, cfg: HydroConfig, device=None):
        import torch

        self.cfg = cfg
        self.device = torch.device(device if device is not None else "cuda")
        self.lib = _lib.lib()
        nbytes = self.lib.snapb_adjoint_workspace_size(ctypes.byref(cfg))
        if nbytes == 0:
            raise _lib.SnapbError("configuration not supported by the adjoint: " +
                                  self.lib.snapb_last_error().decode())
        self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=self.device)

    def _ws(self):
        return _lib.ptr(self.workspace), ctypes.c_size_t(self.workspace.numel())

    def stage(self, stage, dt, u, s, gu_out, gs_out, gu0, gs0):
        """Reverse of one RK stage; returns (gu, gs) and accumulates gu0, gs0."""
        import torch

        gu = torch.empty_like(u)
        gs = torch.empty_like(s) if s is not None else None
        ws, nb = self._ws()
        rc = self.lib.snapb_stage_adjoint(
            ctypes.byref(self.cfg), int(stage), _lib.ptr(dt), _lib.ptr(u), _lib.ptr(s),
            _lib.ptr(gu_out), _lib.ptr(gs_out), _lib.ptr(gu), _lib.ptr(gs), _lib.ptr(gu0),
            _lib.ptr(gs0), ws, nb, _lib.stream_ptr())
        _lib.check(rc, "snapb_stage_adjoint")
        return gu, gs

    def hydro_forward(self, dt, u, g_du):
        import torch

        g_u = torch.empty_like(u)
        ws, nb = self._ws()
        rc = self.lib.snapb_hydro_forward_adjoint(
            ctypes.byref(self.cfg), _lib.ptr(dt), _lib.ptr(u), _lib.ptr(g_du.contiguous()),
            _lib.ptr(g_u), ws, nb, _lib.stream_ptr())
        _lib.check(rc, "snapb_hydro_forward_adjoint")
        return g_u

    def bc(self, g, kind):
        return bc_adjoint(self.cfg, g, kind)


def bc_adjoint(cfg, g, kind):
    """BC^T of a cotangent (out of place)."""
    import torch

    out = torch.empty_like(g)
    rc = _lib.lib().snapb_bc_adjoint(ctypes.byref(cfg), _lib.ptr(g.contiguous()), _lib.ptr(out),
                                     int(g.shape[0]), int(kind), _lib.stream_ptr())
    _lib.check(rc, "snapb_bc_adjoint")
    return out


def _bc_fill(cfg, x, kind):
    y = x.contiguous().clone()
    rc = _lib.lib().snapb_bc_apply(ctypes.byref(cfg), _lib.ptr(y), int(y.shape[0]), int(kind),
                                   _lib.stream_ptr())
    _lib.check(rc, "snapb_bc_apply")
    return y


def _autograd():
    import torch

    class BCFill(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x, cfg, kind):
            ctx.cfg, ctx.kind = cfg, kind
            return _bc_fill(cfg, x, kind)

        @staticmethod
        def backward(ctx, g):
            return bc_adjoint(ctx.cfg, g.contiguous(), ctx.kind), None, None

    class HydroForward(torch.autograd.Function):
        @staticmethod
        def forward(ctx, u, dt, cfg, adj):
            u = u.contiguous()
            du = torch.empty_like(u)
            from .mesh import MeshBlock

            mb = MeshBlock(cfg, device=u.device)
            ws, nb = mb._ws()
            rc = mb.lib.snapb_hydro_forward(ctypes.byref(cfg), _lib.ptr(dt), _lib.ptr(u),
                                            _lib.ptr(mb.hydro_w), _lib.ptr(du), None, ws, nb,
                                            _lib.stream_ptr())
            _lib.check(rc, "snapb_hydro_forward")
            ctx.save_for_backward(u, dt)
            ctx.adj = adj
            return du

        @staticmethod
        def backward(ctx, g):
            u, dt = ctx.saved_tensors
            return ctx.adj.hydro_forward(dt, u, g.contiguous()), None, None, None

    class Rollout(torch.autograd.Function):
        @staticmethod
        def forward(ctx, u, s, dts, runner, k):
            ctx.runner, ctx.k = runner, k
            nsteps = dts.numel()
            cks = []
            kept = None
            runner.load(u, s)
            if k <= 0:  # every step's stage inputs, kept now: no re-run backwards
                kept = [runner.step(dts[n:n + 1], keep=True) for n in range(nsteps)]
            else:
                for n in range(nsteps):
                    if n % k == 0:
                        cks.append(runner.snapshot())
                    runner.step(dts[n:n + 1])
            ctx.cks, ctx.kept = cks, kept
            ctx.save_for_backward(dts)
            uT, sT = runner.snapshot()
            return uT, (sT if sT is not None else torch.zeros(0, device=u.device))

        @staticmethod
        def backward(ctx, gu, gs):
            (dts,) = ctx.saved_tensors
            runner, k = ctx.runner, ctx.k
            adj = runner.adjoint()
            nsteps = dts.numel()
            g = gu.contiguous().clone()
            has_s = runner.cfg.nscalar > 0
            gsc = gs.contiguous().clone() if has_s else None
            if ctx.kept is not None:
                segments = [(0, nsteps, ctx.kept)]
            else:
                segments = []
                for seg in range(len(ctx.cks)):
                    n0 = seg * k
                    segments.append((n0, min(n0 + k, nsteps), None))
            for n0, n1, inputs in reversed(segments):
                if inputs is None:  # re-run the segment from its checkpoint
                    runner.load(*ctx.cks[n0 // k])
                    inputs = [runner.step(dts[n:n + 1], keep=True) for n in range(n0, n1)]
                for n in reversed(range(n0, n1)):
                    dt = dts[n:n + 1]
                    gu0 = torch.zeros_like(g)
                    gs0 = torch.zeros_like(gsc) if has_s else None
                    for st in (2, 1, 0):
                        u_in, s_in = inputs[n - n0][st]
                        g, gsc = adj.stage(st, dt, u_in, s_in, g, gsc, gu0, gs0)
                    g = g + gu0
                    if has_s:
                        gsc = gsc + gs0
            return g, (gsc if has_s else None), None, None, None

    return BCFill, HydroForward, Rollout


_FN = None


def _fns():
    global _FN
    if _FN is None:
        _FN = _autograd()
    return _FN


class StepRunner:
    """Forward stepping of one block with fixed step sizes (FP64, snapb_stage)."""

    def __init__(self, options, device=None):
        from .mesh import MeshBlock

        self.options = _opts(options)
        self.cfg = self.options.hydro
        self.mb = MeshBlock(self.options, device=device)
        self._adj = None

    def adjoint(self) -> Adjoint:
        if self._adj is None:
            self._adj = Adjoint(self.cfg, self.mb.device)
        return self._adj

    def load(self, u, s=None):
        mb = self.mb
        mb.hydro_u.copy_(u)
        if self.cfg.nscalar:
            mb.scalar_s.copy_(s)
            mb.scalar_r.copy_(mb.scalar_s / mb.hydro_u[0:1])

    def snapshot(self):
        mb = self.mb
        return (mb.hydro_u.clone(), mb.scalar_s.clone() if self.cfg.nscalar else None)

    def step(self, dt, keep=False):
        """One RK3 step with the device scalar dt; keep=True returns the three
        stage inputs [(u, s)] * 3."""
        mb = self.mb
        mb.dt.copy_(dt.reshape(1))
        kept = []
        for st in range(3):
            if keep:
                kept.append(self.snapshot())
            mb.forward(st)
        return kept


def bc_apply(cfg, x, kind=CONSERVED):
    """Differentiable boundary fill of a [nv, nc3, nc2, nc1] CUDA tensor."""
    return _fns()[0].apply(x, cfg, kind)


def hydro_forward(cfg, dt, u, adjoint: Adjoint | None = None):
    """du of HydroImpl::forward as a differentiable op (dt: device scalar)."""
    import torch

    adj = adjoint if adjoint is not None else Adjoint(cfg, u.device)
    dt = torch.as_tensor(dt, dtype=torch.float64, device=u.device).reshape(1)
    return _fns()[1].apply(u, dt, cfg, adj)


def rollout(options, u, s=None, dts=None, checkpoint_every: int = 20, runner=None):
    """len(dts) RK3 steps from the full-array state (u, s) as one
    differentiable op; returns (u_T, s_T) (s_T empty without scalars).

    The backward pass re-runs each checkpoint segment once and needs the
    adjoint workspace plus 3 * checkpoint_every saved states;
    checkpoint_every=0 keeps 3 states per step during the forward pass and
    re-runs nothing."""
    import torch

    opts = _opts(options)
    if runner is None:
        runner = StepRunner(opts, device=u.device)
    dts = torch.as_tensor(dts, dtype=torch.float64, device=u.device).reshape(-1).contiguous()
    if s is None:
        s = torch.zeros(0, dtype=torch.float64, device=u.device)
        if opts.hydro.nscalar:
            raise _lib.SnapbError("rollout: scalar_s is required for the scalar model")
    sarg = s if opts.hydro.nscalar else None
    return _fns()[2].apply(u, sarg if sarg is not None else s, dts, runner,
                           int(checkpoint_every))


def initial_state(cfg, w, r=None):
    """(u, s) of MeshBlockImpl::initialize (src/mesh/meshblock.cpp:330-500) as
    differentiable torch ops: primitive boundary fill, W -> U (ideal gas,
    src/eos/ideal_gas_impl.h), conserved boundary fill; s = rho r."""
    import torch

    w = bc_apply(cfg, w, PRIMITIVE)
    rho = w[0:1]
    mom = rho * w[1:4]
    en = w[4:5] / (cfg.gammad - 1.0) + 0.5 * (mom * w[1:4]).sum(dim=0, keepdim=True)
    u = bc_apply(cfg, torch.cat([rho, mom, en]), CONSERVED)
    if r is None:
        return u
    r = bc_apply(cfg, r, SCALAR)
    return u, bc_apply(cfg, rho * r, SCALAR)


def cfl_steps(options, u, s=None, nsteps=1, device=None):
    """Step sizes of a plain forward run (cfl * CFL limit at every step)."""
    import torch

    runner = StepRunner(options, device=device or u.device)
    runner.load(u, s)
    mb = runner.mb
    out = []
    for _ in range(nsteps):
        # the CFL limit needs hydro_w of the current state
        rc = mb.lib.snapb_cons2prim(ctypes.byref(mb.cfg), _lib.ptr(mb.hydro_u),
                                    _lib.ptr(mb.hydro_w), _lib.stream_ptr())
        _lib.check(rc, "snapb_cons2prim")
        dt = mb.max_time_step().clone()
        out.append(dt)
        runner.step(dt)
    return torch.cat(out)


__all__ = ["Adjoint", "StepRunner", "bc_adjoint", "bc_apply", "hydro_forward", "rollout",
           "cfl_steps", "initial_state"]
