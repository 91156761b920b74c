"""Module-level Python surface of the hydro step, mirroring the reference's
torch::nn::Module interfaces (and their pybind mirrors, python/csrc/*.cpp):
each class is built from the options and calls one entry point of
include/snapb.h on CUDA tensors, with caller-owned, preallocated outputs where
the reference has them and the same argument meaning.

* Hydro.forward(dt, u, w=None) -> du, Hydro.max_time_step(w) -> float
  (HydroImpl, src/hydro/hydro.hpp:120-131)
* Reconstruct.forward(w, dim) -> wlr [2, nv, ...]
  (ReconstructImpl, src/recon/reconstruct.hpp:96)
* RiemannSolver.forward(wl, wr, dim, flx, face_pressure=None) -> flx
  (RiemannSolverImpl, src/riemann/riemann_solver.hpp:73-76)
* ImplicitHydro.forward(du, w, dt) -> correction du_new - du_old
  (ImplicitHydroImpl, src/implicit/implicit_hydro.hpp:75-76)
* EquationOfState.compute("U->W" | "W->U", [x]) -> y
  (EquationOfStateImpl::compute, src/eos/equation_of_state.hpp:132-133)

Every class raises on CPU tensors: there is no CPU path.
"""
from __future__ import annotations

import ctypes

from . import _lib
from .config import CONSERVED, PRIMITIVE, RIEMANN, HydroConfig, MeshBlockOptions


def _block_cfg(block) -> HydroConfig:
    """the configuration (geometry, boundaries, scalars) of a parent block"""
    if isinstance(block, HydroConfig):
        return block
    if isinstance(block, MeshBlockOptions):
        return block.hydro
    if hasattr(block, "cfg") and isinstance(block.cfg, HydroConfig):  # a MeshBlock
        return block.cfg
    raise TypeError("block: a MeshBlock, MeshBlockOptions or HydroConfig")


def _cfg(options, block=None) -> HydroConfig:
    """options: MeshBlockOptions / HydroConfig, or the snapy options classes
    (HydroOptions; the geometry then comes from `block`, as the reference's
    modules take their coordinates from the parent mesh block)"""
    from .options import CoordinateOptions, HydroOptions, InterpOptions

    if isinstance(options, MeshBlockOptions):
        return options.hydro
    if isinstance(options, HydroConfig):
        return options
    if isinstance(options, HydroOptions):
        if block is None:
            raise TypeError("HydroOptions need a block for the geometry")
        b = _block_cfg(block)
        coord = CoordinateOptions(nx1=b.nx1, nx2=b.nx2, nx3=b.nx3, nghost=b.nghost,
                                  x1min=b.x1min, x1max=b.x1max, x2min=b.x2min,
                                  x2max=b.x2max, x3min=b.x3min, x3max=b.x3max)
        from .config import BC, RECON

        names = {v: k for k, v in BC.items()}
        rnames = {v: k for k, v in RECON.items()}
        return options.config(coord, bc=tuple(names[int(x)] for x in b.bc), nscalar=b.nscalar,
                              scalar_recon=InterpOptions(rnames[b.scalar_recon_type])
                              .scale(bool(b.scalar_recon_scale)))
    from .config import RECON, RGAS
    from .options import (EquationOfStateOptions, ImplicitOptions, ReconstructOptions,
                          RiemannSolverOptions)

    if isinstance(options, (ReconstructOptions, RiemannSolverOptions, ImplicitOptions,
                            EquationOfStateOptions)):
        # one module's options on the parent block's configuration
        if block is None:
            raise TypeError(f"{type(options).__name__} need a block for the geometry")
        c = _block_cfg(block).copy()
        if isinstance(options, ReconstructOptions):
            it = options.interp() or InterpOptions()
            c.recon1_type = c.recon23_type = RECON[it.type()]
            c.recon1_shock = c.recon23_shock = int(bool(options.shock()))
            c.recon1_scale = c.recon23_scale = int(bool(it.scale()))
        elif isinstance(options, RiemannSolverOptions):
            if options.type() not in ("roe", "lmars", "hllc"):
                raise ValueError(f"unsupported hydro riemann solver {options.type()!r}")
            c.riemann = RIEMANN[options.type()]
        elif isinstance(options, ImplicitOptions):
            options.type()  # rejects unsupported schemes
            c.implicit_scheme = int(options.scheme())
        else:
            if options.type() != "ideal-gas":
                raise ValueError(f"equation of state {options.type()!r} is not on this path")
            c.gammad = float(options.gammad())
            c.rgas = RGAS / float(options.weight())
        return c
    raise TypeError("options: the snapy options classes, MeshBlockOptions or HydroConfig")


def _cuda64(*ts):
    import torch

    for t in ts:
        if t is None:
            continue
        if not t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous():
            raise _lib.SnapbError("expected contiguous float64 CUDA tensors")


def _dt_tensor(dt, device):
    import torch

    if isinstance(dt, torch.Tensor):
        return dt.reshape(1).to(device=device, dtype=torch.float64)
    return torch.tensor([float(dt)], dtype=torch.float64, device=device)


class _Module:
    def __init__(self, options, block=None):
        self.cfg = _cfg(options, block)
        self.options = options
        self.lib = _lib.lib()

    def __call__(self, *args, **kw):
        return self.forward(*args, **kw)

    def _check(self, rc, name):
        _lib.check(rc, name)


class Hydro(_Module):
    """the stage tendency du = -dt div F + forcing (+ implicit correction)"""

    def __init__(self, options, block=None):
        super().__init__(options, block)
        self._ws = None

    def _workspace(self, device):
        import torch

        if self._ws is None or self._ws.device != device:
            n = self.lib.snapb_workspace_size(ctypes.byref(self.cfg))
            if n == 0:
                raise _lib.SnapbError(self.lib.snapb_last_error().decode())
            self._ws = torch.empty(n, dtype=torch.uint8, device=device)
        return self._ws

    def forward(self, dt, u, w=None, mass_corr=None):
        """du (already x dt) of the conserved state u; w receives the
        primitive state (allocated when None)"""
        import torch

        _cuda64(u, w, mass_corr)
        w = torch.empty_like(u) if w is None else w
        du = torch.empty_like(u)
        ws = self._workspace(u.device)
        dtt = _dt_tensor(dt, u.device)
        self._check(self.lib.snapb_hydro_forward(
            ctypes.byref(self.cfg), _lib.ptr(dtt), _lib.ptr(u), _lib.ptr(w), _lib.ptr(du),
            _lib.ptr(mass_corr), _lib.ptr(ws), ctypes.c_size_t(ws.numel()), _lib.stream_ptr()),
            "snapb_hydro_forward")
        return du

    def max_time_step(self, w) -> float:
        import torch

        _cuda64(w)
        ws = self._workspace(w.device)
        out = torch.empty(1, dtype=torch.float64, device=w.device)
        self._check(self.lib.snapb_max_time_step(
            ctypes.byref(self.cfg), _lib.ptr(w), _lib.ptr(out), _lib.ptr(ws),
            ctypes.c_size_t(ws.numel()), _lib.stream_ptr()), "snapb_max_time_step")
        return float(out)


class Reconstruct(_Module):
    """interface states along one axis; group 0 = hydro, 1 = scalars"""

    def __init__(self, options, block=None, group: int = 0):
        super().__init__(options, block)
        self.group = group

    def forward(self, w, dim: int):
        """dim: 3 = x1, 2 = x2, 1 = x3 (the tensor dimension of [nv, nc3,
        nc2, nc1]); returns wlr [2, nv, nc3, nc2, nc1], face i = i-1/2"""
        import torch

        _cuda64(w)
        nv = int(w.shape[0])
        wlr = torch.empty((2,) + tuple(w.shape), dtype=w.dtype, device=w.device)
        self._check(self.lib.snapb_reconstruct(ctypes.byref(self.cfg), int(dim), self.group,
                                               _lib.ptr(w), nv, _lib.ptr(wlr),
                                               _lib.stream_ptr()), "snapb_reconstruct")
        return wlr


class RiemannSolver(_Module):
    """face fluxes of a hydro solver ('roe', 'lmars', 'hllc'; default the
    configuration's)"""

    def __init__(self, options, block=None, solver: str | None = None):
        if isinstance(block, str):  # RiemannSolver(options, "hllc")
            block, solver = None, block
        super().__init__(options, block)
        self.solver = RIEMANN[solver] if solver is not None else int(self.cfg.riemann)

    def forward(self, wl, wr, dim: int, flx, face_pressure=None):
        _cuda64(wl, wr, flx, face_pressure)
        self._check(self.lib.snapb_riemann(
            ctypes.byref(self.cfg), self.solver, int(dim), _lib.ptr(wl), _lib.ptr(wr),
            int(wl.shape[0]), _lib.ptr(flx), _lib.ptr(face_pressure), None,
            _lib.stream_ptr()), "snapb_riemann")
        return flx


class ImplicitHydro(_Module):
    """vertically implicit correction of a stage tendency"""

    def __init__(self, options, block=None):
        super().__init__(options, block)
        self._ws = None

    def forward(self, du, w, dt, mass_corr=None):
        """returns du_new - du_old (du itself is left unchanged)"""
        import torch

        _cuda64(du, w, mass_corr)
        if self._ws is None or self._ws.device != du.device:
            n = self.lib.snapb_workspace_size(ctypes.byref(self.cfg))
            self._ws = torch.empty(n, dtype=torch.uint8, device=du.device)
        out = du.clone()
        dtt = _dt_tensor(dt, du.device)
        self._check(self.lib.snapb_implicit_correction(
            ctypes.byref(self.cfg), _lib.ptr(dtt), _lib.ptr(out), _lib.ptr(w),
            _lib.ptr(mass_corr), _lib.ptr(self._ws), ctypes.c_size_t(self._ws.numel()),
            _lib.stream_ptr()), "snapb_implicit_correction")
        return out - du


class EquationOfState(_Module):
    """the ideal-gas conversions between conserved and primitive states"""

    def compute(self, ab: str, args):
        import torch

        (x,) = args
        _cuda64(x)
        y = torch.empty_like(x)
        if ab == "U->W":
            rc = self.lib.snapb_cons2prim(ctypes.byref(self.cfg), _lib.ptr(x), _lib.ptr(y),
                                          _lib.stream_ptr())
        elif ab == "W->U":
            rc = self.lib.snapb_prim2cons(ctypes.byref(self.cfg), _lib.ptr(x), _lib.ptr(y),
                                          _lib.stream_ptr())
        else:
            raise ValueError(f"conversion {ab!r} is not on this path (U->W, W->U)")
        self._check(rc, "snapb_" + ("cons2prim" if ab == "U->W" else "prim2cons"))
        return y

    def forward(self, u):
        return self.compute("U->W", [u])


__all__ = ["Hydro", "Reconstruct", "RiemannSolver", "ImplicitHydro", "EquationOfState",
           "CONSERVED", "PRIMITIVE"]
