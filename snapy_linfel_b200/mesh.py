"""Python mirror of snapy's MeshBlock for the hydro forward step.

``MeshBlock`` owns the block state on one GPU (``hydro_u``, ``hydro_w``,
``scalar_s``, ``scalar_r``, the stage-0 copies and the workspace) and drives
the C ABI: ``initialize`` (MeshBlockImpl::initialize,
src/mesh/meshblock.cpp:330-500), ``max_time_step``
(src/mesh/meshblock.cpp:511-529), ``forward(dt, stage)`` (advance_local,
src/mesh/meshblock.cpp:577-786) and ``check_redo``
(src/mesh/meshblock.cpp:974-1016).  dt lives on the device between the CFL
reduction and the stages, so a whole step can be captured in a CUDA graph.
"""
from __future__ import annotations

import ctypes

from . import _lib
from .config import CONSERVED, PRIMITIVE, SCALAR, HydroConfig, MeshBlockOptions


def conserved_totals(cfg, var, stream=None):
    """Compensated interior totals of var [nv, nc3, nc2, nc1] (FP64, device)
    times the cell volume, as a [nv] FP64 device tensor."""
    import torch

    L = _lib.lib()
    nv = int(var.shape[0])
    nb = L.snapb_totals_scratch_size(ctypes.byref(cfg), nv)
    scratch = torch.empty(nb, dtype=torch.uint8, device=var.device)
    out = torch.empty(nv, dtype=torch.float64, device=var.device)
    _lib.check(L.snapb_conserved_totals(ctypes.byref(cfg), _lib.ptr(var), nv, _lib.ptr(out),
                                        _lib.ptr(scratch), ctypes.c_size_t(nb),
                                        stream if stream is not None else _lib.stream_ptr()),
               "snapb_conserved_totals")
    return out


class MeshBlock:
    def __init__(self, options: MeshBlockOptions | HydroConfig, device=None):
        import torch

        if isinstance(options, HydroConfig):
            options = MeshBlockOptions(options)
        self.options = options
        self.cfg = options.hydro
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.type != "cuda":
            raise _lib.SnapbError("MeshBlock runs on CUDA devices only")
        self.lib = _lib.lib()
        c = self.cfg
        f64 = dict(dtype=torch.float64, device=self.device)
        self.hydro_u = torch.zeros(c.shape, **f64)
        self.hydro_w = torch.zeros(c.shape, **f64)
        self.hydro_u0 = torch.zeros(c.shape, **f64)
        ns = c.nscalar
        self.scalar_s = torch.zeros(c.scalar_shape, **f64) if ns else None
        self.scalar_s0 = torch.zeros(c.scalar_shape, **f64) if ns else None
        self.scalar_r = torch.zeros(c.scalar_shape, **f64) if ns else None
        nbytes = self.lib.snapb_workspace_size(ctypes.byref(c))
        if nbytes == 0:
            raise _lib.SnapbError("invalid configuration: " + self.lib.snapb_last_error().decode())
        self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        self.dt_raw = torch.zeros(1, **f64)   # CFL limit before the cfl factor
        self.dt = torch.zeros(1, **f64)       # the step's dt
        self.flags = torch.zeros(4, dtype=torch.int32, device=self.device)
        self.cycle = 0
        self.current_redo = 0

    # ---- helpers ----
    def _call(self, name, *args):
        rc = getattr(self.lib, name)(*args)
        _lib.check(rc, name)

    def _stream(self):
        return _lib.stream_ptr()

    def _ws(self):
        return _lib.ptr(self.workspace), ctypes.c_size_t(self.workspace.numel())

    # ---- MeshBlockImpl::initialize ----
    def initialize(self, hydro_w, scalar_r=None):
        """Primitive BCs on w, W->U, conserved BCs on u (and scalar_s = rho r)."""
        import torch

        c = self.cfg
        self.hydro_w.copy_(torch.as_tensor(hydro_w, dtype=torch.float64))
        st = self._stream()
        self._call("snapb_bc_apply", ctypes.byref(c), _lib.ptr(self.hydro_w), c.nvar, PRIMITIVE, st)
        if c.nscalar:
            if scalar_r is None:
                raise _lib.SnapbError("initialize: scalar_r is required for scalar model")
            self.scalar_r.copy_(torch.as_tensor(scalar_r, dtype=torch.float64))
            self._call("snapb_bc_apply", ctypes.byref(c), _lib.ptr(self.scalar_r), c.nscalar,
                       SCALAR, st)
        self._call("snapb_prim2cons", ctypes.byref(c), _lib.ptr(self.hydro_w),
                   _lib.ptr(self.hydro_u), st)
        if c.nscalar:
            self.scalar_s.copy_(self.hydro_w[0:1] * self.scalar_r)
        self._call("snapb_bc_apply", ctypes.byref(c), _lib.ptr(self.hydro_u), c.nvar, CONSERVED,
                   st)
        if c.nscalar:
            self._call("snapb_bc_apply", ctypes.byref(c), _lib.ptr(self.scalar_s), c.nscalar,
                       SCALAR, st)
        return 0.0

    # ---- MeshBlockImpl::max_time_step (device resident) ----
    def max_time_step(self):
        """dt = cfl * 2^-redo * CFL limit of hydro_w, left on the device."""
        c = self.cfg
        st = self._stream()
        ws, nb = self._ws()
        self._call("snapb_max_time_step", ctypes.byref(c), _lib.ptr(self.hydro_w),
                   _lib.ptr(self.dt_raw), ws, nb, st)
        self._call("snapb_scale_dt", _lib.ptr(self.dt_raw), ctypes.c_double(
            self.options.integration.cfl), self.current_redo, _lib.ptr(self.dt), st)
        return self.dt

    def set_dt(self, dt: float):
        self.dt.fill_(float(dt))
        return self.dt

    # ---- MeshBlockImpl::forward / advance_local ----
    def forward(self, stage: int, dt=None):
        if dt is not None and dt is not self.dt:
            self.set_dt(dt)
        c = self.cfg
        ws, nb = self._ws()
        self._call("snapb_stage", ctypes.byref(c), int(stage), _lib.ptr(self.dt),
                   _lib.ptr(self.hydro_u), _lib.ptr(self.hydro_u0), _lib.ptr(self.hydro_w),
                   _lib.ptr(self.scalar_s), _lib.ptr(self.scalar_s0), _lib.ptr(self.scalar_r),
                   ws, nb, self._stream())

    def step(self, dt=None):
        """One RK3 step (three stages); dt defaults to the device CFL value."""
        if dt is None:
            self.max_time_step()
        else:
            self.set_dt(dt)
        for s in range(3):
            self.forward(s)
        self.cycle += 1

    # ---- MeshBlockImpl::check_redo ----
    def check_redo(self) -> int:
        c = self.cfg
        self._call("snapb_check_positive", ctypes.byref(c), _lib.ptr(self.hydro_u),
                   _lib.ptr(self.flags), self._stream())
        f = self.flags.cpu().tolist()
        if f[0] or (f[1] and f[2]):
            self.current_redo += 1
            if self.current_redo > self.options.integration.max_redo:
                return -1
            self.hydro_u.copy_(self.hydro_u0)
            if c.nscalar:
                self.scalar_s.copy_(self.scalar_s0)
            st = self._stream()
            self._call("snapb_bc_apply", ctypes.byref(c), _lib.ptr(self.hydro_u), c.nvar,
                       CONSERVED, st)
            if c.nscalar:
                self._call("snapb_bc_apply", ctypes.byref(c), _lib.ptr(self.scalar_s),
                           c.nscalar, SCALAR, st)
            self.cycle -= 1  # the rejected step does not count (step() counted it)
            return 1
        self.current_redo = 0
        return 0

    # ---- restart files (snapy_linfel_b200/restart.py) ----
    def write_restart(self, output_dir, basename, file_number, current_time, rank=0,
                      final=False, output_file_numbers=(), output_next_times=()):
        """this block's restart part (RestartOutput::write_output_file)"""
        from . import restart

        v = {"hydro_u": self.hydro_u, "hydro_w": self.hydro_w, "scalar_s": self.scalar_s,
             "scalar_r": self.scalar_r}
        return restart.write_part(v, output_dir, basename, rank, file_number, current_time,
                                  self.cycle, final, output_file_numbers, output_next_times)

    def write_netcdf(self, output_dir, basename, file_number, current_time, file_id="out1",
                     variables=("prim",), rank=0, block_loc=(0, 0, 0), blocks=(1, 1, 1)):
        """this block's NetCDF output (NetcdfOutput::write_output_file,
        src/output/netcdf.cpp:34-508; snapy_linfel_b200/netcdf.py), the
        scalars written as mixing ratios with 'prim' and densities with
        'cons'"""
        from . import netcdf

        sc = None
        if self.cfg.nscalar:
            sc = self.scalar_s if "cons" in variables else self.scalar_r
        return netcdf.write_block(self.cfg, self.hydro_w, self.hydro_u, output_dir, basename,
                                  file_number, current_time, file_id, variables, rank,
                                  block_loc, blocks, sc)

    def restore(self, variables):
        """state from restart variables (restart.load_restart): hydro_u,
        hydro_w and scalar_s as stored (hydro_w derived from hydro_u when the
        file has none: it is the last stage's input primitive state, which the
        next CFL step reads), scalar_r = scalar_s / rho; returns the restart's
        last_time"""
        import torch

        c = self.cfg
        u = variables["hydro_u"]
        if tuple(u.shape) != tuple(c.shape):
            raise _lib.SnapbError(f"restart hydro_u has shape {tuple(u.shape)}, the block "
                                  f"{tuple(c.shape)}")
        self.hydro_u.copy_(u.to(self.device, torch.float64))
        if "hydro_w" in variables:
            self.hydro_w.copy_(variables["hydro_w"].to(self.device, torch.float64))
        else:
            self._call("snapb_cons2prim", ctypes.byref(c), _lib.ptr(self.hydro_u),
                       _lib.ptr(self.hydro_w), self._stream())
        if c.nscalar:
            self.scalar_s.copy_(variables["scalar_s"].to(self.device, torch.float64))
            self.scalar_r.copy_(self.scalar_s / self.hydro_u[0:1])
        if "last_cycle" in variables:
            self.cycle = int(variables["last_cycle"].reshape(-1)[0])
        return float(variables["last_time"].reshape(-1)[0]) if "last_time" in variables else 0.0

    # ---- diagnostics ----
    def interior(self, t):
        return t[(slice(None),) + self.cfg.interior()]

    def totals(self):
        """Domain totals of hydro_u * cell volume over the interior (mass0,
        momenta, energy; src/mesh/meshblock.cpp:855-870), compensated sums on
        the device: a [nvar] FP64 device tensor."""
        return conserved_totals(self.cfg, self.hydro_u, self._stream())


class MeshBlockF32:
    """The FP32 perturbation form of MeshBlock.

    hydro_u / hydro_w / scalar_* are FP32 perturbations about an FP64
    reference profile (rho_bar(x1), p_bar(x1)); by default the reference is
    the horizontal mean of the initial state.  ``state64()`` returns the FP64
    conserved state.  Same call sequence as MeshBlock.
    """

    def __init__(self, options: MeshBlockOptions | HydroConfig, device=None):
        import torch

        if isinstance(options, HydroConfig):
            options = MeshBlockOptions(options)
        self.options = options
        self.cfg = options.hydro
        self.device = torch.device(device if device is not None else "cuda")
        self.lib = _lib.lib()
        c = self.cfg
        nbytes = self.lib.snapb_workspace_size_f32(ctypes.byref(c))
        if nbytes == 0:
            raise _lib.SnapbError("configuration not supported by the FP32 form: " +
                                  self.lib.snapb_last_error().decode())
        f32 = dict(dtype=torch.float32, device=self.device)
        f64 = dict(dtype=torch.float64, device=self.device)
        self.hydro_u = torch.zeros(c.shape, **f32)
        self.hydro_u0 = torch.zeros(c.shape, **f32)
        self.hydro_w = torch.zeros(c.shape, **f32)
        ns = c.nscalar
        self.scalar_s = torch.zeros(c.scalar_shape, **f32) if ns else None
        self.scalar_s0 = torch.zeros(c.scalar_shape, **f32) if ns else None
        self.scalar_r = torch.zeros(c.scalar_shape, **f32) if ns else None
        self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        self.ref_rho = torch.zeros(c.nc1, **f64)
        self.ref_p = torch.zeros(c.nc1, **f64)
        self.dt_raw = torch.zeros(1, **f64)
        self.dt = torch.zeros(1, **f64)
        self.cycle = 0
        self.current_redo = 0

    def _call(self, name, *args):
        _lib.check(getattr(self.lib, name)(*args), name)

    def _ws(self):
        return _lib.ptr(self.workspace), ctypes.c_size_t(self.workspace.numel())

    def initialize(self, hydro_w, scalar_r=None, reference="mean"):
        """reference: "mean" (horizontal mean of the initial state at each x1
        level, ghosts included), None (zero reference: plain FP32), or a pair
        (rho_bar, p_bar) of [nc1] arrays."""
        import torch

        c = self.cfg
        st = _lib.stream_ptr()
        w64 = torch.as_tensor(hydro_w, dtype=torch.float64).to(self.device).contiguous()
        self._call("snapb_bc_apply", ctypes.byref(c), _lib.ptr(w64), c.nvar, PRIMITIVE, st)
        it = self.cfg.interior()
        ws, nb = self._ws()
        if reference is None:
            self.ref_rho.zero_()
            self.ref_p.zero_()
            self._call("snapb_reference_f32", ctypes.byref(c), None, None, ws, nb, st)
        else:
            if isinstance(reference, str) and reference == "mean":
                ref_rho = w64[0][it[0], it[1], :].mean(dim=(0, 1))
                ref_p = w64[4][it[0], it[1], :].mean(dim=(0, 1))
            else:
                ref_rho, ref_p = reference
            self.ref_rho.copy_(torch.as_tensor(ref_rho, dtype=torch.float64))
            self.ref_p.copy_(torch.as_tensor(ref_p, dtype=torch.float64))
            self._call("snapb_reference_f32", ctypes.byref(c), _lib.ptr(self.ref_rho),
                       _lib.ptr(self.ref_p), ws, nb, st)
        u64 = torch.empty_like(w64)
        self._call("snapb_prim2cons", ctypes.byref(c), _lib.ptr(w64), _lib.ptr(u64), st)
        s64 = None
        if c.nscalar:
            r64 = torch.as_tensor(scalar_r, dtype=torch.float64).to(self.device).contiguous()
            self._call("snapb_bc_apply", ctypes.byref(c), _lib.ptr(r64), c.nscalar, SCALAR, st)
            s64 = (w64[0:1] * r64).contiguous()
            self._call("snapb_bc_apply", ctypes.byref(c), _lib.ptr(s64), c.nscalar, SCALAR, st)
            self.scalar_s.copy_(s64)
            self.scalar_r.copy_(r64)
        self._call("snapb_bc_apply", ctypes.byref(c), _lib.ptr(u64), c.nvar, CONSERVED, st)
        self._call("snapb_to_perturbation", ctypes.byref(c), CONSERVED, _lib.ptr(u64),
                   _lib.ptr(self.hydro_u), ws, nb, st)
        self._call("snapb_to_perturbation", ctypes.byref(c), PRIMITIVE, _lib.ptr(w64),
                   _lib.ptr(self.hydro_w), ws, nb, st)
        return 0.0

    def max_time_step(self):
        c = self.cfg
        st = _lib.stream_ptr()
        ws, nb = self._ws()
        self._call("snapb_max_time_step_f32", ctypes.byref(c), _lib.ptr(self.hydro_w),
                   _lib.ptr(self.dt_raw), ws, nb, st)
        self._call("snapb_scale_dt", _lib.ptr(self.dt_raw),
                   ctypes.c_double(self.options.integration.cfl), self.current_redo,
                   _lib.ptr(self.dt), st)
        return self.dt

    def set_dt(self, dt: float):
        self.dt.fill_(float(dt))
        return self.dt

    def forward(self, stage: int, dt=None):
        if dt is not None and dt is not self.dt:
            self.set_dt(dt)
        c = self.cfg
        ws, nb = self._ws()
        self._call("snapb_stage_f32", ctypes.byref(c), int(stage), _lib.ptr(self.dt),
                   _lib.ptr(self.hydro_u), _lib.ptr(self.hydro_u0), _lib.ptr(self.hydro_w),
                   _lib.ptr(self.scalar_s), _lib.ptr(self.scalar_s0), _lib.ptr(self.scalar_r),
                   ws, nb, _lib.stream_ptr())

    def step(self, dt=None):
        if dt is None:
            self.max_time_step()
        else:
            self.set_dt(dt)
        for s in range(3):
            self.forward(s)
        self.cycle += 1

    def totals(self):
        """Domain totals of the full conserved state (u_bar + u') * cell volume
        over the interior, compensated sums of the FP32 perturbations plus
        the FP64 reference: a [nvar] FP64 device tensor."""
        import torch

        c = self.cfg
        L = _lib.lib()
        nb = L.snapb_totals_scratch_size(ctypes.byref(c), c.nvar)
        scratch = torch.empty(nb, dtype=torch.uint8, device=self.device)
        out = torch.empty(c.nvar, dtype=torch.float64, device=self.device)
        ws, wb = self._ws()
        self._call("snapb_conserved_totals_f32", ctypes.byref(c), _lib.ptr(self.hydro_u),
                   c.nvar, _lib.ptr(out), ws, wb, _lib.ptr(scratch), ctypes.c_size_t(nb),
                   _lib.stream_ptr())
        return out

    def state64(self):
        """FP64 conserved state u = u_bar + u'."""
        import torch

        c = self.cfg
        out = torch.empty(c.shape, dtype=torch.float64, device=self.device)
        ws, nb = self._ws()
        self._call("snapb_from_perturbation", ctypes.byref(c), CONSERVED, _lib.ptr(self.hydro_u),
                   _lib.ptr(out), ws, nb, _lib.stream_ptr())
        return out

    def interior(self, t):
        return t[(slice(None),) + self.cfg.interior()]
