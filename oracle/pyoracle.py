"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loaded by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
to check or time the CUDA product path; the product never imports it.

``Oracle(kind="port")`` loads ``oracle/liboracle.so`` (the restated kernels),
``Oracle(kind="reference")`` loads ``oracle/_ref/libsnapref.so`` (same
orchestration, point kernels compiled from the reference's own ``*_impl.h``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "need C-contiguous float64"
    return a.ctypes.data_as(_dp)


def lib_path(kind: str = "port") -> str:
    if kind == "port":
        return os.path.join(HERE, "liboracle.so")
    if kind == "reference":
        return os.path.join(HERE, "_ref", "libsnapref.so")
    raise ValueError(kind)


def build(kind: str = "port", ref: str | None = None) -> str:
    """Build the oracle library with its Makefile if it is missing."""
    path = lib_path(kind)
    target = "liboracle.so" if kind == "port" else "ref"
    cmd = ["make", "-s", "-C", HERE, target]
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True)
    return path


class Oracle:
    def __init__(self, kind: str = "port"):
        from snapy_linfel_b200.config import HydroConfig  # struct layout only

        self.kind = kind
        path = lib_path(kind)
        if not os.path.exists(path):
            if kind == "reference":
                raise FileNotFoundError(f"{path} not built (needs the reference sources)")
            build(kind)
        self.lib = L = ctypes.CDLL(path)
        self.Config = HydroConfig
        cp = ctypes.POINTER(HydroConfig)
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_kernels_kind.restype = ctypes.c_int
        L.orc_interp_point.restype = ctypes.c_double
        L.orc_interp_point.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int]
        for name in ("orc_cons2prim", "orc_prim2cons"):
            getattr(L, name).argtypes = [cp, _dp, _dp]
        L.orc_reconstruct.argtypes = [cp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp]
        L.orc_riemann.argtypes = [cp, ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int,
                                  _dp, _dp, _dp]
        L.orc_bc_apply.argtypes = [cp, _dp, ctypes.c_int, ctypes.c_int]
        L.orc_max_time_step.restype = ctypes.c_double
        L.orc_max_time_step.argtypes = [cp, _dp]
        L.orc_block_create.restype = ctypes.c_void_p
        L.orc_block_create.argtypes = [cp]
        L.orc_block_destroy.argtypes = [ctypes.c_void_p]
        L.orc_hydro_forward.argtypes = [ctypes.c_void_p, ctypes.c_double, _dp, _dp, _dp, _dp]
        L.orc_stage.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp, _dp,
                                _dp, _dp, _dp, _dp]
        L.orc_block_flux.restype = _dp
        L.orc_block_flux.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_implicit_correction.argtypes = [cp, ctypes.c_double, _dp, _dp, _dp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        L.orc_vic_redistribute.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_int]

    # -- helpers ----------------------------------------------------------
    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.orc_last_error().decode())

    def set_threads(self, n: int):
        self.lib.orc_set_threads(int(n))

    def threads(self) -> int:
        return self.lib.orc_get_threads()

    # -- point level --------------------------------------------------------
    def interp_point(self, rtype: int, side: int, window, scale=False) -> float:
        win = np.ascontiguousarray(window, dtype=np.float64)
        return self.lib.orc_interp_point(rtype, side, _ptr(win), int(scale))

    # -- array level --------------------------------------------------------
    def cons2prim(self, cfg, u):
        w = np.empty_like(u)
        self._check(self.lib.orc_cons2prim(ctypes.byref(cfg), _ptr(u), _ptr(w)))
        return w

    def prim2cons(self, cfg, w):
        u = np.empty_like(w)
        self._check(self.lib.orc_prim2cons(ctypes.byref(cfg), _ptr(w), _ptr(u)))
        return u

    def reconstruct(self, cfg, dim, group, w):
        nv = w.shape[0]
        wlr = np.empty((2,) + w.shape)
        self._check(self.lib.orc_reconstruct(ctypes.byref(cfg), dim, group, _ptr(w), nv,
                                             _ptr(wlr)))
        return wlr

    def riemann(self, cfg, solver, dim, wl, wr, vel=None, face_pressure=True):
        nv = wl.shape[0]
        flx = np.empty_like(wl)
        fp = np.empty(wl.shape[1:]) if face_pressure else None
        self._check(self.lib.orc_riemann(ctypes.byref(cfg), solver, dim, _ptr(wl), _ptr(wr),
                                         nv, _ptr(flx), _ptr(fp), _ptr(vel)))
        return flx, fp

    def bc_apply(self, cfg, var, kind):
        self._check(self.lib.orc_bc_apply(ctypes.byref(cfg), _ptr(var), var.shape[0], kind))
        return var

    def max_time_step(self, cfg, w) -> float:
        return self.lib.orc_max_time_step(ctypes.byref(cfg), _ptr(w))

    def implicit_correction(self, cfg, dt, du, w, mass=None):
        self._check(self.lib.orc_implicit_correction(ctypes.byref(cfg), dt, _ptr(du), _ptr(w),
                                                     _ptr(mass)))
        return du

    def vic_redistribute(self, du, w, mass, delta, vol, nlayer, n_hydro, ny, nblock):
        self.lib.orc_vic_redistribute(_ptr(du), _ptr(w), _ptr(mass), _ptr(delta), _ptr(vol),
                                      nlayer, n_hydro, ny, nblock)

    def block(self, cfg):
        return OracleBlock(self, cfg)


class OracleBlock:
    """Module buffers of one mesh block (F1..F3, mass_corr) kept across calls."""

    def __init__(self, orc: Oracle, cfg):
        self.orc = orc
        self.cfg = cfg
        self.h = orc.lib.orc_block_create(ctypes.byref(cfg))
        if not self.h:
            raise RuntimeError(orc.lib.orc_last_error().decode())

    def __del__(self):
        try:
            self.orc.lib.orc_block_destroy(self.h)
        except Exception:
            pass

    def hydro_forward(self, dt, u, w, mass_corr=None):
        du = np.empty_like(u)
        self.orc._check(self.orc.lib.orc_hydro_forward(self.h, dt, _ptr(u), _ptr(w), _ptr(du),
                                                       _ptr(mass_corr)))
        return du

    def stage(self, stage, dt, u, u0, w, s=None, s0=None, r=None):
        self.orc._check(self.orc.lib.orc_stage(self.h, stage, dt, _ptr(u), _ptr(u0), _ptr(w),
                                               _ptr(s), _ptr(s0), _ptr(r)))

    def flux(self, axis, shape):
        p = self.orc.lib.orc_block_flux(self.h, axis)
        if not p:
            return None
        n = int(np.prod(shape))
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(shape).copy()
