"""ctypes binding of ``libsnapb.so`` (the C ABI in include/snapb.h).

The library is built in-tree by ``snapy_linfel_b200.build``.  There is no
fallback: if the shared library is missing or a call fails, a
``SnapbError`` is raised.
"""
from __future__ import annotations

import ctypes
import os

from .config import HydroConfig

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsnapb.so")

OK = 0


class SnapbError(RuntimeError):
    pass


_lib = None


def lib():
    """Load libsnapb.so once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise SnapbError(f"{LIB_PATH} is missing: run `python -m snapy_linfel_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    cp = ctypes.POINTER(HydroConfig)
    vp = ctypes.c_void_p
    sz = ctypes.c_size_t
    i = ctypes.c_int
    d = ctypes.c_double
    sig = {
        "snapb_abi_version": (i, []),
        "snapb_last_error": (ctypes.c_char_p, []),
        "snapb_workspace_size": (sz, [cp]),
        "snapb_cons2prim": (i, [cp, vp, vp, vp]),
        "snapb_prim2cons": (i, [cp, vp, vp, vp]),
        "snapb_reconstruct": (i, [cp, i, i, vp, i, vp, vp]),
        "snapb_riemann": (i, [cp, i, i, vp, vp, i, vp, vp, vp, vp]),
        "snapb_hydro_forward": (i, [cp, vp, vp, vp, vp, vp, vp, sz, vp]),
        "snapb_stage": (i, [cp, i, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]),
        "snapb_implicit_correction": (i, [cp, vp, vp, vp, vp, vp, sz, vp]),
        "snapb_implicit_correction_noalloc": (i, [cp, vp, vp, vp, vp, vp]),
        "snapb_bc_apply": (i, [cp, vp, i, i, vp]),
        "snapb_max_time_step": (i, [cp, vp, vp, vp, sz, vp]),
        "snapb_scale_dt": (i, [vp, d, i, vp, vp]),
        "snapb_check_positive": (i, [cp, vp, vp, vp]),
        "snapb_pack_slab": (i, [cp, i, i, i, vp, i, vp, vp]),
        "snapb_unpack_slab": (i, [cp, i, i, i, vp, i, vp, vp]),
        "snapb_workspace_size_f32": (sz, [cp]),
        "snapb_reference_f32": (i, [cp, vp, vp, vp, sz, vp]),
        "snapb_to_perturbation": (i, [cp, i, vp, vp, vp, sz, vp]),
        "snapb_from_perturbation": (i, [cp, i, vp, vp, vp, sz, vp]),
        "snapb_stage_f32": (i, [cp, i, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]),
        "snapb_bc_apply_f32": (i, [cp, vp, i, i, vp, sz, vp]),
        "snapb_max_time_step_f32": (i, [cp, vp, vp, vp, sz, vp]),
        "snapb_adjoint_workspace_size": (sz, [cp]),
        "snapb_stage_adjoint": (i, [cp, i, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]),
        "snapb_hydro_forward_adjoint": (i, [cp, vp, vp, vp, vp, vp, sz, vp]),
        "snapb_bc_adjoint": (i, [cp, vp, vp, i, i, vp]),
        "snapb_riemann_adjoint": (i, [cp, i, i, vp, vp, vp, vp, vp, vp]),
        "snapb_ensemble_create": (i, [vp, i, vp, ctypes.POINTER(vp)]),
        "snapb_ensemble_workspace_size": (sz, [vp]),
        "snapb_ensemble_bind": (i, [vp, vp, sz, vp]),
        "snapb_ensemble_set_tuning": (i, [vp, vp, vp]),
        "snapb_ensemble_dt": (vp, [vp]),
        "snapb_ensemble_max_time_step_f32": (i, [vp, d, vp]),
        "snapb_ensemble_stage_f32": (i, [vp, i, vp]),
        "snapb_ensemble_destroy": (None, [vp]),
        "snapb_totals_scratch_size": (sz, [cp, i]),
        "snapb_conserved_totals": (i, [cp, vp, i, vp, vp, sz, vp]),
        "snapb_conserved_totals_f32": (i, [cp, vp, i, vp, vp, sz, vp, sz, vp]),
        "snapb_timing_enable": (i, [i]),
        "snapb_timing_query": (i, [i, ctypes.POINTER(d), ctypes.POINTER(i)]),
        "snapb_bulk_copy_timeouts": (i, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def exported_symbols():
    """Names of the entry points this binding declares (all in snapb.h)."""
    return ["snapb_abi_version", "snapb_last_error", "snapb_workspace_size", "snapb_cons2prim",
            "snapb_prim2cons", "snapb_reconstruct", "snapb_riemann", "snapb_hydro_forward",
            "snapb_implicit_correction", "snapb_implicit_correction_noalloc", "snapb_stage",
            "snapb_bc_apply", "snapb_max_time_step", "snapb_scale_dt",
            "snapb_check_positive", "snapb_pack_slab", "snapb_unpack_slab",
            "snapb_timing_enable", "snapb_timing_query", "snapb_bulk_copy_timeouts",
            "snapb_workspace_size_f32", "snapb_reference_f32", "snapb_to_perturbation",
            "snapb_from_perturbation", "snapb_stage_f32", "snapb_bc_apply_f32",
            "snapb_max_time_step_f32", "snapb_adjoint_workspace_size", "snapb_stage_adjoint",
            "snapb_hydro_forward_adjoint", "snapb_bc_adjoint", "snapb_riemann_adjoint",
            "snapb_ensemble_create",
            "snapb_ensemble_workspace_size", "snapb_ensemble_bind", "snapb_ensemble_set_tuning",
            "snapb_ensemble_dt", "snapb_ensemble_max_time_step_f32", "snapb_ensemble_stage_f32",
            "snapb_ensemble_destroy", "snapb_totals_scratch_size", "snapb_conserved_totals",
            "snapb_conserved_totals_f32"]


KERNELS = {"x1_sweep": 0, "diffusion": 1, "x2_sweep": 2, "x3_sweep": 3, "finalize": 4,
           "implicit_vic": 5, "boundary": 6, "adj_combine": 7, "adj_recompute": 8,
           "adj_vic": 9, "adj_x2x3": 10, "adj_x1": 11}


def timing_enable(on: bool = True):
    check(lib().snapb_timing_enable(1 if on else 0), "snapb_timing_enable")


def timing_query():
    """{kernel name: (total ms, launches)} of the recorded launches."""
    out = {}
    for name, k in KERNELS.items():
        ms = ctypes.c_double(0.0)
        n = ctypes.c_int(0)
        check(lib().snapb_timing_query(k, ctypes.byref(ms), ctypes.byref(n)),
              "snapb_timing_query")
        if n.value:
            out[name] = (ms.value, n.value)
    return out


def check(rc: int, what: str = "snapb"):
    if rc != OK:
        msg = lib().snapb_last_error().decode()
        raise SnapbError(f"{what} failed ({rc}): {msg}")


def ptr(t):
    """Device pointer of a CUDA tensor (None passes NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise SnapbError("snapb entry points take CUDA tensors")
    if not t.is_contiguous():
        raise SnapbError("snapb entry points take contiguous tensors")
    return ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
