"""The implicit correction that allocates nothing, checked against the
workspace entry point it mirrors.

Callers that cannot allocate device memory at the point where they run the
column solve (a CUDA-graph capture in progress, a pre-partitioned device
heap, a binding with no allocator) use snapb_implicit_correction_noalloc; its
scratch is a fixed array inside the library.  This file is collected last so
that a run stopping at the first failure has run every other test first.
It must pass alone in a fresh process too, so it builds its own inputs.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _setup(scheme, nx2=40, nx1=24):
    from snapy_linfel_b200 import _lib as L
    from snapy_linfel_b200 import problems

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    opts, w, _ = problems.straka(nx2=nx2, nx1=nx1, implicit_scheme=scheme)
    c = opts.hydro
    lib = L.lib()
    st = L.stream_ptr()
    # inputs from the CUDA path itself: hydro_w with revised ghosts and an
    # explicit stage tendency (implicit scheme switched off for that call)
    wg = torch.from_numpy(w).cuda()
    ug = torch.empty_like(wg)
    L.check(lib.snapb_bc_apply(ctypes.byref(c), L.ptr(wg), 5, 0, st), "bc")
    L.check(lib.snapb_prim2cons(ctypes.byref(c), L.ptr(wg), L.ptr(ug), st), "prim2cons")
    L.check(lib.snapb_bc_apply(ctypes.byref(c), L.ptr(ug), 5, 1, st), "bc")
    cexp = c.copy()
    cexp.implicit_scheme = 0
    ws = torch.empty(lib.snapb_workspace_size(ctypes.byref(c)), dtype=torch.uint8, device="cuda")
    du = torch.empty_like(ug)
    dt = torch.tensor([2.0], dtype=torch.float64, device="cuda")
    L.check(lib.snapb_hydro_forward(ctypes.byref(cexp), L.ptr(dt), L.ptr(ug), L.ptr(wg), L.ptr(du),
                                    None, L.ptr(ws), ctypes.c_size_t(ws.numel()), st), "forward")
    torch.cuda.synchronize()
    return L, lib, c, ug, wg, du, ws, dt


def _state_err(a, b, u):
    """largest per-variable error relative to the state's magnitude; any
    non-finite value in either operand fails (it is never dropped by the
    reduction)"""
    assert bool(torch.isfinite(a).all()) and bool(torch.isfinite(b).all()), "non-finite"
    rho = u[0].abs().max()
    en = u[4].abs().max()
    mom = torch.maximum((rho * en).sqrt(), u[1:4].abs().max())
    scale = torch.stack([rho, mom, mom, mom, en])
    err = (a - b).abs().reshape(5, -1).amax(dim=1) / scale
    return float(err.max())


@pytest.mark.parametrize("scheme", [1, 9])
def test_noalloc_matches_workspace_entry_point_twice(scheme):
    L, lib, c, ug, wg, du, ws, dt = _setup(scheme)
    st = L.stream_ptr()
    it = (slice(None),) + c.interior()
    # two calls in a row with different inputs; the second one also checks
    # that nothing of the first call leaks through the shared scratch
    for k, scale in enumerate((1.0, 0.5)):
        du_in = du * scale
        ref, out = du_in.clone(), du_in.clone()
        m_ref = torch.zeros_like(ug)
        m_out = torch.zeros_like(ug)
        L.check(lib.snapb_implicit_correction(ctypes.byref(c), L.ptr(dt), L.ptr(ref), L.ptr(wg),
                                              L.ptr(m_ref), L.ptr(ws), ctypes.c_size_t(ws.numel()),
                                              st), "implicit_correction")
        L.check(lib.snapb_implicit_correction_noalloc(ctypes.byref(c), L.ptr(dt), L.ptr(out),
                                                      L.ptr(wg), L.ptr(m_out), st),
                "implicit_correction_noalloc")
        torch.cuda.synchronize()
        assert _state_err(out[it], ref[it], ug[it]) < 1e-12, k
        assert bool(torch.isfinite(m_out[0]).all()) and bool(torch.isfinite(m_ref[0]).all())
        assert (m_out[0] - m_ref[0]).abs().max().item() / ug[0].abs().max().item() < 1e-12
        assert not torch.equal(out[it], du_in[it])  # the solve did change du


def test_noalloc_rejects_oversize_problem():
    from snapy_linfel_b200 import _lib as L
    from snapy_linfel_b200.config import make_config

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    # 192 layers x 512 x 512 columns needs far more than the built-in 32 MiB
    c = make_config(nx1=192, nx2=512, nx3=512, implicit_scheme=1, grav=(-9.8, 0.0, 0.0))
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = L.lib().snapb_implicit_correction_noalloc(ctypes.byref(c), L.ptr(dummy), L.ptr(dummy),
                                                   L.ptr(dummy), None, L.stream_ptr())
    assert rc == 1
    assert b"built-in buffer" in L.lib().snapb_last_error()
