"""GPU parity of the CUDA path (through the C ABI) against the CPU oracle.

Tolerances: integer/index work (boundary fills) is compared bit for bit.
Single operators (EOS, reconstruction, Riemann fluxes, CFL) are compared by
the per-field relative max error max|gpu - oracle| / max|oracle| (1e-13 /
1e-12, bound at each call).  Step results are compared "relative per step"
as the FP64 target states it: the error in the state change is divided by
the magnitude of the state itself (density, energy, sqrt(rho E) for the
momenta, the scalar's own range), bound 1e-12 per step.  A tendency that is
a cancellation of large fluxes (e.g. du[IVY] of a horizontally uniform
pressure, exactly 0 on the CPU and ~1e-15 on the GPU) is measured against the
state it changes, not against its own near-zero size.
"""
import ctypes

import numpy as np
import pytest

from snapy_linfel_b200 import problems
from snapy_linfel_b200.config import CONSERVED, PRIMITIVE, SCALAR, make_config

from errnorm import assert_finite, relerr, state_err, state_scale  # noqa: F401

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from snapy_linfel_b200 import _lib

    return _lib


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def random_prim(rng, shape):
    w = rng.random(shape)
    w[0] += 1.0
    w[4] += 1.0
    w[1:4] = (w[1:4] - 0.5) * 0.1
    return w


def call(L, name, *args):
    rc = getattr(L.lib(), name)(*args)
    L.check(rc, name)
    torch.cuda.synchronize()


# ---------------------------------------------------------------- EOS ----
def test_eos_roundtrip(L, oracle):
    rng = np.random.default_rng(1)
    c = make_config(nx1=12, nx2=9, nx3=7)
    w = random_prim(rng, c.shape)
    u_ref = oracle.prim2cons(c, w)
    wg, ug = dev(w), torch.empty(c.shape, dtype=torch.float64, device="cuda")
    call(L, "snapb_prim2cons", ctypes.byref(c), L.ptr(wg), L.ptr(ug), L.stream_ptr())
    assert relerr(ug.cpu().numpy(), u_ref) < 1e-14
    w2 = torch.empty_like(ug)
    call(L, "snapb_cons2prim", ctypes.byref(c), L.ptr(ug), L.ptr(w2), L.stream_ptr())
    assert relerr(w2.cpu().numpy(), oracle.cons2prim(c, u_ref)) < 1e-13


# ------------------------------------------------------ reconstruction ----
@pytest.mark.parametrize("rtype", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("shock", [0, 1])
def test_reconstruct_matches_oracle(L, oracle, rtype, shock):
    rng = np.random.default_rng(10 + rtype)
    c = make_config(nx1=11, nx2=8, nx3=6)
    c.recon1_type = c.recon23_type = rtype
    c.recon1_shock = c.recon23_shock = shock
    w = random_prim(rng, c.shape)
    wg = dev(w)
    for dim in (3, 2, 1):
        ref = oracle.reconstruct(c, dim, 0, w)
        out = torch.empty((2,) + c.shape, dtype=torch.float64, device="cuda")
        call(L, "snapb_reconstruct", ctypes.byref(c), dim, 0, L.ptr(wg), 5, L.ptr(out),
             L.stream_ptr())
        got = out.cpu().numpy()
        for side in (0, 1):
            assert relerr(got[side], ref[side]) < 1e-13, (dim, side)


def test_reconstruct_scale_and_scalars(L, oracle):
    rng = np.random.default_rng(3)
    c = make_config(nx1=10, nx2=8, nx3=7)
    c.recon1_type = c.recon23_type = 5
    c.recon1_scale = c.recon23_scale = 1
    c.scalar_recon_type = 5
    w = random_prim(rng, c.shape)
    sc = rng.random((2,) + c.shape[1:]) - 0.3
    for group, arr, nv in ((0, w, 5), (1, sc, 2)):
        g = dev(arr)
        for dim in (3, 2, 1):
            ref = oracle.reconstruct(c, dim, group, arr)
            out = torch.empty((2,) + arr.shape, dtype=torch.float64, device="cuda")
            call(L, "snapb_reconstruct", ctypes.byref(c), dim, group, L.ptr(g), nv, L.ptr(out),
                 L.stream_ptr())
            assert relerr(out.cpu().numpy()[0], ref[0]) < 1e-13
            assert relerr(out.cpu().numpy()[1], ref[1]) < 1e-13


# ------------------------------------------------------------- Riemann ----
@pytest.mark.parametrize("solver", [0, 1, 2])
def test_riemann_matches_oracle(L, oracle, solver):
    rng = np.random.default_rng(20 + solver)
    c = make_config(nx1=10, nx2=8, nx3=6)
    wl, wr = random_prim(rng, c.shape), random_prim(rng, c.shape)
    # a few faces with strong jumps exercise the branch selections (and Roe's LLF switch)
    wr[0, :, :, ::3] *= 8.0
    wr[1, :, :, ::4] += 2.0
    wr[4, :, :, 1::5] *= 20.0
    for dim in (3, 2, 1):
        ref_f, ref_p = oracle.riemann(c, solver, dim, wl, wr)
        f = torch.empty(c.shape, dtype=torch.float64, device="cuda")
        p = torch.empty(c.shape[1:], dtype=torch.float64, device="cuda")
        gl, gr = dev(wl), dev(wr)  # keep the inputs alive across the launch
        call(L, "snapb_riemann", ctypes.byref(c), solver, dim, L.ptr(gl), L.ptr(gr), 5,
             L.ptr(f), L.ptr(p), None, L.stream_ptr())
        assert relerr(f.cpu().numpy(), ref_f) < 1e-12, dim
        assert relerr(p.cpu().numpy(), ref_p) < 1e-13, dim


def test_riemann_upwind(L, oracle):
    rng = np.random.default_rng(5)
    c = make_config(nx1=10, nx2=8, nx3=6)
    wl, wr = rng.random((2,) + c.shape[1:]), rng.random((2,) + c.shape[1:])
    vel = rng.standard_normal(c.shape[1:])
    ref, _ = oracle.riemann(c, 3, 3, wl, wr, vel=vel, face_pressure=False)
    f = torch.empty((2,) + c.shape[1:], dtype=torch.float64, device="cuda")
    gl, gr, gv = dev(wl), dev(wr), dev(vel)
    call(L, "snapb_riemann", ctypes.byref(c), 3, 3, L.ptr(gl), L.ptr(gr), 2, L.ptr(f), None,
         L.ptr(gv), L.stream_ptr())
    np.testing.assert_array_equal(f.cpu().numpy(), ref)


# ------------------------------------------------------ boundary fills ----
BC_SETS = [
    ("reflecting",) * 6,
    ("outflow",) * 6,
    ("periodic",) * 6,
    ("reflecting", "outflow", "periodic", "periodic", "outflow", "reflecting"),
    ("custom", "reflecting", "outflow", "custom", "periodic", "periodic"),
]


@pytest.mark.parametrize("bcs", BC_SETS)
@pytest.mark.parametrize("kind", [PRIMITIVE, CONSERVED, SCALAR])
def test_bc_bit_exact(L, oracle, bcs, kind):
    rng = np.random.default_rng(7)
    c = make_config(nx1=7, nx2=6, nx3=5, bc=bcs)
    var = rng.standard_normal(c.shape)
    ref = oracle.bc_apply(c, var.copy(), kind)
    g = dev(var)
    call(L, "snapb_bc_apply", ctypes.byref(c), L.ptr(g), 5, kind, L.stream_ptr())
    np.testing.assert_array_equal(g.cpu().numpy(), ref)


def test_bc_bit_exact_2d_1d(L, oracle):
    rng = np.random.default_rng(8)
    for kw in (dict(nx1=9, nx2=6), dict(nx1=9), dict(nx1=5, nx3=4)):
        c = make_config(bc=("reflecting", "periodic", "outflow", "reflecting", "periodic",
                            "outflow"), **kw)
        var = rng.standard_normal(c.shape)
        ref = oracle.bc_apply(c, var.copy(), CONSERVED)
        g = dev(var)
        call(L, "snapb_bc_apply", ctypes.byref(c), L.ptr(g), 5, CONSERVED, L.stream_ptr())
        np.testing.assert_array_equal(g.cpu().numpy(), ref)


# ---------------------------------------------------------------- CFL ----
@pytest.mark.parametrize("scheme", [0, 1])
def test_max_time_step(L, oracle, scheme):
    opts, w, _ = problems.straka(nx2=64, nx1=24, implicit_scheme=scheme)
    c = opts.hydro
    oracle.bc_apply(c, w, PRIMITIVE)
    w[1] += 3.0 * np.sin(np.arange(w.shape[-1]))[None, None, :]
    ref = oracle.max_time_step(c, w)
    ws = torch.empty(L.lib().snapb_workspace_size(ctypes.byref(c)), dtype=torch.uint8,
                     device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    wg = dev(w)
    call(L, "snapb_max_time_step", ctypes.byref(c), L.ptr(wg), L.ptr(out), L.ptr(ws),
         ctypes.c_size_t(ws.numel()), L.stream_ptr())
    assert abs(out.item() / ref - 1) < 1e-14


# ------------------------------------------------- hydro forward (du) ----
def _forward_case(L, oracle, opts, w, dt):
    c = opts.hydro
    oracle.bc_apply(c, w, PRIMITIVE)
    u = oracle.prim2cons(c, w)
    oracle.bc_apply(c, u, CONSERVED)
    blk = oracle.block(c)
    w_ref = np.empty_like(u)
    mass_ref = np.zeros_like(u)
    du_ref = blk.hydro_forward(dt, u, w_ref, mass_ref)
    ws = torch.empty(L.lib().snapb_workspace_size(ctypes.byref(c)), dtype=torch.uint8,
                     device="cuda")
    ug, wg = dev(u), torch.empty(c.shape, dtype=torch.float64, device="cuda")
    dug = torch.empty_like(wg)
    mg = torch.empty_like(wg)
    dtg = torch.tensor([dt], dtype=torch.float64, device="cuda")
    call(L, "snapb_hydro_forward", ctypes.byref(c), L.ptr(dtg), L.ptr(ug), L.ptr(wg), L.ptr(dug),
         L.ptr(mg), L.ptr(ws), ctypes.c_size_t(ws.numel()), L.stream_ptr())
    it = (slice(None),) + c.interior()
    du = dug.cpu().numpy()
    # w is compared everywhere (ghosts carry the hydrostatic revision)
    assert relerr(wg.cpu().numpy(), w_ref) < 1e-13
    # du: error of the state change relative to the state (per step)
    err = state_err(du[it], du_ref[it], u[it])
    return err, du[it], du_ref[it], mg.cpu().numpy()[it], mass_ref[it], u[it]


def test_forward_sod(L, oracle):
    opts, w, _ = problems.sod(nx1=256)
    err, *_ = _forward_case(L, oracle, opts, w, 1e-3)
    assert err < 1e-12


@pytest.mark.parametrize("variant", ["column", "fused"])
def test_steps_3d_scalars_implicit_both_variants(L, oracle, variant, monkeypatch):
    """three steps of a 3-D Roe domain with two tracers and VIC 3x3 through
    either implicit-solve variant, against the oracle"""
    if variant == "fused":
        monkeypatch.setenv("SNAPB_VIC_KERNEL", "fused")
    opts, w, r = problems.large_3d(nx3=10, nx2=12, nx1=16, nscalar=2)
    dts = [0.5, 0.5, 0.5]
    mb, _ = _run_gpu(opts, w, r, 3, dts=dts)
    u_ref, s_ref, _ = _run_oracle(oracle, opts, w, r, 3, dts=dts)
    it = (slice(None),) + opts.hydro.interior()
    assert state_err(mb.hydro_u.cpu().numpy()[it], u_ref[it], u_ref[it]) < 1e-12 * 3
    s = mb.scalar_s.cpu().numpy()[it]
    assert_finite(s)
    assert np.max(np.abs(s - s_ref[it])) / np.max(np.abs(s_ref[it])) < 1e-12 * 3


@pytest.mark.parametrize("riemann", ["lmars", "hllc", "roe"])
@pytest.mark.parametrize("scheme", [0, 1, 9])
def test_forward_straka(L, oracle, riemann, scheme):
    opts, w, _ = problems.straka(nx2=48, nx1=20, implicit_scheme=scheme, riemann=riemann)
    err, du, du_ref, m, m_ref, u = _forward_case(L, oracle, opts, w, 0.5)
    assert err < 1e-12, err
    if scheme:
        # implicit mass fix, relative to the density it corrects
        assert np.max(np.abs(m[0] - m_ref[0])) / np.max(np.abs(u[0])) < 1e-12


def test_forward_3d_roe_periodic(L, oracle):
    opts, w, _ = problems.warm_bubble_3d(10, 12, 16, amp=2.0, radius=600.0,
                                          center=(500.0, 600.0, 600.0), riemann="roe",
                                          implicit_scheme=0)
    err, *_ = _forward_case(L, oracle, opts, w, 0.2)
    assert err < 1e-12


def test_forward_variants(L, oracle):
    """PLM / WENO3 / scaled WENO5, non-hydrostatic < 1, disabled x2 flux."""
    for kw in (dict(recon="plm"), dict(recon="weno3"), dict(scale=True), dict(nh=0.3),
               dict(disable=True)):
        opts, w, _ = problems.straka(nx2=32, nx1=16, implicit_scheme=0)
        c = opts.hydro
        if "recon" in kw:
            c.recon1_type = c.recon23_type = {"plm": 1, "weno3": 4}[kw["recon"]]
        if kw.get("scale"):
            c.recon1_scale = c.recon23_scale = 1
        if "nh" in kw:
            c.non_hydrostatic = kw["nh"]
        if kw.get("disable"):
            c.disable_flux[1] = 1
        err, *_ = _forward_case(L, oracle, opts, w, 0.5)
        assert err < 1e-12, (kw, err)


# ---------------------------------------------------- full RK3 steps ----
def _run_gpu(opts, w, r, nsteps, dts=None):
    from snapy_linfel_b200.mesh import MeshBlock

    mb = MeshBlock(opts)
    mb.initialize(w, r)
    used = []
    for n in range(nsteps):
        if dts is None:
            mb.max_time_step()
        else:
            mb.set_dt(dts[n])
        used.append(mb.dt.item())
        for s in range(3):
            mb.forward(s)
    torch.cuda.synchronize()
    return mb, used


def _run_oracle(oracle, opts, w, r, nsteps, dts=None):
    c = opts.hydro
    w = w.copy()
    oracle.bc_apply(c, w, PRIMITIVE)
    u = oracle.prim2cons(c, w)
    s = s0 = rr = None
    if c.nscalar:
        rr = r.copy()
        oracle.bc_apply(c, rr, SCALAR)
        s = w[0:1] * rr
        s0 = np.empty_like(s)
        oracle.bc_apply(c, s, SCALAR)
    oracle.bc_apply(c, u, CONSERVED)
    blk = oracle.block(c)
    u0 = np.empty_like(u)
    used = []
    for n in range(nsteps):
        dt = opts.integration.cfl * oracle.max_time_step(c, w) if dts is None else dts[n]
        used.append(dt)
        for st in range(3):
            blk.stage(st, dt, u, u0, w, s, s0, rr)
    return u, s, used


def test_steps_sod_vs_golden(L, golden_npz):
    opts, w, _ = problems.sod(nx1=256)
    mb, used = _run_gpu(opts, w, None, 30, dts=golden_npz["sod_dts"])
    u = mb.hydro_u.cpu().numpy()
    ref = golden_npz["sod_u_final"]
    assert state_err(u, ref, ref) < 1e-12 * 30


@pytest.mark.parametrize("scheme", [0, 1, 9])
def test_steps_straka_vs_golden(L, golden_npz, scheme):
    opts, w, _ = problems.straka(nx2=24, nx1=12, implicit_scheme=scheme)
    mb, _ = _run_gpu(opts, w, None, 4, dts=golden_npz[f"straka{scheme}_dts"])
    it = (slice(None),) + opts.hydro.interior()
    u = mb.hydro_u.cpu().numpy()
    ref = golden_npz[f"straka{scheme}_u_final"][it]
    assert state_err(u[it], ref, ref) < 1e-12 * 4


def test_steps_cfl_dt_matches_oracle(L, oracle):
    opts, w, _ = problems.sod(nx1=128)
    _, used_gpu = _run_gpu(opts, w, None, 10)
    _, _, used_orc = _run_oracle(oracle, opts, w, None, 10)
    np.testing.assert_allclose(used_gpu, used_orc, rtol=1e-12)


def test_steps_3d_scalars_implicit(L, oracle):
    opts, w, r = problems.large_3d(nx3=10, nx2=12, nx1=16, nscalar=2)
    dts = [0.5, 0.5, 0.5]
    mb, _ = _run_gpu(opts, w, r, 3, dts=dts)
    u_ref, s_ref, _ = _run_oracle(oracle, opts, w, r, 3, dts=dts)
    it = (slice(None),) + opts.hydro.interior()
    assert state_err(mb.hydro_u.cpu().numpy()[it], u_ref[it], u_ref[it]) < 1e-12 * 3
    s = mb.scalar_s.cpu().numpy()[it]
    assert np.max(np.abs(s - s_ref[it])) / np.max(np.abs(s_ref[it])) < 1e-12 * 3


def test_mass_conservation_gpu(L):
    opts, w, _ = problems.straka(nx2=96, nx1=32, implicit_scheme=1)
    from snapy_linfel_b200.mesh import MeshBlock

    mb = MeshBlock(opts)
    mb.initialize(w)
    m0 = mb.totals()[0].item()
    for _ in range(10):
        mb.step()
    assert abs(mb.totals()[0].item() / m0 - 1.0) < 1e-12
    assert mb.check_redo() == 0


@pytest.fixture(scope="module")
def golden_npz():
    import os

    return np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_kernels.npz"))


# ------------------------------------------------ implicit correction ----
@pytest.mark.parametrize("variant", ["column", "fused"])
@pytest.mark.parametrize("scheme", [1, 9])
def test_implicit_correction_matches_oracle(L, oracle, scheme, variant, monkeypatch):
    """both implicit-solve variants: the column + finish kernels and the
    fused kernel (SNAPB_VIC_KERNEL=fused)"""
    if variant == "fused":
        monkeypatch.setenv("SNAPB_VIC_KERNEL", "fused")
    opts, w, _ = problems.straka(nx2=40, nx1=24, implicit_scheme=scheme)
    c = opts.hydro
    oracle.bc_apply(c, w, PRIMITIVE)
    u = oracle.prim2cons(c, w)
    rng = np.random.default_rng(scheme)
    # a stage tendency of realistic size: one explicit forward plus noise
    blk = oracle.block(c)
    cexp = c.copy()
    cexp.implicit_scheme = 0
    w_full = np.empty_like(u)
    du = oracle.block(cexp).hydro_forward(2.0, u, w_full)
    du += 1e-3 * rng.standard_normal(du.shape) * np.abs(du).max(axis=(1, 2, 3), keepdims=True)
    du_ref, m_ref = du.copy(), np.zeros_like(u)
    oracle.implicit_correction(c, 2.0, du_ref, w_full, m_ref)
    ws = torch.empty(L.lib().snapb_workspace_size(ctypes.byref(c)), dtype=torch.uint8,
                     device="cuda")
    dug, wg = dev(du), dev(w_full)
    mg = torch.zeros_like(wg)
    dtg = torch.tensor([2.0], dtype=torch.float64, device="cuda")
    call(L, "snapb_implicit_correction", ctypes.byref(c), L.ptr(dtg), L.ptr(dug), L.ptr(wg),
         L.ptr(mg), L.ptr(ws), ctypes.c_size_t(ws.numel()), L.stream_ptr())
    it = (slice(None),) + c.interior()
    assert state_err(dug.cpu().numpy()[it], du_ref[it], u[it]) < 1e-12
    m = mg.cpu().numpy()
    assert np.max(np.abs(m[0][it[1:]] - m_ref[0][it[1:]])) / np.max(np.abs(u[0])) < 1e-12
    del blk
