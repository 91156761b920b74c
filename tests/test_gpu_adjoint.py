"""Adjoint of the FP64 step on the GPU, checked against FP64 central finite
differences of the forward path (both through the C ABI).

For a random cotangent g and a random direction v, the reverse gives
<g, J v> = <J^T g, v>; the forward gives the same number as the central
difference D(eps) = (<g, f(x + eps v)> - <g, f(x - eps v)>) / (2 eps), taken
here Richardson-extrapolated, (4 D(eps/2) - D(eps)) / 3, which removes the
eps^2 truncation term (plain D(1e-6) is off by ~1e-6 relative on these
states; the extrapolated one agrees to ~1e-9).  Bound: 1e-6 relative.
Points are generic (smooth random states), away from the solvers' switches.
"""
import ctypes

import numpy as np
import pytest

from snapy_linfel_b200 import problems
from snapy_linfel_b200.config import CONSERVED, PRIMITIVE, SCALAR, make_config

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL = 1e-6


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from snapy_linfel_b200 import _lib

    return _lib


def smooth_field(shape, rng, modes=3):
    """sum of a few random sine modes on the index grid, in [-1, 1]"""
    k3, k2, k1 = np.meshgrid(*[np.arange(n) / max(n, 1) for n in shape], indexing="ij")
    f = np.zeros(shape)
    for _ in range(modes):
        a = rng.uniform(0.5, 2.0, 3) * 2 * np.pi
        ph = rng.uniform(0, 2 * np.pi)
        f += np.sin(a[0] * k1 + a[1] * k2 + a[2] * k3 + ph)
    return f / modes


def make_state(cfg, seed, grav, vel=5.0):
    """primitive state: isentropic column (grav) or a smooth uniform-ish gas"""
    rng = np.random.default_rng(seed)
    shape = cfg.shape[1:]
    w = np.zeros(cfg.shape)
    if grav:
        rd, cp = cfg.rgas, cfg.rgas * cfg.gammad / (cfg.gammad - 1.0)
        X1, _, _ = problems._grids(cfg)
        temp, p = problems._isentropic(X1, 1.0e5, 300.0, -cfg.grav1, rd, cp)
        temp = temp + 1.5 * smooth_field(shape, rng)
        w[0] = p / (rd * temp)
        w[4] = p * (1.0 + 1e-3 * smooth_field(shape, rng))
    else:
        w[0] = 1.0 + 0.2 * smooth_field(shape, rng)
        w[4] = 1.0 + 0.2 * smooth_field(shape, rng)
    for v in (1, 2, 3):
        w[v] = vel * smooth_field(shape, rng)
    if cfg.nscalar:
        r = 0.5 + 0.4 * np.stack([smooth_field(shape, rng) for _ in range(cfg.nscalar)])
    else:
        r = None
    return w, r


def block(cfg, w, r):
    from snapy_linfel_b200.mesh import MeshBlock

    mb = MeshBlock(cfg, device="cuda")
    mb.initialize(w, r)
    return mb


def scales(u):
    """per-variable magnitudes of a conserved state [nv, ...]"""
    s = u.abs().amax(dim=(1, 2, 3))
    return s.clamp_min(1e-30).view(-1, 1, 1, 1)


def dot(a, b):
    return float((a * b).sum())


def bc_direction(L, cfg, v, kind):
    """a perturbation that keeps the boundary structure of the state (ghosts
    are the images of the interior), so wall faces stay mirror-symmetric and
    their Riemann switches are not crossed"""
    v = v.contiguous().clone()
    L.check(L.lib().snapb_bc_apply(ctypes.byref(cfg), L.ptr(v), int(v.shape[0]), kind,
                                   L.stream_ptr()))
    return v


def richardson(J, eps):
    """(4 D(eps/2) - D(eps)) / 3 of the central difference D of J(t) at t = 0"""
    d1 = (J(eps) - J(-eps)) / (2 * eps)
    d2 = (J(eps / 2) - J(-eps / 2)) / eps
    return (4 * d2 - d1) / 3


def check(fd, ad, what):
    err = abs(fd - ad) / max(abs(fd), abs(ad), 1e-300)
    assert err < TOL, f"{what}: finite difference {fd:.12e} vs adjoint {ad:.12e} (rel {err:.2e})"
    return err


CONFIGS = {
    "sod1d_weno5shock_hllc": dict(
        cfg=dict(nx1=24, x1=(0.0, 1.0), recon1="weno5", shock1=True, recon23="weno5",
                 riemann="hllc", bc=("outflow",) * 6), grav=False),
    "col2d_lmars_vic3": dict(
        cfg=dict(nx1=16, nx2=12, x1=(0.0, 1600.0), x2=(0.0, 1200.0), gammad=1004.0 / 717.0,
                 rgas=287.0, recon1="weno5", recon23="weno5", riemann="lmars",
                 implicit_scheme=1, grav=(-9.81, 0.0, 0.0),
                 bc=("reflecting", "reflecting", "periodic", "periodic", "reflecting",
                     "reflecting")), grav=True),
    "box3d_roe_vic5_scalars": dict(
        cfg=dict(nx1=10, nx2=6, nx3=6, x1=(0.0, 1000.0), x2=(0.0, 600.0), x3=(0.0, 600.0),
                 gammad=1004.0 / 717.0, rgas=287.0, recon1="weno5", recon23="weno5",
                 riemann="roe", implicit_scheme=9, grav=(-9.81, 0.0, 0.0), nscalar=2,
                 scalar_recon="weno5",
                 bc=("reflecting", "reflecting", "periodic", "periodic", "outflow", "outflow")),
        grav=True),
    "col2d_plm_hllc_weno3scaled": dict(
        cfg=dict(nx1=12, nx2=10, x1=(0.0, 1200.0), x2=(0.0, 1000.0), gammad=1.4, rgas=287.0,
                 recon1="plm", recon23="weno3", scale23=True, riemann="hllc",
                 grav=(-9.81, 0.0, 0.0), nscalar=1, scalar_recon="plm",
                 bc=("reflecting", "outflow", "periodic", "periodic", "reflecting",
                     "reflecting")), grav=True),
}


def cfg_of(name):
    return make_config(**CONFIGS[name]["cfg"])


def test_bc_adjoint_is_the_transpose(L):
    from snapy_linfel_b200.adjoint import bc_adjoint

    cfg = make_config(nx1=8, nx2=6, nx3=5, nscalar=1,
                      bc=("reflecting", "outflow", "periodic", "periodic", "outflow",
                          "reflecting"))
    g = torch.Generator(device="cuda").manual_seed(3)
    for kind, nv in ((CONSERVED, 5), (PRIMITIVE, 5), (SCALAR, 1)):
        x = torch.randn((nv,) + cfg.shape[1:], generator=g, device="cuda", dtype=torch.float64)
        y = torch.randn_like(x)
        bx = x.clone()
        L.check(L.lib().snapb_bc_apply(ctypes.byref(cfg), L.ptr(bx), nv, kind, L.stream_ptr()))
        bty = bc_adjoint(cfg, y, kind)
        a, b = dot(y, bx), dot(bty, x)
        assert abs(a - b) <= 1e-12 * max(abs(a), abs(b)), (kind, a, b)


@pytest.mark.parametrize("name", list(CONFIGS))
def test_hydro_forward_adjoint_fd(L, name):
    from snapy_linfel_b200.adjoint import Adjoint

    cfg = cfg_of(name)
    w, r = make_state(cfg, 11, CONFIGS[name]["grav"])
    mb = block(cfg, w, r)
    u = mb.hydro_u.clone()
    dt = mb.max_time_step().clone() * 0.5
    ws, nb = mb._ws()
    du = torch.zeros_like(u)

    def f(x):
        L.check(L.lib().snapb_hydro_forward(ctypes.byref(cfg), L.ptr(dt), L.ptr(x),
                                            L.ptr(mb.hydro_w), L.ptr(du), None, ws, nb,
                                            L.stream_ptr()), "hydro_forward")
        return du.clone()

    gen = torch.Generator(device="cuda").manual_seed(5)
    it = (slice(None),) + cfg.interior()
    gdu = torch.zeros_like(u)
    gdu[it] = torch.randn(gdu[it].shape, generator=gen, device="cuda", dtype=torch.float64)
    gdu = gdu / scales(f(u)).clamp_min(1e-300)
    adj = Adjoint(cfg)
    gu = adj.hydro_forward(dt, u, gdu)
    for trial in range(2):
        v = torch.randn(u.shape, generator=gen, device="cuda", dtype=torch.float64) * scales(u)
        v = bc_direction(L, cfg, v, CONSERVED)
        fd = richardson(lambda t: dot(gdu, f(u + t * v)), 2e-7)
        check(fd, dot(gu, v), f"{name} trial {trial}")


@pytest.mark.parametrize("stage", [0, 1, 2])
@pytest.mark.parametrize("name", ["box3d_roe_vic5_scalars", "col2d_lmars_vic3"])
def test_stage_adjoint_fd(L, name, stage):
    """d/d(u, u0, s, s0) of <g, stage output> through snapb_stage vs the reverse"""
    from snapy_linfel_b200.adjoint import Adjoint

    cfg = cfg_of(name)
    w, r = make_state(cfg, 17 + stage, CONFIGS[name]["grav"])
    mb = block(cfg, w, r)
    u = mb.hydro_u.clone()
    s = mb.scalar_s.clone() if cfg.nscalar else None
    # a step-start state that differs from the stage input
    w0, r0 = make_state(cfg, 99, CONFIGS[name]["grav"])
    mb0 = block(cfg, w0, r0)
    u0 = mb0.hydro_u.clone()
    s0 = mb0.scalar_s.clone() if cfg.nscalar else None
    dt = mb.max_time_step().clone() * 0.5

    def f(x, x0, y, y0):
        mb.hydro_u.copy_(x)
        mb.hydro_u0.copy_(x0)
        if cfg.nscalar:
            mb.scalar_s.copy_(y)
            mb.scalar_s0.copy_(y0)
            mb.scalar_r.copy_(y / x[0:1])
        mb.dt.copy_(dt)
        mb.forward(stage)
        return mb.hydro_u.clone(), (mb.scalar_s.clone() if cfg.nscalar else None)

    gen = torch.Generator(device="cuda").manual_seed(23 + stage)
    uo, so = f(u, u0, s, s0)
    gout = torch.randn(u.shape, generator=gen, device="cuda", dtype=torch.float64) / scales(uo)
    gsout = (torch.randn(s.shape, generator=gen, device="cuda", dtype=torch.float64)
             / scales(so)) if cfg.nscalar else None
    adj = Adjoint(cfg)
    gu0 = torch.zeros_like(u)
    gs0 = torch.zeros_like(s) if cfg.nscalar else None
    gu, gs = adj.stage(stage, dt, u, s, gout, gsout, gu0, gs0)
    if stage == 0:
        # u0 is the stage input itself at stage 0
        gu = gu + gu0
        if cfg.nscalar:
            gs = gs + gs0

    def J(x, x0, y, y0):
        a, b = f(x, x0, y, y0)
        out = dot(gout, a)
        if cfg.nscalar:
            out += dot(gsout, b)
        return out

    for trial in range(2):
        v = torch.randn(u.shape, generator=gen, device="cuda", dtype=torch.float64) * scales(u)
        v = bc_direction(L, cfg, v, CONSERVED)
        v0 = (v if stage == 0 else
              torch.randn(u.shape, generator=gen, device="cuda", dtype=torch.float64) * scales(u))
        vs = vs0 = None
        if cfg.nscalar:
            vs = torch.randn(s.shape, generator=gen, device="cuda", dtype=torch.float64) * scales(s)
            vs = bc_direction(L, cfg, vs, SCALAR)
            vs0 = vs if stage == 0 else torch.randn(
                s.shape, generator=gen, device="cuda", dtype=torch.float64) * scales(s)
        def pert(e):
            return J(u + e * v, u0 + e * v0, None if s is None else s + e * vs,
                     None if s0 is None else s0 + e * vs0)

        fd = richardson(pert, 2e-7)
        ad = dot(gu, v) + (0. if stage == 0 else dot(gu0, v0))
        if cfg.nscalar:
            ad += dot(gs, vs) + (0. if stage == 0 else dot(gs0, vs0))
        check(fd, ad, f"{name} stage {stage} trial {trial}")


AUTOGRAD_CONFIGS = {
    "col2d_lmars_vic3": CONFIGS["col2d_lmars_vic3"],
    "sod1d_weno5shock_hllc": CONFIGS["sod1d_weno5shock_hllc"],
    "box3d_hllc_vic3": dict(
        cfg=dict(nx1=10, nx2=6, nx3=6, x1=(0.0, 1000.0), x2=(0.0, 600.0), x3=(0.0, 600.0),
                 gammad=1004.0 / 717.0, rgas=287.0, riemann="hllc", implicit_scheme=1,
                 grav=(-9.81, 0.0, 0.0),
                 bc=("reflecting", "reflecting", "periodic", "periodic", "outflow",
                     "outflow")), grav=True),
    "box3d_roe_cp5": dict(
        cfg=dict(nx1=8, nx2=6, nx3=5, recon23="cp5", riemann="roe",
                 bc=("outflow", "reflecting", "periodic", "periodic", "outflow",
                     "reflecting")), grav=False),
}


@pytest.mark.parametrize("stage", [0, 1, 2])
@pytest.mark.parametrize("name", list(AUTOGRAD_CONFIGS))
def test_stage_adjoint_matches_torch_autograd(L, name, stage):
    """the hand-written reverse of one stage against torch autograd through
    the torch restatement of the same stage (pinned to the C++ oracle on the
    CPU): every entry of d<g, stage(u, u0)>/du and /du0, ghosts included.
    Bound: 1e-6 of each variable's largest gradient entry."""
    from oracle import torch_step

    from snapy_linfel_b200.adjoint import Adjoint

    spec = AUTOGRAD_CONFIGS[name]
    cfg = make_config(**spec["cfg"])
    w, _ = make_state(cfg, 31 + stage, spec["grav"])
    mb = block(cfg, w, None)
    u = mb.hydro_u.clone()
    u0 = u.clone()
    if stage:
        w0, _ = make_state(cfg, 77, spec["grav"])
        u0 = block(cfg, w0, None).hydro_u.clone()
    dt = mb.max_time_step().clone() * 0.5
    gen = torch.Generator(device="cuda").manual_seed(41 + stage)
    gout = torch.randn(u.shape, generator=gen, device="cuda", dtype=torch.float64) / scales(u)

    adj = Adjoint(cfg)
    gu0 = torch.zeros_like(u)
    gu, _ = adj.stage(stage, dt, u, None, gout, None, gu0, None)
    torch.cuda.synchronize()

    ut = u.clone().requires_grad_(True)
    u0t = ut if stage == 0 else u0.clone().requires_grad_(True)
    out = torch_step.stage(ut, u0t, stage, float(dt.reshape(-1)[0]), cfg)
    (out * gout).sum().backward()
    pairs = [("u", gu + gu0 if stage == 0 else gu, ut.grad)]
    if stage:
        pairs.append(("u0", gu0, u0t.grad))
    for what, got, want in pairs:
        for v in range(5):
            scale = float(want[v].abs().max())
            err = float((got[v] - want[v]).abs().max()) / max(scale, 1e-300)
            assert err < TOL, f"{name} stage {stage} d/d{what}[{v}]: rel {err:.2e}"


@pytest.mark.parametrize("stage", [0, 2])
@pytest.mark.parametrize("name", ["col2d_lmars_vic3", "box3d_hllc_vic3"])
def test_vic_adjoint_solvers_agree(L, name, stage, monkeypatch):
    """The adjoint's column solve by the two-pass block-Thomas sweep and by
    block cyclic reduction (the default for few columns): the same stage
    gradient up to FP64 rounding (bound 1e-11 of each variable's largest
    entry)."""
    from snapy_linfel_b200.adjoint import Adjoint

    spec = AUTOGRAD_CONFIGS[name]
    cfg = make_config(**spec["cfg"])
    w, _ = make_state(cfg, 53 + stage, spec["grav"])
    u = block(cfg, w, None).hydro_u.clone()
    w0, _ = make_state(cfg, 59, spec["grav"])
    u0 = block(cfg, w0, None).hydro_u.clone()
    dt = block(cfg, w, None).max_time_step().clone() * 0.5
    gen = torch.Generator(device="cuda").manual_seed(61 + stage)
    gout = torch.randn(u.shape, generator=gen, device="cuda", dtype=torch.float64) / scales(u)
    got = {}
    for solver in ("sweep", "cr"):
        monkeypatch.setenv("SNAPB_VADJ_SOLVE", solver)
        gu0 = torch.zeros_like(u)
        gu, _ = Adjoint(cfg).stage(stage, dt, u, None, gout, None, gu0, None)
        torch.cuda.synchronize()
        got[solver] = (gu.clone(), gu0.clone())
    for k in range(2):
        a, b = got["sweep"][k], got["cr"][k]
        for v in range(5):
            scale = float(a[v].abs().max())
            if scale == 0.:
                assert float(b[v].abs().max()) == 0.
                continue
            err = float((a[v] - b[v]).abs().max()) / scale
            assert err < 1e-11, f"{name} stage {stage} output {k} var {v}: rel {err:.2e}"


def test_rollout_gradient_fd(L):
    """J = kinetic energy after 6 RK3 steps (checkpoints every 2 steps) of a
    warm bubble, gradient wrt the initial potential-temperature perturbation
    through torch.autograd, against central differences along random
    directions.  A weak seeded flow is added to the bubble at rest so that
    no face sits exactly on the HLLC contact / PVRS switches (a resting,
    horizontally uniform pressure puts every x2 face on them)."""
    from snapy_linfel_b200 import adjoint as A

    opts, w, _ = problems.adjoint_bubble(nx2=24, nx1=16, seed=3)
    cfg = opts.hydro
    rng = np.random.default_rng(4)
    w[1] = 0.3 * smooth_field(cfg.shape[1:], rng)
    w[2] = 0.3 * smooth_field(cfg.shape[1:], rng)
    base = torch.from_numpy(w).cuda()
    X1 = torch.from_numpy(problems._grids(cfg)[0]).cuda()
    rd, cp = cfg.rgas, cfg.rgas * cfg.gammad / (cfg.gammad - 1.0)
    p = base[4]
    temp0 = p / (rd * base[0])

    def state(dth):
        wt = base.clone()
        wt = torch.cat([(p / (rd * (temp0 + dth * (p / 1.0e5) ** (rd / cp))))[None], wt[1:]])
        return A.initial_state(cfg, wt)

    dth0 = torch.zeros(cfg.shape[1:], dtype=torch.float64, device="cuda")
    dts = A.cfl_steps(opts, state(dth0).detach(), nsteps=6)
    it = cfg.interior()

    def J(dth):
        uT, _ = A.rollout(opts, state(dth), None, dts, checkpoint_every=2)
        ke = 0.5 * (uT[1] ** 2 + uT[2] ** 2 + uT[3] ** 2) / uT[0]
        return ke[it].sum()

    x = dth0.clone().requires_grad_(True)
    j = J(x)
    (grad,) = torch.autograd.grad(j, x)
    assert float(grad.abs().max()) > 0
    gen = torch.Generator(device="cuda").manual_seed(8)
    for trial in range(3):
        v = torch.randn(x.shape, generator=gen, device="cuda", dtype=torch.float64)
        with torch.no_grad():
            fd = richardson(lambda t: float(J(dth0 + t * v)), 1e-3)
        check(fd, dot(grad, v), f"rollout trial {trial}")
    # keeping every step's stage inputs in the forward pass (checkpoint_every=0)
    # gives the gradient of the checkpointed re-run exactly
    x0 = dth0.clone().requires_grad_(True)
    uT, _ = A.rollout(opts, state(x0), None, dts, checkpoint_every=0)
    j0 = (0.5 * (uT[1] ** 2 + uT[2] ** 2 + uT[3] ** 2) / uT[0])[it].sum()
    (grad0,) = torch.autograd.grad(j0, x0)
    assert torch.equal(grad0, grad)


def _face_states(cfg, regime, dim, gen):
    """random left/right primitive states on every face of the array"""
    shape = cfg.shape
    u = lambda lo, hi: lo + (hi - lo) * torch.rand(shape[1:], generator=gen, device="cuda",
                                                   dtype=torch.float64)
    ivx = 4 - dim
    wl = torch.empty(shape, dtype=torch.float64, device="cuda")
    wr = torch.empty_like(wl)
    for w in (wl, wr):
        w[0] = u(0.5, 2.0)
        w[4] = u(0.5, 2.0)
        for v in (1, 2, 3):
            w[v] = u(-0.5, 0.5)
    if regime == "smooth":
        wr.copy_(wl * (1.0 + 0.1 * (torch.rand(shape, generator=gen, device="cuda",
                                               dtype=torch.float64) - 0.5)))
    elif regime == "supersonic":  # every wave one way: upwind / one-sided branches
        wl[ivx] = u(2.5, 4.0)
        wr[ivx] = u(2.5, 4.0)
        half = shape[1] // 2
        wl[ivx][:half] *= -1.0
        wr[ivx][:half] *= -1.0
    else:  # strong rarefaction and pressure jumps: Roe's LLF fallback, shocked PVRS
        wl[ivx] = u(-4.0, -2.0)
        wr[ivx] = u(2.0, 4.0)
        wr[4] = wr[4] * 10.0
    return wl, wr


@pytest.mark.parametrize("regime", ["smooth", "supersonic", "strong"])
@pytest.mark.parametrize("dim", [3, 2, 1])
@pytest.mark.parametrize("solver", ["hllc", "lmars", "roe"])
def test_riemann_adjoint_fd(L, solver, dim, regime):
    """the hand-written reverse of each Riemann solver (snapb_riemann_adjoint)
    against central differences of snapb_riemann, in every branch regime"""
    from snapy_linfel_b200.config import RIEMANN

    cfg = make_config(nx1=8, nx2=8, nx3=8, gammad=1.4)
    sid = RIEMANN[solver]
    gen = torch.Generator(device="cuda").manual_seed(100 + 10 * dim + len(regime))
    wl, wr = _face_states(cfg, regime, dim, gen)
    flx = torch.empty_like(wl)

    def F(a, b):
        L.check(L.lib().snapb_riemann(ctypes.byref(cfg), sid, dim, L.ptr(a), L.ptr(b), 5,
                                      L.ptr(flx), None, None, L.stream_ptr()), "riemann")
        return flx.clone()

    g = torch.randn(wl.shape, generator=gen, device="cuda", dtype=torch.float64)
    gwl, gwr = torch.empty_like(wl), torch.empty_like(wr)
    L.check(L.lib().snapb_riemann_adjoint(ctypes.byref(cfg), sid, dim, L.ptr(wl), L.ptr(wr),
                                          L.ptr(g), L.ptr(gwl), L.ptr(gwr), L.stream_ptr()),
            "riemann_adjoint")
    for trial in range(2):
        vl = torch.randn(wl.shape, generator=gen, device="cuda", dtype=torch.float64) * wl.abs()
        vr = torch.randn(wr.shape, generator=gen, device="cuda", dtype=torch.float64) * wr.abs()
        fd = richardson(lambda t: dot(g, F(wl + t * vl, wr + t * vr)), 2e-7)
        check(fd, dot(gwl, vl) + dot(gwr, vr), f"{solver} dim {dim} {regime} trial {trial}")
