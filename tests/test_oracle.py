"""CPU tests of the oracle: it is pinned to the reference's known answers,
fixtures and own point kernels before anything is checked against it."""
import os

import numpy as np
import pytest

from snapy_linfel_b200 import problems
from snapy_linfel_b200.config import CONSERVED, PRIMITIVE, make_config

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_kernels.npz")


# ---- known answers (tests/test_weno.cpp:145-184, tests/test_plm.cpp:20-27) ----
def test_weno5_known_answer(oracle):
    # interp_weno5(1, 2, 3, 4, 5) = 2.5000000000000004 in the reference
    assert oracle.interp_point(5, 1, [1, 2, 3, 4, 5]) == pytest.approx(2.5000000000000004,
                                                                       abs=1e-10)


def test_weno3_known_answer(oracle):
    assert oracle.interp_point(4, 1, [1, 2, 3]) == pytest.approx(1.5, abs=1e-10)


def test_plm_known_answer(oracle):
    assert oracle.interp_point(1, 1, [1, 2, 3]) == pytest.approx(1.5, abs=1e-10)


def test_weno5_smooth_limit_is_cp5(oracle):
    eps = 1e-7
    win = [1 + eps, 1 + 2 * eps, 1 + 4 * eps, 1 + 8 * eps, 1 + 16 * eps]
    for side in (0, 1):
        assert oracle.interp_point(5, side, win) == pytest.approx(
            oracle.interp_point(3, side, win), abs=1e-6)


# ---- face-pressure closed forms (tests/test_riemann.cpp:412-540) ----
def _seeded_states(seed, shape):
    torch = pytest.importorskip("torch")
    torch.manual_seed(seed)
    wl = torch.rand(shape, dtype=torch.float64)
    wr = torch.rand(shape, dtype=torch.float64)
    for w in (wl, wr):
        w[0].add_(1.0)
        w[4].add_(1.0)
        w[1:4].sub_(0.5).mul_(0.1)
    return wl.numpy().copy(), wr.numpy().copy()


@pytest.fixture
def small_cfg():
    # the reference test block: 10 x 8 x 6 cells, 3 ghosts, ideal gas 1.4
    return make_config(nx1=10, nx2=8, nx3=6, nghost=3, gammad=1.4)


def test_hllc_face_pressure(oracle, small_cfg):
    wl, wr = _seeded_states(77, small_cfg.shape)
    g = 1.4
    cl = np.sqrt(g * wl[4] / wl[0])
    cr = np.sqrt(g * wr[4] / wr[0])
    rhoa = 0.5 * (wl[0] + wr[0])
    ca = 0.5 * (cl + cr)
    pmid = 0.5 * (wl[4] + wr[4] + (wl[1] - wr[1]) * rhoa * ca)
    ql = np.where(pmid <= wl[4], 1.0, np.sqrt(1.0 + (g + 1) / (2 * g) * (pmid / wl[4] - 1.0)))
    qr = np.where(pmid <= wr[4], 1.0, np.sqrt(1.0 + (g + 1) / (2 * g) * (pmid / wr[4] - 1.0)))
    al = wl[1] - cl * ql
    ar = wr[1] + cr * qr
    vxl, vxr = wl[1] - al, wr[1] - ar
    tl = wl[4] + vxl * wl[0] * wl[1]
    tr = wr[4] + vxr * wr[0] * wr[1]
    ml, mr = wl[0] * vxl, -(wr[0] * vxr)
    expected = np.maximum((ml * tr + mr * tl) / (ml + mr), 0.0)
    _, fp = oracle.riemann(small_cfg, 2, 3, wl, wr)
    np.testing.assert_allclose(fp, expected, rtol=1e-10, atol=1e-10)


def test_lmars_face_pressure(oracle, small_cfg):
    wl, wr = _seeded_states(78, small_cfg.shape)
    g = 1.4
    rhobar = 0.5 * (wl[0] + wr[0])
    cbar = np.sqrt(g * 0.5 * (wl[4] + wr[4]) / rhobar)
    expected = 0.5 * (wl[4] + wr[4]) + 0.5 * (rhobar * cbar) * (wl[1] - wr[1])
    _, fp = oracle.riemann(small_cfg, 1, 3, wl, wr)
    np.testing.assert_allclose(fp, expected, rtol=1e-10, atol=1e-10)


def test_roe_face_pressure(oracle, small_cfg):
    wl, wr = _seeded_states(79, small_cfg.shape)
    g = 1.4
    ul = oracle.prim2cons(small_cfg, wl)
    ur = oracle.prim2cons(small_cfg, wr)
    sl, sr = np.sqrt(wl[0]), np.sqrt(wr[0])
    isd = 1.0 / (sl + sr)
    hbar = ((ul[4] + wl[4]) / sl + (ur[4] + wr[4]) / sr) * isd
    vbar = (sl * wl[1:4] + sr * wr[1:4]) * isd
    cs = np.sqrt((g - 1.0) * (hbar - 0.5 * (vbar ** 2).sum(0)))
    expected = 0.5 * (wl[4] + wr[4] + sl * sr * cs * (wl[1] - wr[1]))
    flx, fp = oracle.riemann(small_cfg, 0, 3, wl, wr)
    np.testing.assert_allclose(fp, expected, rtol=1e-10, atol=1e-10)
    assert np.abs(flx).sum() > 0


# ---- VIC redistribution fixture (tests/test_backward_substitution.cpp:25-153) ----
def test_vic_redistribution_fixture(oracle):
    nlayer, ny = 4, 3
    nh = 5 + ny
    du = np.zeros((nh, nlayer))
    w = np.zeros((nh, nlayer))
    vol = np.array([1.0, 2.0, 1.5, 0.5])
    corr = [0.4, -0.2, 0.1, -0.3]
    rho = [3.0, 2.5, 4.0, 1.8]
    delta = np.zeros((nlayer, 3))
    for i in range(nlayer):
        vf, cf, tf = 0.10 + 0.02 * i, 0.05 + 0.01 * i, 0.02 + 0.005 * i
        dry = 1.0 - vf - cf - tf
        et = 1.5 + 0.2 * i
        du[0, i] = et * dry
        du[1, i] = 10.0 + i
        du[4, i] = 20.0 + i
        du[5, i], du[6, i], du[7, i] = et * vf, et * cf, et * tf
        w[5, i], w[6, i], w[7, i] = vf, cf, tf
        w[0, i] = rho[i]
        delta[i] = (et + corr[i], 100.0 + i, 200.0 + i)
    orig = du.copy()
    mass = np.zeros_like(du)
    implicit_total = delta[:, 0].copy()
    oracle.vic_redistribute(du, w, mass, delta, vol, nlayer, nh, ny, 3)
    col = lambda a, v: float((vol * a[v]).sum())  # noqa: E731
    for v in (0, 5):
        assert col(du, v) == pytest.approx(col(orig, v), abs=1e-1)
    sum_a2 = float(((np.array(rho) * vol) ** 2).sum())
    for v in (0, 5):
        if v == 0:
            frac_b = 1.0 - w[5] - w[6] - w[7]
            frac = 1.0 - w[5] - w[6]
        else:
            frac_b = frac = w[v]
        b_j = float(((orig[0] + orig[5] + orig[6] - implicit_total) * frac_b * vol).sum())
        for i in range(nlayer):
            et = orig[0, i] + orig[5, i] + orig[6, i] + orig[7, i]
            struct = rho[i] * (rho[i] * vol[i]) * b_j / sum_a2
            exp = orig[v, i] + (implicit_total[i] - et) * frac[i] + struct
            assert du[v, i] == pytest.approx(exp, abs=1e-1)
    for i in range(nlayer):
        et = orig[0, i] + orig[5, i] + orig[6, i] + orig[7, i]
        assert mass[0, i] == pytest.approx(implicit_total[i] - et, abs=1e-12)
        for v in (6, 7):
            exp = orig[v, i] + (implicit_total[i] - et) * w[v, i]
            assert du[v, i] == pytest.approx(exp, abs=1e-12)
    # momentum / energy take the implicit solution
    np.testing.assert_array_equal(du[1], delta[:, 1])
    np.testing.assert_array_equal(du[4], delta[:, 2])


# ---- the oracle reproduces the reference kernels' fixtures bit for bit ----
@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _golden_cfg():
    return make_config(nx1=5, nx2=4, nx3=3, nghost=3)


@pytest.mark.parametrize("name,t", [("weno5", 5), ("weno3", 4), ("plm", 1), ("cp5", 3),
                                    ("cp3", 2), ("dc", 0)])
def test_golden_reconstruct(oracle, golden, name, t):
    w = golden["recon_w"]
    for shock in ((0, 1) if name.startswith("weno") else (0,)):
        c = _golden_cfg()
        c.recon1_type = c.recon23_type = t
        c.recon1_shock = c.recon23_shock = shock
        for dim in (3, 2, 1):
            np.testing.assert_array_equal(oracle.reconstruct(c, dim, 0, w),
                                          golden[f"recon_{name}_s{shock}_d{dim}"])


def test_golden_reconstruct_scale_and_scalar(oracle, golden):
    w = golden["recon_w"]
    c = _golden_cfg()
    c.recon1_type = c.recon23_type = 5
    c.recon1_scale = c.recon23_scale = 1
    for dim in (3, 2, 1):
        np.testing.assert_array_equal(oracle.reconstruct(c, dim, 0, w),
                                      golden[f"recon_weno5scale_d{dim}"])
    c = _golden_cfg()
    c.scalar_recon_type = 5
    for dim in (3, 2, 1):
        out = oracle.reconstruct(c, dim, 1, golden["recon_scalar_in"])
        np.testing.assert_array_equal(out, golden[f"recon_scalar_d{dim}"])
        assert out.min() >= 0.0


@pytest.mark.parametrize("name,s", [("roe", 0), ("lmars", 1), ("hllc", 2)])
def test_golden_riemann(oracle, golden, name, s):
    c = _golden_cfg()
    for dim in (3, 2, 1):
        f, p = oracle.riemann(c, s, dim, golden["riemann_wl"], golden["riemann_wr"])
        np.testing.assert_array_equal(f, golden[f"riemann_{name}_d{dim}_flx"])
        np.testing.assert_array_equal(p, golden[f"riemann_{name}_d{dim}_fp"])


def test_golden_upwind_and_eos(oracle, golden):
    c = _golden_cfg()
    f, _ = oracle.riemann(c, 3, 3, golden["riemann_wl"], golden["riemann_wr"],
                          vel=golden["riemann_vel"], face_pressure=False)
    np.testing.assert_array_equal(f, golden["riemann_upwind_d3_flx"])
    np.testing.assert_array_equal(oracle.prim2cons(c, golden["recon_w"]), golden["eos_u"])
    np.testing.assert_array_equal(oracle.cons2prim(c, golden["eos_u"]), golden["eos_w"])


def _run_steps(oracle, cfg, u, nsteps, cfl=0.9):
    w = oracle.cons2prim(cfg, u)
    blk = oracle.block(cfg)
    u0 = np.empty_like(u)
    dts = []
    for _ in range(nsteps):
        dt = cfl * oracle.max_time_step(cfg, w)
        dts.append(dt)
        for s in range(3):
            blk.stage(s, dt, u, u0, w)
    return np.array(dts)


def test_golden_sod_steps(oracle, golden):
    opts, _, _ = problems.sod(nx1=256)
    u = golden["sod_u_init"].copy()
    # the fixture started from hydro_w after the primitive boundary fill
    w = oracle.cons2prim(opts.hydro, u)
    blk = oracle.block(opts.hydro)
    u0 = np.empty_like(u)
    for n, dt in enumerate(golden["sod_dts"]):
        assert 0.9 * oracle.max_time_step(opts.hydro, w) == dt or n == 0
        for s in range(3):
            blk.stage(s, dt, u, u0, w)
    np.testing.assert_array_equal(u, golden["sod_u_final"])


@pytest.mark.parametrize("scheme", [0, 1, 9])
def test_golden_straka_steps(oracle, golden, scheme):
    opts, _, _ = problems.straka(nx2=24, nx1=12, implicit_scheme=scheme)
    u = golden[f"straka{scheme}_u_init"].copy()
    w = oracle.cons2prim(opts.hydro, u)
    blk = oracle.block(opts.hydro)
    u0 = np.empty_like(u)
    for dt in golden[f"straka{scheme}_dts"]:
        for s in range(3):
            blk.stage(s, dt, u, u0, w)
    np.testing.assert_array_equal(u, golden[f"straka{scheme}_u_final"])


def _vic_case(scheme, case):
    if case == "straka":
        opts, _, _ = problems.straka(nx2=16, nx1=20, implicit_scheme=scheme)
    else:
        opts, _, _ = problems.warm_bubble_3d(4, 5, 12, amp=2.0, radius=500.0,
                                              center=(200.0, 250.0, 500.0),
                                              implicit_scheme=scheme)
    return opts.hydro


@pytest.mark.parametrize("scheme", [1, 9])
@pytest.mark.parametrize("case", ["straka", "box"])
def test_golden_implicit_correction(oracle, golden, scheme, case):
    """the restated VIC reproduces the reference's own implicit code
    (oracle/_ref, Eigen subset shim) bit for bit on the fixture"""
    c = _vic_case(scheme, case)
    key = f"vic{scheme}_{case}"
    du = golden[key + "_du_in"].copy()
    mass = np.zeros_like(du)
    oracle.implicit_correction(c, 2.0, du, golden[key + "_w"], mass)
    np.testing.assert_array_equal(du, golden[key + "_du_out"])
    np.testing.assert_array_equal(mass, golden[key + "_mass"])
    assert not np.array_equal(du, golden[key + "_du_in"])


# ---- restated kernels == the reference's own kernels on fresh inputs ----
def test_port_matches_reference_kernels(oracle, ref_oracle):
    rng = np.random.default_rng(99)
    c = make_config(nx1=9, nx2=7, nx3=6, nghost=3)
    w = rng.random(c.shape) + 0.5
    w[1:4] -= 1.0
    for t in (0, 1, 2, 3, 4, 5):
        c.recon1_type = c.recon23_type = t
        for dim in (3, 2, 1):
            np.testing.assert_array_equal(oracle.reconstruct(c, dim, 0, w),
                                          ref_oracle.reconstruct(c, dim, 0, w))
    wl = rng.random(c.shape) + 0.5
    wr = rng.random(c.shape) + 0.5
    for s in (0, 1, 2):
        for dim in (3, 2, 1):
            a = oracle.riemann(c, s, dim, wl, wr)
            b = ref_oracle.riemann(c, s, dim, wl, wr)
            np.testing.assert_array_equal(a[0], b[0])
            np.testing.assert_array_equal(a[1], b[1])


@pytest.mark.parametrize("scheme", [1, 9])
def test_port_vic_matches_reference_code(oracle, ref_oracle, scheme):
    """restated implicit solve vs the reference's vic_assemble_*_impl.h /
    ForwardSweep / vic_backward_reduce / vic_redistribute_cell, on a seeded
    flow (bound 1e-13 per field; identical in practice)"""
    for case in ("straka", "bubble"):
        if case == "straka":
            opts, w, _ = problems.straka(nx2=40, nx1=24, implicit_scheme=scheme)
        else:
            opts, w, _ = problems.warm_bubble_3d(6, 7, 18, amp=2.0, radius=700.0,
                                                  center=(300.0, 350.0, 800.0),
                                                  implicit_scheme=scheme)
        c = opts.hydro
        rng = np.random.default_rng(40 + scheme)
        w[1:4] += 0.3 * rng.standard_normal(w[1:4].shape)
        oracle.bc_apply(c, w, PRIMITIVE)
        u = oracle.prim2cons(c, w)
        oracle.bc_apply(c, u, CONSERVED)
        ce = c.copy()
        ce.implicit_scheme = 0
        wf = np.empty_like(u)
        du = oracle.block(ce).hydro_forward(2.0, u, wf)
        du += 1e-3 * rng.standard_normal(du.shape) * np.abs(du).max(axis=(1, 2, 3),
                                                                  keepdims=True)
        a, b = du.copy(), du.copy()
        ma, mb = np.zeros_like(u), np.zeros_like(u)
        oracle.implicit_correction(c, 2.0, a, wf, ma)
        ref_oracle.implicit_correction(c, 2.0, b, wf, mb)
        it = (slice(None),) + c.interior()
        for v in range(5):
            assert np.abs(a[it][v] - b[it][v]).max() <= 1e-13 * np.abs(b[it][v]).max(), v
        assert np.abs(ma - mb).max() <= 1e-13 * np.abs(u[0]).max()
        # the two full stages (explicit sweep + VIC + RK) agree as well
        u1, u2 = u.copy(), u.copy()
        w1, w2 = np.empty_like(u), np.empty_like(u)
        z1, z2 = np.empty_like(u), np.empty_like(u)
        oracle.block(c).stage(0, 1.0, u1, z1, w1)
        ref_oracle.block(c).stage(0, 1.0, u2, z2, w2)
        np.testing.assert_allclose(u1, u2, rtol=1e-13, atol=0)


# ---- example-level mass conservation (tests/run_example_mass_check.py) ----
def test_sod_mass_conservation(oracle):
    opts, w, _ = problems.sod(nx1=256)
    c = opts.hydro
    oracle.bc_apply(c, w, PRIMITIVE)
    u = oracle.prim2cons(c, w)
    oracle.bc_apply(c, u, CONSERVED)
    it = c.interior()
    m0 = u[0][it].sum()
    _run_steps(oracle, c, u, 40)
    assert abs(u[0][it].sum() / m0 - 1.0) <= 1e-8


def test_straka_implicit_mass_conservation(oracle):
    for scheme in (1, 9):
        opts, w, _ = problems.straka(nx2=48, nx1=16, implicit_scheme=scheme)
        c = opts.hydro
        oracle.bc_apply(c, w, PRIMITIVE)
        u = oracle.prim2cons(c, w)
        oracle.bc_apply(c, u, CONSERVED)
        it = c.interior()
        m0 = u[0][it].sum()
        _run_steps(oracle, c, u, 5)
        assert abs(u[0][it].sum() / m0 - 1.0) <= 1e-12
        assert np.isfinite(u).all()


def test_thread_count_does_not_change_results(oracle):
    opts, w, _ = problems.straka(nx2=32, nx1=12, implicit_scheme=1)
    c = opts.hydro
    oracle.bc_apply(c, w, PRIMITIVE)
    u1 = oracle.prim2cons(c, w)
    oracle.bc_apply(c, u1, CONSERVED)
    u2 = u1.copy()
    n0 = oracle.threads()
    oracle.set_threads(1)
    _run_steps(oracle, c, u1, 2)
    oracle.set_threads(max(n0, 3))
    _run_steps(oracle, c, u2, 2)
    oracle.set_threads(n0)
    np.testing.assert_array_equal(u1, u2)
