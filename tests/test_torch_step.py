"""CPU pin of the differentiable torch restatement of one RK stage
(oracle/torch_step.py) against the C++ oracle's stage, so that the torch
autograd gradient used to check the GPU adjoint differentiates the same
function the oracle computes.  Bound: 1e-10 of each variable's stage
increment (the two agree to ~1e-14; the implicit cases to ~1e-12, where the
mass redistribution subtracts nearly equal column sums)."""
import numpy as np
import pytest

from snapy_linfel_b200 import problems
from snapy_linfel_b200.config import CONSERVED, make_config

torch = pytest.importorskip("torch")

TOL = 1e-10

CASES = {
    "sod1d_weno5shock_hllc": dict(
        cfg=dict(nx1=24, x1=(0.0, 1.0), recon1="weno5", shock1=True, riemann="hllc",
                 bc=("outflow",) * 6), grav=False),
    "box2d_cp5_hllc": dict(
        cfg=dict(nx1=10, nx2=8, recon1="weno5", recon23="weno5", riemann="hllc",
                 bc=("reflecting", "outflow", "periodic", "periodic", "reflecting",
                     "reflecting")), grav=False),
    "box3d_roe": dict(
        cfg=dict(nx1=8, nx2=6, nx3=5, recon23="cp5", riemann="roe",
                 bc=("outflow", "reflecting", "periodic", "periodic", "outflow",
                     "reflecting")), grav=False),
    "col2d_lmars_vic3": dict(
        cfg=dict(nx1=16, nx2=12, x1=(0.0, 1600.0), x2=(0.0, 1200.0), gammad=1004.0 / 717.0,
                 rgas=287.0, recon1="weno5", recon23="weno5", riemann="lmars",
                 implicit_scheme=1, grav=(-9.81, 0.0, 0.0),
                 bc=("reflecting", "reflecting", "periodic", "periodic", "reflecting",
                     "reflecting")), grav=True),
    "box3d_hllc_vic3": dict(
        cfg=dict(nx1=10, nx2=6, nx3=6, x1=(0.0, 1000.0), x2=(0.0, 600.0), x3=(0.0, 600.0),
                 gammad=1004.0 / 717.0, rgas=287.0, riemann="hllc", implicit_scheme=1,
                 grav=(-9.81, 0.0, 0.0),
                 bc=("reflecting", "reflecting", "periodic", "periodic", "outflow",
                     "outflow")), grav=True),
}


def _field(shape, rng, modes=3):
    k3, k2, k1 = np.meshgrid(*[np.arange(n) / max(n, 1) for n in shape], indexing="ij")
    f = np.zeros(shape)
    for _ in range(modes):
        a = rng.uniform(0.5, 2.0, 3) * 2 * np.pi
        f += np.sin(a[0] * k1 + a[1] * k2 + a[2] * k3 + rng.uniform(0, 2 * np.pi))
    return f / modes


def primitive_state(cfg, seed, grav):
    """isentropic column plus smooth noise (grav), else a smooth gas"""
    rng = np.random.default_rng(seed)
    shape = cfg.shape[1:]
    w = np.zeros(cfg.shape)
    if grav:
        rd, cp = cfg.rgas, cfg.rgas * cfg.gammad / (cfg.gammad - 1.0)
        X1, _, _ = problems._grids(cfg)
        temp, p = problems._isentropic(X1, 1.0e5, 300.0, -cfg.grav1, rd, cp)
        temp = temp + 1.5 * _field(shape, rng)
        w[0] = p / (rd * temp)
        w[4] = p * (1.0 + 1e-3 * _field(shape, rng))
        vel = 5.0
    else:
        w[0] = 1.0 + 0.2 * _field(shape, rng)
        w[4] = 1.0 + 0.2 * _field(shape, rng)
        vel = 0.3
    for v in (1, 2, 3):
        w[v] = vel * _field(shape, rng)
    return w


def conserved(oracle, cfg, w):
    u = oracle.prim2cons(cfg, w)
    oracle.bc_apply(cfg, u, CONSERVED)
    return u


@pytest.mark.parametrize("stage", [0, 1, 2])
@pytest.mark.parametrize("name", list(CASES))
def test_torch_stage_matches_oracle(oracle, name, stage):
    from oracle import torch_step

    cfg = make_config(**CASES[name]["cfg"])
    grav = CASES[name]["grav"]
    u = conserved(oracle, cfg, primitive_state(cfg, 5 + stage, grav))
    u0 = u.copy() if stage == 0 else conserved(oracle, cfg, primitive_state(cfg, 40, grav))
    dt = 0.5 * oracle.max_time_step(cfg, oracle.cons2prim(cfg, u))
    ref, ref0, w = u.copy(), u0.copy(), np.empty_like(u)
    oracle.block(cfg).stage(stage, dt, ref, ref0, w)
    got = torch_step.stage(torch.from_numpy(u), torch.from_numpy(u0), stage, dt, cfg).numpy()
    W = torch_step.RK3[stage]
    inc = ref - (W[0] * u0 + W[1] * u)
    for v in range(5):
        scale = max(np.abs(inc[v]).max(), 1e-300)
        err = np.abs(got[v] - ref[v]).max() / scale
        assert err < TOL, f"{name} stage {stage} var {v}: {err:.2e}"


def test_torch_stage_refuses_uncovered_options():
    from oracle import torch_step

    cfg = make_config(nx1=8, nx2=6, implicit_scheme=9, grav=(-9.81, 0.0, 0.0))
    u = torch.zeros(cfg.shape, dtype=torch.float64)
    with pytest.raises(ValueError):
        torch_step.stage(u, u, 0, 1e-3, cfg)
