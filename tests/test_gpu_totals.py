"""Compensated conserved totals on the GPU (snapb_conserved_totals and
snapb_conserved_totals_f32) against exactly rounded host sums (math.fsum),
bit-identical repeats, and domain-total mass drift of the FP32 perturbation
form over a run, bounded by the reference's own example tolerance (mass
rtol 1e-8, tests/run_example_mass_check.py)."""
import math

import numpy as np
import pytest

from snapy_linfel_b200 import problems
from snapy_linfel_b200.config import make_config

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return "cuda"


def exact_totals(cfg, x):
    """vol * (exactly rounded interior sum) per variable, on the host"""
    it = (slice(None),) + cfg.interior()
    a = x[it]
    vol = ((cfg.x1max - cfg.x1min) / cfg.nx1) * ((cfg.x2max - cfg.x2min) / cfg.nx2) * (
        (cfg.x3max - cfg.x3min) / cfg.nx3)
    return [vol * math.fsum(a[v].ravel().tolist()) for v in range(a.shape[0])]


def test_totals_fp64_exactly_rounded(dev):
    from snapy_linfel_b200.mesh import conserved_totals

    cfg = make_config(nx1=64, nx2=40, nx3=12, x1=(0.0, 640.0), x2=(0.0, 400.0),
                      x3=(0.0, 120.0))
    rng = np.random.default_rng(3)
    x = rng.standard_normal(cfg.shape) * 10.0 ** rng.integers(-8, 9, cfg.shape)
    got = conserved_totals(cfg, torch.from_numpy(x).to(dev)).cpu().numpy()
    want = exact_totals(cfg, x)
    for v in range(cfg.nvar):
        assert abs(got[v] - want[v]) <= 2 * math.ulp(abs(want[v])), (v, got[v], want[v])


def test_totals_fp64_cancellation(dev):
    """+1e16, 1, -1e16 triples: a plain double sum loses the ones"""
    from snapy_linfel_b200.mesh import conserved_totals

    cfg = make_config(nx1=96, nx2=33, x1=(0.0, 96.0), x2=(0.0, 33.0))
    x = np.zeros(cfg.shape)
    it = (slice(None),) + cfg.interior()
    inner = x[it]
    flat = inner.reshape(cfg.nvar, -1)
    pattern = np.tile([1e16, 1.0, -1e16], flat.shape[1] // 3 + 1)[:flat.shape[1]]
    flat[:] = pattern
    x[it] = flat.reshape(inner.shape)
    got = conserved_totals(cfg, torch.from_numpy(x).to(dev)).cpu().numpy()
    want = exact_totals(cfg, x)
    for v in range(cfg.nvar):
        assert got[v] == want[v] == 1056.0, (v, got[v], want[v])


def test_totals_repeat_bit_identical(dev):
    from snapy_linfel_b200.mesh import conserved_totals

    cfg = make_config(nx1=128, nx2=128, nx3=24)
    x = torch.randn(cfg.shape, dtype=torch.float64, device=dev)
    a = conserved_totals(cfg, x)
    b = conserved_totals(cfg, x)
    assert torch.equal(a, b)


def test_totals_fp32_form_matches_fp64_state(dev):
    from snapy_linfel_b200.mesh import MeshBlockF32

    opts, w, r = problems.large_3d(nx3=16, nx2=16, nx1=48, nscalar=0)
    m32 = MeshBlockF32(opts)
    m32.initialize(w, r)
    for _ in range(2):
        m32.step(0.5)
    got = m32.totals().cpu().numpy()
    u = m32.state64().cpu().numpy()
    want = exact_totals(opts.hydro, u)
    mag = exact_totals(opts.hydro, np.abs(u))
    for v in range(opts.hydro.nvar):
        # state64 rounds u_bar + u' once per cell (2^-53 of each |u|); the
        # totals add u_bar and u' without that rounding
        assert abs(got[v] - want[v]) <= 4e-16 * mag[v] + 1e-300, (v, got[v], want[v], mag[v])


def test_fp32_form_mass_drift_within_reference_rtol(dev):
    from snapy_linfel_b200.mesh import MeshBlockF32

    opts, w, _ = problems.straka(nx2=128, nx1=32, implicit_scheme=1)
    opts.hydro.nu_iso = opts.hydro.kappa_iso = 0.0
    m32 = MeshBlockF32(opts)
    m32.initialize(w)
    m0 = float(m32.totals()[0])
    for _ in range(20):
        m32.step()
    m1 = float(m32.totals()[0])
    drift = abs(m1 / m0 - 1.0)
    print(f"FP32 form mass drift over 20 steps: {drift:.3e}")
    assert drift < 1e-8
