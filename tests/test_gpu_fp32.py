"""FP32 perturbation form against the FP64 plain form (both on the GPU,
same initial state, same dt sequence).

Reported per field: rel L1 = sum|a - b| / sum|b| and L-inf = max|a - b| /
max|b| over the interior.  Bounds: rel L1 <= 1e-5 on the full conserved
fields (the accuracy target of the FP32 form); the momentum fields are
themselves perturbations (zero base state), so their bound is the
perturbation bound, and the density / energy perturbations about the
reference are checked with a bound written at the call.
"""
import numpy as np
import pytest

from snapy_linfel_b200 import problems

from errnorm import rel_l1_linf

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _errors(a, b, it):
    return rel_l1_linf(np.stack([a[v][it] for v in range(a.shape[0])]),
                       np.stack([b[v][it] for v in range(b.shape[0])]))


def _run_pair(opts, w, r, dts, reference="mean"):
    from snapy_linfel_b200.mesh import MeshBlock, MeshBlockF32

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    m64 = MeshBlock(opts)
    m64.initialize(w, r)
    m32 = MeshBlockF32(opts)
    m32.initialize(w, r, reference=reference)
    for dt in dts:
        m64.step(dt)
        m32.step(dt)
    torch.cuda.synchronize()
    u64 = m64.hydro_u.cpu().numpy()
    u32 = m32.state64().cpu().numpy()
    rho_bar = m32.ref_rho.cpu().numpy()
    return u32, u64, rho_bar, m32, m64


def test_fp32_sod_plain():
    opts, w, _ = problems.sod(nx1=256)
    u32, u64, *_ = _run_pair(opts, w, None, [1e-3] * 20, reference=None)
    it = opts.hydro.interior()
    err = _errors(u32, u64, it)
    for v in (0, 4):
        assert err[v][0] < 1e-5, (v, err[v])


@pytest.mark.parametrize("riemann", ["lmars", "hllc", "roe"])
def test_fp32_straka_implicit(riemann):
    opts, w, _ = problems.straka(nx2=96, nx1=32, implicit_scheme=1, riemann=riemann)
    opts.hydro.nu_iso = opts.hydro.kappa_iso = 0.0
    u32, u64, rho_bar, *_ = _run_pair(opts, w, None, [0.5] * 10)
    it = opts.hydro.interior()
    err = _errors(u32, u64, it)
    for v in range(5):
        assert err[v][0] < 1e-5, (v, err[v])
    # density perturbation about the reference
    rp32 = u32[0][it] - rho_bar[None, None, it[2]]
    rp64 = u64[0][it] - rho_bar[None, None, it[2]]
    assert np.abs(rp32 - rp64).sum() / np.abs(rp64).sum() < 1e-3


@pytest.mark.parametrize("recon23", ["plm", "weno3"])
def test_fp32_run_time_dispatch(recon23):
    """A configuration outside the FP32 sweeps' compile-time face profiles
    (WENO3 along x1, whose pressure interpolation is the linear cp3 that the
    reference pressure needs, and PLM or WENO3 along x2), so every face takes
    the run-time reconstruction and solver dispatch: the same bounds as the
    profiled Straka runs."""
    from snapy_linfel_b200.config import RECON

    opts, w, _ = problems.straka(nx2=96, nx1=32, implicit_scheme=1, riemann="hllc")
    opts.hydro.nu_iso = opts.hydro.kappa_iso = 0.0
    opts.hydro.recon1_type = RECON["weno3"]
    opts.hydro.recon23_type = RECON[recon23]
    u32, u64, rho_bar, *_ = _run_pair(opts, w, None, [0.5] * 10)
    it = opts.hydro.interior()
    err = _errors(u32, u64, it)
    for v in range(5):
        assert err[v][0] < 1e-5, (v, err[v])
    rp32 = u32[0][it] - rho_bar[None, None, it[2]]
    rp64 = u64[0][it] - rho_bar[None, None, it[2]]
    assert np.abs(rp32 - rp64).sum() / np.abs(rp64).sum() < 1e-3


def test_fp32_3d_roe_vic_tracers():
    opts, w, r = problems.large_3d(nx3=24, nx2=24, nx1=48, nscalar=2)
    u32, u64, rho_bar, m32, m64 = _run_pair(opts, w, r, [0.5] * 6)
    it = opts.hydro.interior()
    err = _errors(u32, u64, it)
    for v in (0, 4):
        assert err[v][0] < 1e-5, (v, err[v])
    s32 = m32.scalar_s.cpu().numpy()
    s64 = m64.scalar_s.cpu().numpy()
    es = _errors(s32.astype(np.float64), s64, it)
    for n in range(2):
        assert es[n][0] < 1e-5, (n, es[n])
