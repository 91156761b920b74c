"""The module-level Python surface (snapy_linfel_b200.modules: Hydro,
Reconstruct, RiemannSolver, ImplicitHydro, EquationOfState) against the CPU
oracle, on the GPU: the same bounds as the C-ABI parity tests (1e-13 per
field for single operators, 1e-12 of the state for a tendency)."""
import numpy as np
import pytest

from snapy_linfel_b200 import problems
from snapy_linfel_b200.config import CONSERVED, PRIMITIVE

from errnorm import assert_finite, relerr

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _rel(a, b):
    return relerr(a, b)


@pytest.fixture(scope="module")
def case(oracle):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    opts, w, _ = problems.straka(nx2=40, nx1=24, implicit_scheme=1)
    c = opts.hydro
    # a seeded flow on the resting column, so no flux is an exact zero that
    # one side rounds differently
    rng = np.random.default_rng(8)
    w[1:4] += rng.standard_normal(w[1:4].shape)
    w[0] *= 1.0 + 0.01 * rng.standard_normal(w[0].shape)
    oracle.bc_apply(c, w, PRIMITIVE)
    u = oracle.prim2cons(c, w)
    oracle.bc_apply(c, u, CONSERVED)
    return opts, w, u


def test_eos_module(case, oracle):
    from snapy_linfel_b200.modules import EquationOfState

    opts, w, u = case
    eos = EquationOfState(opts)
    wg = eos.compute("U->W", [torch.from_numpy(u).cuda()])
    assert _rel(wg.cpu().numpy(), oracle.cons2prim(opts.hydro, u)) < 1e-13
    ug = eos.compute("W->U", [wg])
    assert _rel(ug.cpu().numpy(), u) < 1e-13
    with pytest.raises(ValueError):
        eos.compute("W->T", [wg])
    with pytest.raises(Exception):
        eos.compute("U->W", [torch.from_numpy(u)])  # CPU tensor: no CPU path


def test_reconstruct_and_riemann_modules(case, oracle):
    from snapy_linfel_b200.modules import Reconstruct, RiemannSolver

    opts, w, u = case
    c = opts.hydro
    wg = torch.from_numpy(w).cuda()
    rec = Reconstruct(opts)
    rs = RiemannSolver(opts)
    for dim in (3, 2):
        wlr = rec(wg, dim)
        ref = oracle.reconstruct(c, dim, 0, w)
        it = (slice(None), slice(None)) + c.interior()
        assert _rel(wlr.cpu().numpy()[it].reshape(2 * 5, -1),
                    ref[it].reshape(2 * 5, -1)) < 1e-13
        flx = torch.empty_like(wg)
        fp = torch.empty(wg.shape[1:], dtype=torch.float64, device="cuda")
        rs(wlr[0].contiguous(), wlr[1].contiguous(), dim, flx, fp)
        ref_f, ref_p = oracle.riemann(c, c.riemann, dim, np.ascontiguousarray(ref[0]),
                                      np.ascontiguousarray(ref[1]))
        ii = (slice(None),) + c.interior()
        assert _rel(flx.cpu().numpy()[ii], ref_f[ii]) < 1e-12


def test_hydro_and_implicit_modules(case, oracle):
    from snapy_linfel_b200.modules import Hydro, ImplicitHydro

    opts, w, u = case
    c = opts.hydro
    hyd = Hydro(opts)
    ug = torch.from_numpy(u).cuda()
    du = hyd(0.5, ug)
    w_ref = np.empty_like(u)
    du_ref = oracle.block(c).hydro_forward(0.5, u, w_ref)
    it = (slice(None),) + c.interior()
    scale = np.abs(u[it]).max(axis=(1, 2, 3), keepdims=True)
    assert_finite(du)
    assert (np.abs(du.cpu().numpy()[it] - du_ref[it]) / scale).max() < 1e-12
    # CFL limit of the primitive state
    dt = hyd.max_time_step(torch.from_numpy(w_ref).cuda())
    assert dt > 0.0
    # the implicit correction as a difference, on the explicit tendency
    cexp = c.copy()
    cexp.implicit_scheme = 0
    w_full = np.empty_like(u)
    du_e = oracle.block(cexp).hydro_forward(0.5, u, w_full)
    corr = ImplicitHydro(opts)(torch.from_numpy(du_e).cuda(), torch.from_numpy(w_full).cuda(),
                               0.5)
    ref = du_e.copy()
    oracle.implicit_correction(c, 0.5, ref, w_full)
    assert_finite(corr)
    assert (np.abs(corr.cpu().numpy()[it] - (ref - du_e)[it]) / scale).max() < 1e-12
