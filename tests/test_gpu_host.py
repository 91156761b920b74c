"""The C++ host modules (libtorch, _snapb_host) against the CPU oracle."""
import numpy as np
import pytest

from snapy_linfel_b200 import problems
from snapy_linfel_b200.config import CONSERVED, PRIMITIVE

from errnorm import assert_finite, state_err

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _cfg_dict(c):
    d = {f: getattr(c, f) for f, _ in c._fields_ if f not in ("bc", "disable_flux", "reserved")}
    d["bc"] = list(c.bc)
    d["disable_flux"] = list(c.disable_flux)
    return d


def test_host_meshblock_matches_oracle(oracle):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from snapy_linfel_b200 import _snapb_host

    opts, w, _ = problems.straka(nx2=48, nx1=16, implicit_scheme=1)
    c = opts.hydro
    mb = _snapb_host.MeshBlock(_cfg_dict(c), opts.integration.cfl, 0)
    mb.initialize(torch.from_numpy(w).cuda())
    for _ in range(3):
        mb.step(0.7)
    torch.cuda.synchronize()
    w0 = w.copy()
    oracle.bc_apply(c, w0, PRIMITIVE)
    u = oracle.prim2cons(c, w0)
    oracle.bc_apply(c, u, CONSERVED)
    blk = oracle.block(c)
    u0 = np.empty_like(u)
    for _ in range(3):
        for s in range(3):
            blk.stage(s, 0.7, u, u0, w0)
    it = (slice(None),) + c.interior()
    got = mb.hydro_u.cpu().numpy()[it]
    ref = u[it]
    assert state_err(got, ref, ref) < 3e-12
    assert mb.check_redo() == 0


def test_host_hydro_forward_and_dt(oracle):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from snapy_linfel_b200 import _snapb_host

    opts, w, _ = problems.sod(nx1=128)
    c = opts.hydro
    h = _snapb_host.Hydro(_cfg_dict(c))
    oracle.bc_apply(c, w, PRIMITIVE)
    u = oracle.prim2cons(c, w)
    oracle.bc_apply(c, u, CONSERVED)
    ug = torch.from_numpy(u).cuda()
    wg = torch.empty_like(ug)
    du = h.forward(1e-3, ug, wg)
    w_ref = np.empty_like(u)
    du_ref = oracle.block(c).hydro_forward(1e-3, u, w_ref)
    it = (slice(None),) + c.interior()
    assert_finite(du)
    assert np.abs(du.cpu().numpy()[it] - du_ref[it]).max() / np.abs(u).max() < 1e-13
    assert abs(h.max_time_step(wg) / oracle.max_time_step(c, w_ref) - 1) < 1e-13
