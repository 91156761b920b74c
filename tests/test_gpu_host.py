"""The C++ host modules (libtorch, _snapb_host) against the CPU oracle."""
import numpy as np
import pytest

from snapy_linfel_b200 import problems
from snapy_linfel_b200.config import CONSERVED, PRIMITIVE

from errnorm import assert_finite, state_err

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _cfg_dict(c):
    from snapy_linfel_b200.config import config_dict

    return config_dict(c)


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


def test_host_fp32_block_and_ensemble_match_python_paths():
    """the C++ MeshBlockF32 and Ensemble (libtorch host code over the C ABI)
    advance exactly as the Python-driven FP32 block and ensemble"""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from snapy_linfel_b200 import _snapb_host
    from snapy_linfel_b200.ensemble import Ensemble
    from snapy_linfel_b200.mesh import MeshBlockF32

    members = problems.ensemble_members(n=3, seed=7, horiz=(16, 24), vert=(16, 32))
    cpp = []
    for opts, w, r in members:
        b = _snapb_host.MeshBlockF32(_cfg_dict(opts.hydro), opts.integration.cfl, 0)
        b.initialize(torch.from_numpy(w), None, "mean")
        cpp.append(b)
    # one block, two steps, against the Python FP32 block
    opts, w, r = members[0]
    py = MeshBlockF32(opts)
    py.initialize(w, r)
    solo = _snapb_host.MeshBlockF32(_cfg_dict(opts.hydro), opts.integration.cfl, 0)
    solo.initialize(torch.from_numpy(w), None, "mean")
    for _ in range(2):
        py.step()
        solo.step()
    torch.cuda.synchronize()
    assert torch.equal(py.hydro_u, solo.hydro_u)
    assert torch.equal(py.state64(), solo.state64())
    # the ensembles
    ens_py = Ensemble(members)
    ens_cpp = _snapb_host.Ensemble(cpp, members[0][0].integration.cfl)
    for _ in range(2):
        ens_py.step_eager()
        ens_cpp.step()
    torch.cuda.synchronize()
    assert torch.equal(ens_py.dts(), ens_cpp.dts())
    for a, b in zip(ens_py.blocks, cpp):
        assert bool(torch.isfinite(b.hydro_u).all())
        assert torch.equal(a.hydro_u, b.hydro_u)
    assert ens_cpp.cells() == ens_py.cells
