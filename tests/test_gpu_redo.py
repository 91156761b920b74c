"""Failure detection and step rejection (MeshBlockImpl::check_redo,
src/mesh/meshblock.cpp:974-1016), with the failure made on the host: after a
step, a bad value is written into hydro_u from the host, then check_redo is
asked for its verdict.  No kernel is made to fault.

The reference rejects the step when the interior holds a density <= 0, or
when its conserved energy screen (some E <= 0) trips and a cons2prim
pressure <= 0 confirms it.  On a rejection it restores hydro_u (and
scalar_s) from the stage-0 copies, counts current_redo up (the next CFL dt is
cfl * 2^-redo * limit), takes the step back off the cycle count, and returns
1; past max_redo it returns -1.  A healthy step resets current_redo to 0.
The stage-0 copies here keep the interior; the restore fills the ghost cells
from it with the boundary functions, so the restored array equals the state
at the start of the step everywhere, ghosts included.
"""
import numpy as np
import pytest

from snapy_linfel_b200 import problems

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _block(nscalar=0):
    from snapy_linfel_b200.mesh import MeshBlock

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if nscalar:
        opts, w, r = problems.large_3d(nx3=8, nx2=10, nx1=16, nscalar=nscalar)
    else:
        opts, w, r = problems.straka(nx2=48, nx1=16, implicit_scheme=1)
    mb = MeshBlock(opts)
    mb.initialize(w, r)
    return mb


def _dt_pair(mb):
    """(dt at the block's current_redo, dt at current_redo = 0) from the same
    hydro_w: the retried step's limit is the CFL limit of the state hydro_w
    holds (the last stage's input, as in the reference), scaled by 2^-redo"""
    d1 = float(mb.max_time_step().item())
    r = mb.current_redo
    mb.current_redo = 0
    d0 = float(mb.max_time_step().item())
    mb.current_redo = r
    mb.max_time_step()
    return d1, d0


def _cell(mb):
    c = mb.cfg
    return (c.nghost + 1 if c.nx3 > 1 else 0, c.nghost + 2 if c.nx2 > 1 else 0, c.nghost + 3)


def test_negative_density_rejects_and_restores_bit_for_bit():
    mb = _block(nscalar=2)
    mb.step()
    assert mb.check_redo() == 0
    mb.max_time_step()
    u_start = mb.hydro_u.clone()
    s_start = mb.scalar_s.clone()
    for s in range(3):
        mb.forward(s)
    mb.cycle += 1
    cycle = mb.cycle
    mb.hydro_u[(0,) + _cell(mb)] = -1.0  # planted on the host
    assert mb.check_redo() == 1
    assert torch.equal(mb.hydro_u, u_start)  # restored, ghosts included
    assert torch.equal(mb.scalar_s, s_start)
    assert mb.current_redo == 1
    assert mb.cycle == cycle - 1
    # the retried step's CFL dt carries the factor 2^-1
    d1, d0 = _dt_pair(mb)
    assert d1 == 0.5 * d0
    # a healthy retry clears the redo count
    for s in range(3):
        mb.forward(s)
    assert mb.check_redo() == 0
    assert mb.current_redo == 0


def test_negative_pressure_needs_the_energy_screen():
    """A negative pressure under a positive total energy passes, as in the
    reference (its energy screen does not trip); a non-positive energy with a
    negative pressure rejects the step."""
    mb = _block()
    u_start = mb.hydro_u.clone()
    mb.step()
    c = mb.cfg
    k, j, i = _cell(mb)
    rho = float(mb.hydro_u[0, k, j, i])
    en = float(mb.hydro_u[4, k, j, i])
    saved = mb.hydro_u.clone()
    # kinetic energy above E: p = (gamma-1)(E - KE) < 0 with E > 0
    mb.hydro_u[2, k, j, i] = np.sqrt(4.0 * rho * en)
    assert mb.check_redo() == 0
    mb.hydro_u.copy_(saved)
    mb.hydro_u[4, k, j, i] = -abs(en)
    assert mb.check_redo() == 1
    assert torch.equal(mb.hydro_u, u_start)


def test_gives_up_past_max_redo():
    mb = _block()
    mb.step()
    max_redo = mb.options.integration.max_redo
    for n in range(max_redo):
        d1, d0 = _dt_pair(mb)
        assert d1 == 2.0 ** -n * d0
        for s in range(3):
            mb.forward(s)
        mb.hydro_u[(0,) + _cell(mb)] = 0.0  # density <= 0 every time
        assert mb.check_redo() == 1
        assert mb.current_redo == n + 1
    for s in range(3):
        mb.forward(s)
    mb.hydro_u[(0,) + _cell(mb)] = -2.0
    assert mb.check_redo() == -1


def test_host_module_check_redo():
    """the C++ host module takes the same decisions"""
    from snapy_linfel_b200 import _snapb_host

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    opts, w, _ = problems.straka(nx2=48, nx1=16, implicit_scheme=1)
    c = opts.hydro
    d = {f: getattr(c, f) for f, _ in c._fields_ if f not in ("bc", "disable_flux", "reserved")}
    d["bc"] = list(c.bc)
    d["disable_flux"] = list(c.disable_flux)
    mb = _snapb_host.MeshBlock(d, opts.integration.cfl, 0)
    mb.initialize(torch.from_numpy(w).cuda())
    mb.step(0.5)
    assert mb.check_redo(5) == 0
    u_start = mb.hydro_u.clone()
    mb.step(0.5)
    cyc = mb.cycle
    mb.hydro_u[0, 0, c.nghost + 2, c.nghost + 3] = -1.0
    assert mb.check_redo(5) == 1
    assert torch.equal(mb.hydro_u, u_start)
    assert mb.cycle == cyc - 1
    mb.step(0.5)
    mb.hydro_u[0, 0, c.nghost + 2, c.nghost + 3] = -1.0
    assert mb.check_redo(0) == -1
