"""GPU parity against the CPU oracle at the benchmark configurations' full
sizes (FP64 plain form, through the C ABI).

* Sod shock tube, 1024 cells, WENO5 + HLLC, every step to t = 0.2;
* Straka density current, 1024 x 128 cells, WENO5 + LMARS, nu = kappa = 75,
  VIC 3x3, 20 steps;
* one full-size 128 x 128 x 128 warm-bubble member, WENO5 + LMARS, VIC 3x3,
  3 steps;
* the 384 x 384 x 192 H2-He domain with two tracers, WENO5 + Roe, VIC 3x3,
  one step.

Each step is checked from a shared state: before the step, the GPU block is
loaded with the oracle's state (hydro_u, hydro_w, scalars), both compute the
CFL dt (compared to 1e-12) and both advance one RK3 step with the oracle's
dt.  Two errors are reported per step and field v:

* relative to the state: max|u_gpu - u_orc| / scale_v(u), scale = density,
  sqrt(rho E) for the momenta, total energy (bound 1e-12, the FP64 target);
* relative to the step's own change: max|du_gpu - du_orc| / max|du_orc| with
  du = u_after - u_before (bound written at each test; the smallest changes,
  e.g. the vertical momentum of a resting hydrostatic column, are a
  cancellation of O(1) pressure and gravity terms, so their relative error
  is larger than the state's).

A free-running comparison (both sides take their own CFL dt) is reported for
Sod at t = 0.2.  Any NaN or Inf fails.  With SNAPB_PARITY_REPORT set to a
file name, the per-step errors are appended there as JSON lines.
"""
import json
import os

import numpy as np
import pytest

from snapy_linfel_b200 import problems
from snapy_linfel_b200.config import CONSERVED, PRIMITIVE, SCALAR

from errnorm import assert_finite, state_errs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _report(name, rows):
    path = os.environ.get("SNAPB_PARITY_REPORT")
    if not path:
        return
    with open(path, "a") as f:
        for r in rows:
            f.write(json.dumps(dict(case=name, **r)) + "\n")


class Lockstep:
    """the oracle block and the GPU block of one configuration, advanced
    step by step from the oracle's state"""

    def __init__(self, oracle, opts, w, r=None):
        from snapy_linfel_b200.mesh import MeshBlock

        if not torch.cuda.is_available():
            pytest.skip("no CUDA device")
        self.orc, self.opts = oracle, opts
        c = self.c = opts.hydro
        w = np.ascontiguousarray(w.copy())
        oracle.bc_apply(c, w, PRIMITIVE)
        self.w = w
        self.u = oracle.prim2cons(c, w)
        oracle.bc_apply(c, self.u, CONSERVED)
        self.u0 = np.empty_like(self.u)
        self.s = self.s0 = self.r = None
        if c.nscalar:
            self.r = np.ascontiguousarray(r.copy())
            oracle.bc_apply(c, self.r, SCALAR)
            self.s = np.ascontiguousarray(w[0:1] * self.r)
            oracle.bc_apply(c, self.s, SCALAR)
            self.s0 = np.empty_like(self.s)
        self.blk = oracle.block(c)
        self.mb = MeshBlock(opts)
        self.it = (slice(None),) + c.interior()

    def load_gpu(self):
        mb = self.mb
        mb.hydro_u.copy_(torch.from_numpy(self.u))
        mb.hydro_w.copy_(torch.from_numpy(self.w))
        if self.c.nscalar:
            mb.scalar_s.copy_(torch.from_numpy(self.s))
            mb.scalar_r.copy_(torch.from_numpy(self.r))

    def step(self, dt_override=None):
        """one step of both sides from the oracle's state; returns the
        per-field errors and the two dts"""
        c, it = self.c, self.it
        self.load_gpu()
        dt_orc = self.opts.integration.cfl * self.orc.max_time_step(c, self.w)
        dt_gpu = float(self.mb.max_time_step().item())
        dt = dt_orc if dt_override is None else dt_override
        before = self.u[it].copy()
        s_before = self.s[it].copy() if c.nscalar else None
        self.mb.set_dt(dt)
        for st in range(3):
            self.mb.forward(st)
            self.blk.stage(st, dt, self.u, self.u0, self.w, self.s, self.s0, self.r)
        torch.cuda.synchronize()
        got = self.mb.hydro_u.cpu().numpy()[it]
        want = self.u[it]
        assert_finite(got, what="GPU state")
        e_state = state_errs(got, want, want)
        d_got, d_want = got - before, want - before
        # a field whose change is below 1e-14 of the state (e.g. the
        # tangential momenta of the 1-D tube, exactly 0) is measured against
        # that floor instead of its own size
        floor = 1e-14 * np.abs(want).reshape(c.nvar, -1).max(axis=1)
        floor[1:4] = 1e-14 * np.max(np.abs(want[[0, 4]]))
        e_du = np.zeros(c.nvar)
        for v in range(c.nvar):
            den = max(np.abs(d_want[v]).max(), floor[v])
            e_du[v] = np.abs(d_got[v] - d_want[v]).max() / den
        row = dict(dt_orc=dt_orc, dt_gpu=dt_gpu, state=e_state.tolist(), du=e_du.tolist())
        if c.nscalar:
            sg = self.mb.scalar_s.cpu().numpy()[it]
            sw = self.s[it]
            assert_finite(sg, what="GPU scalars")
            row["scalar_state"] = float(np.abs(sg - sw).max() / np.abs(sw).max())
            ds_w = sw - s_before
            row["scalar_du"] = float(np.abs((sg - s_before) - ds_w).max() / np.abs(ds_w).max())
        return row


def _run_lockstep(name, oracle, opts, w, r=None, nsteps=None, tlim=None, du_bound=None,
                  state_bound=1e-12):
    ls = Lockstep(oracle, opts, w, r)
    rows, t, n = [], 0.0, 0
    while True:
        if nsteps is not None and n >= nsteps:
            break
        if tlim is not None and t >= tlim * (1 - 1e-14):
            break
        dt_override = None
        if tlim is not None:
            dt_next = opts.integration.cfl * oracle.max_time_step(ls.c, ls.w)
            if t + dt_next > tlim:
                dt_override = tlim - t
        row = ls.step(dt_override)
        t += row["dt_orc"] if dt_override is None else dt_override
        row.update(step=n, t=t)
        rows.append(row)
        n += 1
        assert abs(row["dt_gpu"] / row["dt_orc"] - 1.0) < 1e-12, (n, row)
        assert max(row["state"]) < state_bound, (n, row)
        if du_bound is not None:
            assert max(row["du"]) < du_bound, (n, row)
        if "scalar_state" in row:
            assert row["scalar_state"] < state_bound, (n, row)
    _report(name, rows)
    worst = dict(state=np.max([r["state"] for r in rows], axis=0).tolist(),
                 du=np.max([r["du"] for r in rows], axis=0).tolist(), steps=n)
    print(f"{name}: {n} steps, worst per-field state err {worst['state']}, "
          f"du err {worst['du']}")
    return ls, rows


def test_sod_1024_every_step_to_t02(oracle):
    opts, w, _ = problems.sod(nx1=1024)
    ls, rows = _run_lockstep("sod_1024", oracle, opts, w, tlim=0.2, du_bound=1e-12)
    assert rows[-1]["t"] == pytest.approx(0.2, rel=1e-14)
    assert len(rows) > 200


def test_sod_1024_free_running_to_t02(oracle):
    """both sides take their own CFL dt from their own state"""
    from snapy_linfel_b200.mesh import MeshBlock

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    opts, w, _ = problems.sod(nx1=1024)
    c = opts.hydro
    mb = MeshBlock(opts)
    mb.initialize(w)
    ww = np.ascontiguousarray(w.copy())
    oracle.bc_apply(c, ww, PRIMITIVE)
    u = oracle.prim2cons(c, ww)
    oracle.bc_apply(c, u, CONSERVED)
    blk = oracle.block(c)
    u0 = np.empty_like(u)
    t_g = t_o = 0.0
    n = 0
    while t_o < 0.2 * (1 - 1e-14):
        dto = min(opts.integration.cfl * oracle.max_time_step(c, ww), 0.2 - t_o)
        dtg = min(float(mb.max_time_step().item()), 0.2 - t_g)
        mb.step(dtg)
        for st in range(3):
            blk.stage(st, dto, u, u0, ww)
        t_g += dtg
        t_o += dto
        n += 1
    torch.cuda.synchronize()
    it = (slice(None),) + c.interior()
    got = mb.hydro_u.cpu().numpy()[it]
    e = state_errs(got, u[it], u[it])
    _report("sod_1024_free", [dict(steps=n, t_gpu=t_g, t_orc=t_o, state=e.tolist())])
    assert abs(t_g - t_o) < 1e-12
    assert float(np.max(e)) < 1e-12, e


def test_straka_1024x128_vic_diffusion_20_steps(oracle):
    opts, w, _ = problems.straka(nx2=1024, nx1=128, implicit_scheme=1)
    c = opts.hydro
    assert c.nu_iso == 75.0 and c.kappa_iso == 75.0
    _run_lockstep("straka_1024x128", oracle, opts, w, nsteps=20, du_bound=1e-7)


def test_warm_bubble_member_128x128x128_3_steps(oracle):
    opts, w, _ = problems.warm_bubble_3d(128, 128, 128, amp=2.5, radius=1.5e3,
                                          center=(6.4e3, 6.4e3, 3.0e3))
    _run_lockstep("warm_bubble_128^3", oracle, opts, w, nsteps=3, du_bound=1e-7)


def test_large_3d_384x384x192_two_tracers_one_step(oracle):
    opts, w, r = problems.large_3d()
    assert (opts.hydro.nx3, opts.hydro.nx2, opts.hydro.nx1, opts.hydro.nscalar) == (384, 384, 192, 2)
    _run_lockstep("large_3d_384x384x192", oracle, opts, w, r, nsteps=1, du_bound=1e-7)
