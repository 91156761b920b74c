"""Generate the golden fixtures under tests/golden/ from the reference's own
point kernels.

Run in a container that has the reference sources:

    make -C oracle ref            # builds oracle/_ref/libsnapref.so from
                                  # the reference's src/*/*_impl.h
    python tests/golden/make_golden.py

``oracle/_ref/libsnapref.so`` evaluates WENO5/WENO3/cp5/cp3 (interp_impl.h),
HLLC/LMARS/Roe (hllc_impl.h, lmars_impl.h, roe_impl.h), the ideal-gas
cons2prim (ideal_gas_impl.h) and the vertically implicit solve
(vic_assemble_{partial,full}_impl.h, forward_sweep_impl.h,
vic_redistribute_impl.h, math/{ludcmp,lubksb}.h, compiled against the Eigen
subset in oracle/ref_shim/Eigen) with the reference's code; the
orchestration around them (reconstruction grouping and edge fills, PLM,
divergence, forcing, boundary fills, RK3) is the oracle's.  Inputs are
seeded, so the fixtures are reproducible.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.pyoracle import Oracle  # noqa: E402
from snapy_linfel_b200 import problems  # noqa: E402
from snapy_linfel_b200.config import make_config  # noqa: E402


def random_prim(rng, shape):
    w = rng.random(shape)
    w[0] += 1.0
    w[4] += 1.0
    w[1:4] = (w[1:4] - 0.5) * 0.1
    return w


def main():
    R = Oracle("reference")
    assert R.lib.orc_kernels_kind() == 1
    rng = np.random.default_rng(20261203)
    out = {}
    # ---- reconstruction: every type, hydro grouping, all three axes ----
    cfg = make_config(nx1=5, nx2=4, nx3=3, nghost=3)
    w = random_prim(rng, cfg.shape)
    out["recon_w"] = w
    for name, t in (("weno5", 5), ("weno3", 4), ("plm", 1), ("cp5", 3), ("cp3", 2), ("dc", 0)):
        for shock in ((0, 1) if name.startswith("weno") else (0,)):
            c = cfg.copy()
            c.recon1_type = c.recon23_type = t
            c.recon1_shock = c.recon23_shock = shock
            for dim in (3, 2, 1):
                out[f"recon_{name}_s{shock}_d{dim}"] = R.reconstruct(c, dim, 0, w)
    c = cfg.copy()
    c.recon1_type = c.recon23_type = 5
    c.recon1_scale = c.recon23_scale = 1
    for dim in (3, 2, 1):
        out[f"recon_weno5scale_d{dim}"] = R.reconstruct(c, dim, 0, w)
    # scalar group: interp1 everywhere, clamped at 0
    c = cfg.copy()
    c.scalar_recon_type = 5
    sc = rng.random((2,) + cfg.shape[1:]) - 0.2
    out["recon_scalar_in"] = sc
    for dim in (3, 2, 1):
        out[f"recon_scalar_d{dim}"] = R.reconstruct(c, dim, 1, sc)
    # ---- Riemann solvers ----
    wl = random_prim(rng, cfg.shape)
    wr = random_prim(rng, cfg.shape)
    out["riemann_wl"], out["riemann_wr"] = wl, wr
    for name, s in (("roe", 0), ("lmars", 1), ("hllc", 2)):
        for dim in (3, 2, 1):
            f, p = R.riemann(cfg, s, dim, wl, wr)
            out[f"riemann_{name}_d{dim}_flx"] = f
            out[f"riemann_{name}_d{dim}_fp"] = p
    vel = rng.standard_normal(cfg.shape[1:])
    out["riemann_vel"] = vel
    f, _ = R.riemann(cfg, 3, 3, wl, wr, vel=vel, face_pressure=False)
    out["riemann_upwind_d3_flx"] = f
    # ---- EOS ----
    u = R.prim2cons(cfg, w)
    out["eos_u"] = u
    out["eos_w"] = R.cons2prim(cfg, u)
    # ---- Sod shock tube: 30 RK3 steps at 256 cells ----
    opts, w0, _ = problems.sod(nx1=256)
    c = opts.hydro
    w0 = w0.copy()
    R.bc_apply(c, w0, 0)
    u = R.prim2cons(c, w0)
    R.bc_apply(c, u, 1)
    out["sod_u_init"] = u.copy()
    blk = R.block(c)
    u0 = np.empty_like(u)
    dts = []
    for _ in range(30):
        dt = 0.9 * R.max_time_step(c, w0)
        dts.append(dt)
        for s in range(3):
            blk.stage(s, dt, u, u0, w0)
    out["sod_dts"] = np.array(dts)
    out["sod_u_final"] = u
    # ---- small Straka with gravity, diffusion and the implicit solves ----
    for scheme in (0, 1, 9):
        opts, w0, _ = problems.straka(nx2=24, nx1=12, implicit_scheme=scheme)
        c = opts.hydro
        R.bc_apply(c, w0, 0)
        u = R.prim2cons(c, w0)
        R.bc_apply(c, u, 1)
        blk = R.block(c)
        u0 = np.empty_like(u)
        out[f"straka{scheme}_u_init"] = u.copy()
        dts = []
        for _ in range(4):
            dt = 0.9 * R.max_time_step(c, w0)
            dts.append(dt)
            for s in range(3):
                blk.stage(s, dt, u, u0, w0)
        out[f"straka{scheme}_dts"] = np.array(dts)
        out[f"straka{scheme}_u_final"] = u
    # ---- the implicit correction alone (schemes 1 and 9): a Straka column
    # set with a seeded flow and a noisy explicit tendency, and a 3-D box ----
    for scheme in (1, 9):
        for case in ("straka", "box"):
            if case == "straka":
                opts, w0, _ = problems.straka(nx2=16, nx1=20, implicit_scheme=scheme)
            else:
                opts, w0, _ = problems.warm_bubble_3d(4, 5, 12, amp=2.0, radius=500.0,
                                                       center=(200.0, 250.0, 500.0),
                                                       implicit_scheme=scheme)
            c = opts.hydro
            w0[1:4] += 0.3 * rng.standard_normal(w0[1:4].shape)
            R.bc_apply(c, w0, 0)
            u = R.prim2cons(c, w0)
            R.bc_apply(c, u, 1)
            ce = c.copy()
            ce.implicit_scheme = 0
            wf = np.empty_like(u)
            du = R.block(ce).hydro_forward(2.0, u, wf)
            du += 1e-3 * rng.standard_normal(du.shape) * np.abs(du).max(axis=(1, 2, 3),
                                                                      keepdims=True)
            key = f"vic{scheme}_{case}"
            out[key + "_w"], out[key + "_du_in"] = wf, du.copy()
            mass = np.zeros_like(u)
            R.implicit_correction(c, 2.0, du, wf, mass)
            out[key + "_du_out"], out[key + "_mass"] = du, mass
    path = os.path.join(HERE, "ref_kernels.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
