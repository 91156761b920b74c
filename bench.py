"""Benchmark of the hydro forward step (one JSON line on rank 0).

Workload (default ``c3``): the batched ensemble of the benchmark
configurations — 48 independent 3-D dry warm-bubble domains of seeded uneven
sizes ({64,96,128}^2 x {64,128}, 48.2 M cells in all), WENO5 + LMARS,
vertically implicit solve (3x3 VIC), doubly periodic, CFL 0.8.  The head
value is the batched FP32 perturbation form (one persistent launch per sweep
over all members, the step replayed from a CUDA graph, tile shapes picked by
the autotuner); the plain FP64 form (member after member through
snapb_stage) runs the same members beside it, and both are compared field by
field over a few steps with the same dt.  A "step" is one RK3 step (3 stages)
of every member; the unit counts interior cells x RK stages.  The line also
carries the adjoint/forward time of the 2-D warm-bubble adjoint workload
(512 x 256, WENO5 + HLLC, vertical implicit).

Other workloads: ``c3s`` (the first 12 members, for profiling captures),
``c5`` (384 x 384 x 192 H2-He single domain, WENO5 + Roe, 2 tracers; FP32
form vs FP64 form and the adjoint on that domain), ``c5s``, ``c2``, ``c1``.

Arms:
  --impl ours       (default) the CUDA path through the C ABI
  --impl reference  the reference's CPU implementation of the path: the
                    oracle/_ref build (the reference's own *_impl.h kernels
                    under the restated orchestration), all host threads, on a
                    bounded sub-domain of the same workload.
Multi-GPU (one process per GPU): the ensemble's members are sharded over
the ranks by size (no data-path exchange; the step is the whole ensemble,
``scaling: strong``); a single-domain workload is split into x2 slabs with
the ghost exchange after every stage and a MIN all-reduce of dt
(``--decomp slab``, ``scaling: strong``) or run as replicas
(``--decomp replicas``, ``scaling: weak``).  Every time is the maximum over
the ranks of CUDA-event durations.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "Mcell-updates/s batched FP32 vs plain FP64 at rel L1<=1e-5; adjoint/fwd time"
UNIT = "Mcell-updates/s"


WORKLOAD_DESC = {
    "c3": "ensemble_48_warm_bubbles_3d_{64,96,128}^2x{64,128}_weno5_lmars_vic3",
    "c3s": "ensemble_first_12_of_48_warm_bubbles_3d_weno5_lmars_vic3",
    "c4": "adjoint_bubble_2d_512x256_weno5_hllc_vic3_200steps",
    "c5": "large_3d_h2he_384x384x192_weno5_roe_vic3_2tracers",
    "c5s": "large_3d_h2he_96x96x192_weno5_roe_vic3_2tracers",
    "c2": "straka_1024x128_weno5_lmars_vic3_diffusion",
    "c1": "sod_1024_weno5_hllc",
}


def workload(name: str):
    from snapy_linfel_b200 import problems

    if name == "c5":
        opts, w, r = problems.large_3d()
        desc = "large_3d_h2he_384x384x192_weno5_roe_vic3_2tracers"
    elif name == "c5s":  # smaller variant for quick checks
        opts, w, r = problems.large_3d(nx3=96, nx2=96, nx1=192)
        desc = "large_3d_h2he_96x96x192_weno5_roe_vic3_2tracers"
    elif name == "c2":
        opts, w, r = problems.straka()
        desc = "straka_1024x128_weno5_lmars_vic3_diffusion"
    elif name == "c1":
        opts, w, r = problems.sod()
        desc = "sod_1024_weno5_hllc"
    else:
        raise SystemExit(f"unknown workload {name}")
    return opts, w, r, desc


def interior_cells(cfg) -> int:
    return cfg.nx1 * cfg.nx2 * cfg.nx3


def algo_bytes_per_cell_update(cfg, elem=8) -> int:
    """Compulsory traffic of one fused RK stage: read u, read u0, write u."""
    return 3 * (cfg.nvar + cfg.nscalar) * elem


def kernel_io_bytes_per_cell(name, cfg, elem=8) -> int:
    """The bytes a stage kernel must move per interior cell given the
    kernel split (its inputs and outputs, each once), reported beside the
    roofline; the roofline itself uses the fused-stage bytes of
    algo_bytes_per_cell_update.

    x1 sweep: read u, s; write w, r and the x1 flux sums (3 NV values).
    x2/x3 sweep: read w, r and the running sums; write the sums (3 NV values).
    implicit_vic (one fused kernel: blocks, elimination, redistribution, RK
    update): read w, du, u, u0, and per scalar s, s0, r, ds; write u, s, r;
    the FP64 plain form also writes the FP64 mass correction.
    """
    nv = cfg.nvar + cfg.nscalar
    ns = cfg.nscalar
    if name in ("x1_sweep", "x2_sweep", "x3_sweep"):
        return 3 * nv * elem
    if name == "implicit_vic":
        return (5 + 5 + 5 + 5 + 4 * ns + 5 + 2 * ns) * elem + (8 if elem == 8 else 0)
    return 0


def launches_per_step(cfg) -> int:
    diff = cfg.nu_iso > 0 or cfg.kappa_iso > 0
    a2, a3 = cfg.nx2 > 1, cfg.nx3 > 1
    sep_final = (not a2 and not a3) and diff
    per_stage = 1 + int(diff) + int(a2) + int(a3) + int(sep_final) + 3 * int(cfg.implicit_scheme != 0)
    per_stage += 1 + int(cfg.nscalar > 0)  # boundary fills of u (and s)
    return 3 * per_stage + 4  # + CFL fill / reduce / final + dt scaling


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
              "timestamp")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None
        return self

    def mark_start(self):
        """the timed region starts now (samples outside it are dropped)"""
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def _in_window(self, stamp):
        if self.t0 is None or self.t1 is None:
            return True
        try:
            t = datetime.datetime.strptime(stamp.strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return True
        return self.t0 - 0.06 <= t <= self.t1 + 0.06

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) > 9 and not self._in_window(f[9]):
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------------------
# CPU arm / baseline (the checker's builds; only bench.py's baseline legs run them)
# --------------------------------------------------------------------------
def cpu_sample_problem(workload_name: str, nx_h: int = 64):
    """A bounded sub-domain of a workload for the host-core timing."""
    from snapy_linfel_b200 import problems

    if workload_name in ("c3", "c3s"):
        m = problems.ensemble(n=1, seed=2024)[0]
        m.update(nx3=nx_h, nx2=nx_h, nx1=64)
        opts, w, _ = problems.warm_bubble_3d(**m)
        return opts, w, None, (f"one {nx_h}x{nx_h}x64 member of the same ensemble "
                               "(WENO5+LMARS+VIC3)")
    opts, w, r = problems.large_3d(nx3=nx_h, nx2=nx_h, nx1=192)
    return opts, w, r, (f"{nx_h}x{nx_h}x192 sub-domain of the same workload "
                        "(WENO5+Roe+VIC3+2 tracers)")


def cpu_sample_run(kind: str, steps: int, warmup: int, threads: int | None = None,
                   nx_h: int = 64, workload_name: str = "c5"):
    """Time RK3 steps of a bounded sub-domain of the workload on the host."""
    from oracle.pyoracle import Oracle
    from snapy_linfel_b200.config import CONSERVED, PRIMITIVE, SCALAR

    orc = Oracle(kind)
    nthreads = threads or os.cpu_count() or 1
    orc.set_threads(nthreads)
    opts, w, r, what = cpu_sample_problem(workload_name, nx_h)
    c = opts.hydro
    orc.bc_apply(c, w, PRIMITIVE)
    u = orc.prim2cons(c, w)
    orc.bc_apply(c, u, CONSERVED)
    u0 = np.empty_like(u)
    s = s0 = None
    if c.nscalar:
        orc.bc_apply(c, r, SCALAR)
        s = w[0:1] * r
        orc.bc_apply(c, s, SCALAR)
        s0 = np.empty_like(s)
    else:
        r = None
    blk = orc.block(c)
    times = []
    for n in range(warmup + steps):
        t0 = time.perf_counter()
        dt = opts.integration.cfl * orc.max_time_step(c, w)
        for st in range(3):
            blk.stage(st, dt, u, u0, w, s, s0, r)
        if n >= warmup:
            times.append(time.perf_counter() - t0)
    cells = interior_cells(c)
    per_step = statistics.median(times)
    value = cells * 3 / per_step / 1e6
    sample = f"{what}, {steps} RK3 step(s), median wall time"
    return value, per_step, nthreads, sample, orc.kind


def run_reference(args):
    from oracle.pyoracle import lib_path

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    desc = WORKLOAD_DESC[args.workload]
    kind = "reference" if os.path.exists(lib_path("reference")) else "port"
    value, per_step, cores, sample, _ = cpu_sample_run(kind, args.steps, args.warmup,
                                                       workload_name=args.workload)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "form": "plain_fp64", "cpu_sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------
_STATE_CACHE = {}


def workload_state(name):
    """The initial (w, r) of a workload, kept so both forms start alike."""
    return _STATE_CACHE.get(name)


def rel_errors(a, b, it):
    """per-field rel L1 and L-inf over the interior (it: the 3-D interior index)"""
    out = {"rel_l1": [], "linf": []}
    for v in range(a.shape[0]):
        x, y = a[v][it], b[v][it]
        out["rel_l1"].append(float((x - y).abs().sum() / y.abs().sum().clamp_min(1e-300)))
        out["linf"].append(float((x - y).abs().max() / y.abs().max().clamp_min(1e-300)))
    return out


# DRAM bytes per interior cell of one launch (dram__bytes_read.sum +
# dram__bytes_write.sum) of the batched FP32 kernels, from one-kernel ncu
# captures of the first 12 ensemble members, scaled to a launch by the cells
# it processes (their traffic grows in proportion to the cells).  None: not
# captured for the current build.
# member groups of the end-to-end form (copies of one group overlap the others' steps)
E2E_GROUPS = 4

NCU_TRAFFIC_PER_CELL_F32 = {"x1_sweep": 69.3, "x2_sweep": 66.1, "x3_sweep": 66.1,
                            "implicit_vic": 347.2}


def dominant_roofline(kern, cfg, cells, elem, peak, peak_src):
    """Roofline line of the kernel with the largest share of the timed region:
    achieved = the fused stage's algorithmic bytes per cell update (read u,
    read u0, write u: 3 (nvar + nscalar) values) x the cells of one launch,
    over the launch's CUDA-event duration."""
    if not kern:
        return None
    name, (tot_ms, n) = max(kern.items(), key=lambda kv: kv[1][0])
    per_launch_s = tot_ms / n / 1e3
    per_cell = algo_bytes_per_cell_update(cfg, elem)
    ach = per_cell * cells / per_launch_s / 1e9
    share = tot_ms / sum(v[0] for v in kern.values())
    traffic = None
    if elem == 4 and NCU_TRAFFIC_PER_CELL_F32.get(name) is not None:
        traffic = NCU_TRAFFIC_PER_CELL_F32[name] * cells
    io = kernel_io_bytes_per_cell(name, cfg, elem)
    return {"kernel": name, "bound": "hbm", "achieved": ach, "peak": peak,
            "peak_source": peak_src, "unit": "GB/s", "frac": ach / peak,
            "traffic": traffic,
            "traffic_source": ("one-kernel ncu capture of the first 12 ensemble members, "
                               "DRAM bytes per cell x cells" if traffic is not None else None),
            "algorithmic_bytes_per_cell": per_cell,
            "kernel_io_bytes_per_cell": io,
            "kernel_io_frac": io * cells / per_launch_s / 1e9 / peak,
            "cells_per_launch": cells, "ms_per_launch": per_launch_s * 1e3,
            "share_of_timed_kernels": share}


def run_fp32_form(args, opts, state, mb64, cells, stream, barrier, world):
    import torch

    from snapy_linfel_b200 import _lib
    from snapy_linfel_b200.mesh import MeshBlock, MeshBlockF32

    w, r = state
    m32 = MeshBlockF32(opts, device=mb64.device)
    m32.initialize(w, r)
    for _ in range(args.warmup):
        m32.step()
    barrier()
    _lib.timing_enable(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        m32.step()
    e1.record(stream)
    barrier()
    ms = e0.elapsed_time(e1)
    kern_raw = _lib.timing_query()
    kern = {k: round(v[0] / v[1], 4) for k, v in kern_raw.items()}
    _lib.timing_enable(False)
    # e2e with host buffers (the FP32 perturbation state is the API's state)
    hu = torch.empty(opts.hydro.shape, dtype=torch.float32).pin_memory()
    hu.copy_(m32.hydro_u.cpu())
    hs = None
    if opts.hydro.nscalar:
        hs = torch.empty(opts.hydro.scalar_shape, dtype=torch.float32).pin_memory()
        hs.copy_(m32.scalar_s.cpu())
    nbytes = hu.numel() * 4 + (hs.numel() * 4 if hs is not None else 0)
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        m32.hydro_u.copy_(hu, non_blocking=True)
        if hs is not None:
            m32.scalar_s.copy_(hs, non_blocking=True)
        m32.step()
        hu.copy_(m32.hydro_u, non_blocking=True)
        if hs is not None:
            hs.copy_(m32.scalar_s, non_blocking=True)
    e1.record(stream)
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    e2e = world * cells * 3 * args.steps / (e2e_ms / 1e3) / 1e6
    # accuracy: both forms from the same initial state, same dt sequence
    a64 = MeshBlock(opts, device=mb64.device)
    a64.initialize(w, r)
    a32 = MeshBlockF32(opts, device=mb64.device)
    a32.initialize(w, r)
    for _ in range(args.acc_steps):
        dt = a64.max_time_step().clone()
        a64.step(dt)
        a32.step(dt)
    torch.cuda.synchronize()
    it = (slice(None),) + opts.hydro.interior()
    acc = rel_errors(a32.state64(), a64.hydro_u, it[1:])
    acc["steps"] = args.acc_steps
    if opts.hydro.nscalar:
        sacc = rel_errors(a32.scalar_s.double(), a64.scalar_s, it[1:])
        acc["scalar_rel_l1"] = sacc["rel_l1"]
    # perturbation fields: density about the reference, momenta
    rb = a32.ref_rho.view(1, 1, -1)
    rp32 = (a32.state64()[0] - rb)[it[1:]]
    rp64 = (a64.hydro_u[0] - rb)[it[1:]]
    acc["rho_prime_rel_l1"] = float((rp32 - rp64).abs().sum() / rp64.abs().sum())
    del a64, a32
    return {"ms": ms, "kern": kern, "kern_raw": kern_raw, "acc": acc,
            "e2e": {"value": e2e, "unit": UNIT}, "h2d": nbytes, "d2h": nbytes}


def run_adjoint_timing(args, opts, state, cells, stream, barrier):
    """FP64 adjoint cost on the same workload: one RK3 step forward vs the
    reverse of that step (three stage reverses from the kept stage inputs),
    and the checkpointed rollout's backward (segment re-run + reverses)."""
    import torch

    from snapy_linfel_b200 import _lib
    from snapy_linfel_b200.adjoint import StepRunner, rollout
    from snapy_linfel_b200.mesh import MeshBlock

    w, r = state
    mb = MeshBlock(opts, device="cuda")
    mb.initialize(w, r)
    dt = mb.max_time_step().clone()
    u0 = mb.hydro_u.clone()
    s0 = mb.scalar_s.clone() if opts.hydro.nscalar else None
    del mb
    runner = StepRunner(opts, device="cuda")
    adj = runner.adjoint()
    nsteps = max(1, min(args.steps, args.adj_steps)) if cells >= 1_000_000 else 10
    runner.load(u0, s0)
    for _ in range(2):  # warm-up
        runner.step(dt)
    runner.load(u0, s0)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(nsteps):
        runner.step(dt)
    e1.record(stream)
    barrier()
    fwd_ms = e0.elapsed_time(e1) / nsteps
    runner.load(u0, s0)
    kept = [runner.step(dt, keep=True) for _ in range(nsteps)]
    g = torch.ones_like(u0) * 1e-3
    gs = torch.ones_like(s0) * 1e-3 if s0 is not None else None
    # warm-up reverse
    gu0 = torch.zeros_like(g)
    gs0 = torch.zeros_like(gs) if gs is not None else None
    adj.stage(2, dt, kept[-1][2][0], kept[-1][2][1], g, gs, gu0, gs0)
    barrier()
    _lib.timing_enable(True)
    e0.record(stream)
    gg, ggs = g, gs
    for n in reversed(range(nsteps)):
        gu0 = torch.zeros_like(g)
        gs0 = torch.zeros_like(gs) if gs is not None else None
        for st in (2, 1, 0):
            gg, ggs = adj.stage(st, dt, kept[n][st][0], kept[n][st][1], gg, ggs, gu0, gs0)
        gg = gg + gu0
        if ggs is not None:
            ggs = ggs + gs0
    e1.record(stream)
    barrier()
    rev_ms = e0.elapsed_time(e1) / nsteps
    kern = {k: round(v[0] / v[1], 4) for k, v in _lib.timing_query().items()}
    _lib.timing_enable(False)
    del kept
    # the checkpointed rollout: forward + backward through torch.autograd
    dts = dt.repeat(nsteps)
    xw = u0.clone().requires_grad_(True)  # warm-up: first launches of every kernel
    uw, _ = rollout(opts, xw, s0, dts, checkpoint_every=nsteps, runner=runner)
    uw.backward(torch.ones_like(uw) * 1e-3)
    del xw, uw
    x = u0.clone().requires_grad_(True)
    barrier()
    e0.record(stream)
    uT, _ = rollout(opts, x, s0, dts, checkpoint_every=nsteps, runner=runner)
    e1.record(stream)
    barrier()
    roll_fwd_ms = e0.elapsed_time(e1) / nsteps
    e0.record(stream)
    uT.backward(torch.ones_like(uT) * 1e-3)
    e1.record(stream)
    barrier()
    roll_bwd_ms = e0.elapsed_time(e1) / nsteps
    del x, uT
    # the same rollout keeping every step's stage inputs (no re-run backwards)
    x = u0.clone().requires_grad_(True)
    barrier()
    e0.record(stream)
    uT, _ = rollout(opts, x, s0, dts, checkpoint_every=0, runner=runner)
    e1.record(stream)
    barrier()
    keep_fwd_ms = e0.elapsed_time(e1) / nsteps
    e0.record(stream)
    uT.backward(torch.ones_like(uT) * 1e-3)
    e1.record(stream)
    barrier()
    keep_bwd_ms = e0.elapsed_time(e1) / nsteps
    del x, uT, runner, adj
    torch.cuda.empty_cache()
    return {"steps": nsteps, "forward_ms_per_step": fwd_ms, "reverse_ms_per_step": rev_ms,
            "adjoint_over_forward": rev_ms / fwd_ms,
            "checkpointed": {"forward_ms_per_step": roll_fwd_ms,
                             "backward_ms_per_step": roll_bwd_ms,
                             "backward_over_forward": roll_bwd_ms / roll_fwd_ms,
                             "checkpoint_every": nsteps},
            "stage_inputs_kept": {"forward_ms_per_step": keep_fwd_ms,
                                  "backward_ms_per_step": keep_bwd_ms,
                                  "backward_over_forward": keep_bwd_ms / fwd_ms,
                                  "memory": "3 states per step kept by the forward pass"},
            "reverse_kernel_ms_per_stage": kern, "dtype": "f64",
            "value": cells * 3 / (rev_ms / 1e3) / 1e6, "unit": "Mcell-updates/s (reverse)"}


def ensemble_launches_per_step(cfg, tuning=None) -> int:
    """kernels of one batched step: CFL fill + reduce + final, then per stage
    the x1 ghost revision (gravity along x1), the x1, x2, x3 sweeps, the
    implicit solve (one cyclic-reduction or fused launch, or column + finish)
    and the boundary fill(s)"""
    kernel = (tuning or {}).get("vic_kernel", 0)
    cyclic = (kernel == 1 and cfg.implicit_scheme and not (cfg.implicit_scheme >> 3) & 1
              and cfg.nx1 <= 256)
    vic = 1 if kernel == 2 or cyclic else 2
    per_stage = (1 + int(cfg.grav1 != 0) + int(cfg.nx2 > 1) + int(cfg.nx3 > 1) +
                 (vic if cfg.implicit_scheme else 0) + 1 + int(cfg.nscalar > 0))
    return 3 + 3 * per_stage


def cpu_baseline_block(workload_name):
    """the reference CPU path on the host cores (all threads, and one
    thread), on a bounded sample of the workload"""
    try:
        from oracle.pyoracle import lib_path

        kind = "reference" if os.path.exists(lib_path("reference")) else "port"
        v, per_step, cores, sample, _ = cpu_sample_run(kind, 1, 0, workload_name=workload_name)
        v1, per1, _, sample1, _ = cpu_sample_run(kind, 1, 0, threads=1,
                                                 workload_name=workload_name, nx_h=32)
        return {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample,
                "single_core": {"value": v1, "unit": UNIT, "cores": 1, "sample": sample1}}
    except Exception as e:  # the baseline is reported, never required
        return {"value": None, "unit": UNIT, "cores": None, "kind": None,
                "sample": f"failed: {e}"}


def run_single_domain_forms(args, stream, barrier, nx=(384, 384, 192), acc_steps=10):
    """The 384 x 384 x 192 H2-He domain (WENO5 + Roe + VIC, two tracers):
    the FP64 plain form and the FP32 perturbation form timed on the same
    state, and compared per field after acc_steps steps with the same dt."""
    import torch

    from snapy_linfel_b200 import problems
    from snapy_linfel_b200.mesh import MeshBlock, MeshBlockF32

    opts, w, r = problems.large_3d(nx3=nx[0], nx2=nx[1], nx1=nx[2])
    cells = interior_cells(opts.hydro)
    steps = max(1, min(args.steps, 5))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"workload": WORKLOAD_DESC["c5"], "steps": steps}
    for name, cls in (("fp64_plain", MeshBlock), ("fp32_perturbation", MeshBlockF32)):
        mb = cls(opts, device="cuda")
        mb.initialize(w, r)
        for _ in range(args.warmup):
            mb.step()
        barrier()
        ev0.record(stream)
        for _ in range(steps):
            mb.step()
        ev1.record(stream)
        barrier()
        ms = ev0.elapsed_time(ev1)
        out[name] = {"value": cells * 3 * steps / (ms / 1e3) / 1e6,
                     "ms_per_step": ms / steps}
        del mb
        torch.cuda.empty_cache()
    out["fp32_over_fp64"] = out["fp32_perturbation"]["value"] / out["fp64_plain"]["value"]
    a64 = MeshBlock(opts, device="cuda")
    a64.initialize(w, r)
    a32 = MeshBlockF32(opts, device="cuda")
    a32.initialize(w, r)
    for _ in range(acc_steps):
        dt = a64.max_time_step().clone()
        a64.step(dt)
        a32.step(dt)
    torch.cuda.synchronize()
    it = (slice(None),) + opts.hydro.interior()
    acc = rel_errors(a32.state64(), a64.hydro_u, it[1:])
    acc["steps"] = acc_steps
    sacc = rel_errors(a32.scalar_s.double(), a64.scalar_s, it[1:])
    acc["scalar_rel_l1"] = sacc["rel_l1"]
    rb = a32.ref_rho.view(1, 1, -1)
    rp32 = (a32.state64()[0] - rb)[it[1:]]
    rp64 = (a64.hydro_u[0] - rb)[it[1:]]
    acc["rho_prime_rel_l1"] = float((rp32 - rp64).abs().sum() / rp64.abs().sum())
    out["accuracy_fp32_vs_fp64"] = acc
    del a64, a32
    torch.cuda.empty_cache()
    return out


def perturbation_fields(u, cfg, rb, pb):
    """rho' = rho - rho_bar, theta' = theta - theta_bar (p0 = 1e5 Pa) and the
    vertical velocity of a conserved FP64 state, interior cells"""
    it = cfg.interior()
    gm1 = cfg.gammad - 1.0
    kappa = gm1 / cfg.gammad
    rho = u[0]
    ke = 0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / rho
    p = gm1 * (u[4] - ke)
    theta = p / (rho * cfg.rgas) * (1.0e5 / p) ** kappa
    rbv, pbv = rb.view(1, 1, -1), pb.view(1, 1, -1)
    theta_bar = pbv / (rbv * cfg.rgas) * (1.0e5 / pbv) ** kappa
    return [(rho - rbv)[it], (theta - theta_bar)[it], (u[1] / rho)[it]]


def run_cpp_host_ensemble(members, tuning, args, stream, barrier, max_ms, cells_total):
    """Mcell-updates/s of the ensemble stepped by the C++ host module's
    Ensemble (eager launches on the current stream), or None if that module
    is not built."""
    import torch

    try:
        from snapy_linfel_b200 import _snapb_host
    except ImportError as e:
        return {"value": None, "unavailable": f"C++ host module not built: {e}"}
    from snapy_linfel_b200.config import config_dict

    blocks = []
    for opts, w, r in members:
        b = _snapb_host.MeshBlockF32(config_dict(opts.hydro), opts.integration.cfl, 0)
        b.initialize(torch.from_numpy(w), None if r is None else torch.from_numpy(r), "mean")
        blocks.append(b)
    keys = ("x1_columns", "march_segment", "ctas_per_sm", "vic_block", "vic_regs", "vic_kernel")
    ens = _snapb_host.Ensemble(blocks, members[0][0].integration.cfl,
                               [int(tuning.get(k, 0)) for k in keys])
    for _ in range(args.warmup):
        ens.step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ens.step()
    e1.record(stream)
    barrier()
    ms = max_ms(e0.elapsed_time(e1))
    del ens, blocks
    torch.cuda.empty_cache()
    return {"value": cells_total * 3 * args.steps / (ms / 1e3) / 1e6,
            "ms_per_step": ms / args.steps,
            "form": "C++ host module (_snapb_host.Ensemble over MeshBlockF32), eager launches"}


def run_ensemble(args):
    import torch
    import torch.distributed as dist

    from snapy_linfel_b200 import _lib, problems
    from snapy_linfel_b200.ensemble import Ensemble, StreamedEnsemble
    from snapy_linfel_b200.mesh import MeshBlock

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = f"cuda:{local}"
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_ms(ms):
        from snapy_linfel_b200.replicas import max_over_ranks

        return max_over_ranks(ms, dev)

    everyone = problems.ensemble_members(n=48, seed=2024)
    if args.workload == "c3s":  # a quarter of the ensemble, for profiling captures
        everyone = everyone[:12]
    sizes = [o.hydro.nx1 * o.hydro.nx2 * o.hydro.nx3 for o, _, _ in everyone]
    # the members are independent: on N GPUs each rank advances its share
    # (size-balanced), no data-path exchange; the step is the whole ensemble
    if world > 1:
        from snapy_linfel_b200.replicas import shard_members

        mine = shard_members(sizes, world)[rank]
    else:
        mine = list(range(len(everyone)))
    members = [everyone[k] for k in mine]
    cfg0 = members[0][0].hydro
    cells = sum(sizes[k] for k in mine)          # this rank's cells
    cells_total = sum(sizes)                     # the whole ensemble
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    # ---- batched FP32: autotune, capture, replay ----
    ens = Ensemble(members, device=dev)
    init32 = ens.save()
    if args.tuning:
        # fixed tile shapes (reproducible launch sequence, e.g. for profiling)
        fixed = {k: int(v) for k, v in (kv.split("=") for kv in args.tuning.split(","))}
        ens.set_tuning(**fixed)
        tune = {"best": ens.tuning.as_dict(), "fixed": True}
    else:
        tune = ens.tune(steps=1)
    ens.restore(init32)
    ens.capture()
    with ClockSampler(local) as clk:
        for _ in range(args.warmup):
            ens.step()
        barrier()
        clk.mark_start()
        ev0.record(stream)
        for _ in range(args.steps):
            ens.step()
        ev1.record(stream)
        barrier()
        clk.mark_end()
    ms32 = max_ms(ev0.elapsed_time(ev1))
    value32 = cells_total * 3 * args.steps / (ms32 / 1e3) / 1e6
    _lib.timing_enable(True)
    for _ in range(2):
        ens.step_eager()
    torch.cuda.synchronize()
    kern32 = _lib.timing_query()
    _lib.timing_enable(False)
    # the same ensemble stepped through the C++ host module (libtorch host
    # code over the C ABI: MeshBlockF32 members and the Ensemble plan), eager
    host_cpp = run_cpp_host_ensemble(members, tune["best"], args, stream, barrier, max_ms,
                                     cells_total)

    # end to end: every member's state from pinned host memory and back, per
    # step.  (a) StreamedEnsemble: members in groups, each on its own stream,
    # so one group's copies overlap the other groups' steps; (b) one group:
    # all copies in, the step, all copies out on one stream.
    def e2e_rate(groups):
        sens = StreamedEnsemble(members, groups=groups, device=dev, tuning=tune["best"])
        sens.capture()
        hus = sens.host_states()
        nb = sum(h.numel() * 4 for h in hus)
        for _ in range(args.warmup):
            sens.step(hus)
        sens.wait()
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            sens.step(hus)
        sens.wait()
        ev1.record(stream)
        barrier()
        rate = cells_total * 3 * args.steps / (max_ms(ev0.elapsed_time(ev1)) / 1e3) / 1e6
        del sens, hus
        torch.cuda.empty_cache()
        return rate, nb

    e2e, nbytes = e2e_rate(E2E_GROUPS)
    e2e_serial, _ = e2e_rate(1)

    # ---- plain FP64: member after member through snapb_stage, the whole
    # step (every member's CFL and three stages) replayed from one CUDA graph
    # like the batched form, and eagerly for reference ----
    blocks = []
    for opts, w, r in members:
        mb = MeshBlock(opts, device=dev)
        mb.initialize(w, r)
        blocks.append(mb)
    for _ in range(args.warmup):
        for mb in blocks:
            mb.step()
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        for mb in blocks:
            mb.step()
    ev1.record(stream)
    barrier()
    ms64_eager = max_ms(ev0.elapsed_time(ev1))
    g64 = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g64):
        for mb in blocks:
            mb.step()
    for _ in range(args.warmup):
        g64.replay()
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        g64.replay()
    ev1.record(stream)
    barrier()
    ms64 = max_ms(ev0.elapsed_time(ev1))
    del g64
    value64 = cells_total * 3 * args.steps / (ms64 / 1e3) / 1e6
    value64_eager = cells_total * 3 * args.steps / (ms64_eager / 1e3) / 1e6

    # ---- accuracy: both forms from the same state with the same dt ----
    ens.restore(init32)
    for (opts, w, r), mb in zip(members, blocks):
        mb.initialize(w, r)
    # domain-total mass per member (compensated device sums), both forms
    mass0_32 = [float(b.totals()[0]) for b in ens.blocks]
    mass0_64 = [float(b.totals()[0]) for b in blocks]
    for _ in range(args.acc_steps):
        ens.max_time_step()
        dts = ens.dts().clone()
        for m, mb in enumerate(blocks):
            mb.step(dts[m:m + 1])
        for k in range(3):
            ens.stage(k)
    torch.cuda.synchronize()
    names = ["rho", "mom1", "mom2", "mom3", "energy", "rho_prime", "theta_prime", "w_vertical"]
    num = np.zeros(len(names))
    den = np.zeros(len(names))
    emax = np.zeros(len(names))
    vmax = np.zeros(len(names))
    for b32, b64 in zip(ens.blocks, blocks):
        c = b64.cfg
        it = c.interior()
        a = b32.state64()
        b = b64.hydro_u
        fa = [a[v][it] for v in range(5)] + perturbation_fields(a, c, b32.ref_rho, b32.ref_p)
        fb = [b[v][it] for v in range(5)] + perturbation_fields(b, c, b32.ref_rho, b32.ref_p)
        for k, (x, y) in enumerate(zip(fa, fb)):
            d = (x - y).abs()
            num[k] += float(d.sum())
            den[k] += float(y.abs().sum())
            emax[k] = max(emax[k], float(d.max()))
            vmax[k] = max(vmax[k], float(y.abs().max()))
    drift32 = max(abs(float(b.totals()[0]) / m - 1.0) for b, m in zip(ens.blocks, mass0_32))
    drift64 = max(abs(float(b.totals()[0]) / m - 1.0) for b, m in zip(blocks, mass0_64))
    acc = {"steps": args.acc_steps, "fields": names,
           "rel_l1": [float(n / max(d, 1e-300)) for n, d in zip(num, den)],
           "linf": [float(e / max(v, 1e-300)) for e, v in zip(emax, vmax)],
           "mass_drift_max_member": {"fp32_form": drift32, "fp64_form": drift64}}
    del blocks
    torch.cuda.empty_cache()

    # ---- adjoint / forward time on the 2-D warm-bubble adjoint workload ----
    adj = None
    if not args.no_adjoint:
        aopts, aw, _ = problems.adjoint_bubble()
        adj = run_adjoint_timing(args, aopts, (aw, None), interior_cells(aopts.hydro), stream,
                                 barrier)
        adj["workload"] = "adjoint_bubble_2d_512x256_weno5_hllc_vic3"

    # ---- the single 384 x 384 x 192 domain: FP32 form vs FP64 form ----
    single = None
    if world == 1 and not args.no_single_domain:
        single = run_single_domain_forms(args, stream, barrier)

    # ---- roofline of the dominant batched kernel ----
    peak, peak_src = measured_peaks()
    roof = dominant_roofline(kern32, cfg0, cells, 4, peak, peak_src)
    st32 = ms32 / 1e3 / (3 * args.steps)
    bw32 = algo_bytes_per_cell_update(cfg0, 4) * cells_total / st32 / 1e9

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline_block("c3")

    if rank == 0:
        line = {
            "metric": METRIC, "value": value32, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32 / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 (perturbation over f64 reference)", "data": "synthetic",
            "config": {"workload": WORKLOAD_DESC[args.workload], "members": len(everyone),
                       "cells": cells_total, "cells_rank0": cells, "rk_stages_per_step": 3,
                       "form": "batched_fp32_perturbation (persistent work queue, CUDA graph)",
                       "tuning": tune["best"],
                       "l2_policy": "inputs larger than L2 (ensemble state > 126 MB)",
                       "parallelism": (f"members sharded over {world} ranks" if world > 1
                                       else "one GPU")},
            "forms": {
                "batched_fp32": {"value": value32, "ms_per_step": ms32 / args.steps,
                                 "kernel_ms_per_launch": {k: round(v[0] / v[1], 4)
                                                          for k, v in kern32.items()},
                                 "stage_roofline": {"achieved": bw32, "peak": peak,
                                                    "unit": "GB/s", "frac": bw32 / peak}},
                "plain_fp64_member_by_member_graph": {"value": value64,
                                                      "ms_per_step": ms64 / args.steps},
                "plain_fp64_member_by_member_eager": {"value": value64_eager,
                                                      "ms_per_step": ms64_eager / args.steps},
                "batched_fp32_cpp_host": host_cpp,
                "batched_fp32_over_plain_fp64": value32 / value64,
                "batched_fp32_over_plain_fp64_eager": value32 / value64_eager,
                "single_domain_384x384x192": single,
                "accuracy_fp32_vs_fp64": acc,
                "autotuner": tune,
            },
            "roofline": roof,
            "adjoint": adj,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                    "form": f"StreamedEnsemble, {E2E_GROUPS} groups on their own streams",
                    "one_stream_value": e2e_serial,
                    "d2h_bytes_per_step": nbytes},
            "gpu_launches": ensemble_launches_per_step(cfg0, tune["best"]) * args.steps,
            "gpu_launches_counts": "this rank's kernels in the timed region",
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_adjoint_check(args):
    """The 2-D warm-bubble adjoint workload: 512 x 256 cells, WENO5 + HLLC +
    VIC, 200 RK3 steps at CFL 0.8 with checkpoints every 20 steps,
    J = domain-integrated kinetic energy at the final time; dJ/dtheta'(x, z)
    through the hand-written adjoint (torch.autograd) against Richardson-
    extrapolated FP64 central differences along 64 seeded random directions.
    A weak seeded flow (0.3 m/s) is added to the bubble at rest: a resting,
    horizontally uniform pressure puts every x2 face exactly on the HLLC
    contact switch, where one-sided derivatives differ and a finite
    difference is not a derivative."""
    import torch

    from snapy_linfel_b200 import adjoint as A
    from snapy_linfel_b200 import problems

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    nsteps = args.adj_nsteps
    opts, w, _ = problems.adjoint_bubble()
    cfg = opts.hydro
    rng = np.random.default_rng(4)
    k3, k2, k1 = np.meshgrid(*[np.arange(n) / n for n in cfg.shape[1:]], indexing="ij")
    w[1] = 0.3 * np.sin(2 * np.pi * (k1 + 2 * k2) + rng.uniform(0, 6.28))
    w[2] = 0.3 * np.cos(2 * np.pi * (2 * k1 - k2) + rng.uniform(0, 6.28))
    base = torch.from_numpy(w).cuda()
    rd, cp = cfg.rgas, cfg.rgas * cfg.gammad / (cfg.gammad - 1.0)
    p = base[4]
    temp0 = p / (rd * base[0])
    it = cfg.interior()

    def state(dth):
        wt = torch.cat([(p / (rd * (temp0 + dth * (p / 1.0e5) ** (rd / cp))))[None], base[1:]])
        return A.initial_state(cfg, wt)

    dth0 = torch.zeros(cfg.shape[1:], dtype=torch.float64, device="cuda")
    dts = A.cfl_steps(opts, state(dth0).detach(), nsteps=nsteps)
    runner = A.StepRunner(opts, device="cuda")

    def J(dth):
        uT, _ = A.rollout(opts, state(dth), None, dts, checkpoint_every=args.adj_every,
                          runner=runner)
        return (0.5 * (uT[1] ** 2 + uT[2] ** 2 + uT[3] ** 2) / uT[0])[it].sum()

    x = dth0.clone().requires_grad_(True)
    torch.autograd.grad(J(x), x)  # warm-up
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    torch.cuda.synchronize()
    e0.record()
    j = J(x)
    e1.record()
    (grad,) = torch.autograd.grad(j, x)
    e2.record()
    torch.cuda.synchronize()
    fwd_ms, bwd_ms = e0.elapsed_time(e1), e1.elapsed_time(e2)
    mask = torch.zeros_like(dth0)
    mask[it] = 1.0
    gen = torch.Generator(device="cuda").manual_seed(2024)
    errs = []
    eps = 1e-3
    with torch.no_grad():
        for _ in range(args.adj_dirs):
            v = torch.randn(dth0.shape, generator=gen, device="cuda", dtype=torch.float64) * mask
            f = lambda t: float(J(dth0 + t * v))
            d1 = (f(eps) - f(-eps)) / (2 * eps)
            d2 = (f(eps / 2) - f(-eps / 2)) / eps
            fd = (4 * d2 - d1) / 3
            ad = float((grad * v).sum())
            errs.append(abs(fd - ad) / max(abs(fd), abs(ad), 1e-300))
    cells = interior_cells(cfg)
    # one step's reverse (from kept stage inputs) against one forward step
    stream = torch.cuda.current_stream()
    per_step = run_adjoint_timing(args, opts, (w, None), cells, stream, torch.cuda.synchronize)
    line = {
        "metric": METRIC, "value": cells * 3 * nsteps / (bwd_ms / 1e3) / 1e6, "unit": UNIT,
        "n_gpus": 1, "steps": nsteps, "warmup": 1, "ms_per_step": bwd_ms / nsteps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "adjoint_bubble_2d_512x256_weno5_hllc_vic3_200steps",
                   "checkpoint_every": args.adj_every, "objective": "kinetic energy at t_end",
                   "value_is": "reverse (checkpointed backward) cell-updates per second"},
        "adjoint": {"forward_ms": fwd_ms, "backward_ms": bwd_ms,
                    "backward_over_forward": bwd_ms / fwd_ms,
                    "step": {"forward_ms": per_step["forward_ms_per_step"],
                             "reverse_ms": per_step["reverse_ms_per_step"],
                             "reverse_over_forward": per_step["adjoint_over_forward"],
                             "reverse_kernel_ms_per_stage":
                                 per_step["reverse_kernel_ms_per_stage"]},
                    "fd_directions": len(errs), "fd_rel_err_max": max(errs),
                    "fd_rel_err_median": float(np.median(errs)),
                    "fd_within_1e-6": int(sum(e < 1e-6 for e in errs)),
                    "fd": "Richardson-extrapolated central differences, eps = 1e-3 K"},
        "gpu_launches": None,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist

    from snapy_linfel_b200 import _lib
    from snapy_linfel_b200.mesh import MeshBlock

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    opts, w, r, desc = workload(args.workload)
    _STATE_CACHE[args.workload] = (w, r)
    cfg = opts.hydro
    cells = interior_cells(cfg)  # the whole domain
    # on N GPUs the domain is split into N x2 slabs (whole vertical columns),
    # one per rank, with the ghost exchange after every stage and the MIN
    # all-reduce of dt: the total work is fixed
    decomposed = world > 1 and args.decomp == "slab"
    if decomposed:
        from snapy_linfel_b200.config import BC
        from snapy_linfel_b200.layout import SlabBlock, SlabLayout

        if cfg.nx2 < 2 or cfg.nx2 % world:
            raise SystemExit(f"{args.workload}: {cfg.nx2} x2 cells do not split into {world} slabs")
        lay = SlabLayout(world, 1, periodic_x=cfg.bc[2] == BC["periodic"])
        slab = SlabBlock(opts, lay, rank, device=f"cuda:{local}")
        slab.initialize(w, r)
        mb = slab.block
        stepper = slab.step
        args.no_fp32 = True     # the exchange moves the FP64 state
        args.no_adjoint = True
    else:
        mb = MeshBlock(opts, device=f"cuda:{local}")
        mb.initialize(w, r)
        stepper = mb.step
    mult = 1 if decomposed else world  # replicas multiply the work
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident throughput (value) ----
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        for _ in range(args.warmup):
            stepper()
        barrier()
        _lib.timing_enable(True)
        clk.mark_start()
        ev0.record(stream)
        for _ in range(args.steps):
            stepper()
        ev1.record(stream)
        barrier()
        clk.mark_end()
    ms = ev0.elapsed_time(ev1)
    kern = _lib.timing_query()
    _lib.timing_enable(False)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = t.item()
    value = mult * cells * 3 * args.steps / (ms_max / 1e3) / 1e6

    # ---- end to end through the public API with host buffers ----
    hu = torch.empty(cfg.shape, dtype=torch.float64).pin_memory()
    hu.copy_(mb.hydro_u.cpu())
    hs = None
    if cfg.nscalar:
        hs = torch.empty(cfg.scalar_shape, dtype=torch.float64).pin_memory()
        hs.copy_(mb.scalar_s.cpu())
    h2d = hu.numel() * 8 + (hs.numel() * 8 if hs is not None else 0)
    d2h = h2d
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        mb.hydro_u.copy_(hu, non_blocking=True)
        if hs is not None:
            mb.scalar_s.copy_(hs, non_blocking=True)
        stepper()
        hu.copy_(mb.hydro_u, non_blocking=True)
        if hs is not None:
            hs.copy_(mb.scalar_s, non_blocking=True)
    e1.record(stream)
    barrier()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e = mult * cells * 3 * args.steps / (t.item() / 1e3) / 1e6

    # ---- roofline of the dominant kernel (live CUDA-event durations) ----
    peak, peak_src = measured_peaks()
    local_cells = interior_cells(mb.cfg)
    roof64 = dominant_roofline(kern, cfg, local_cells, 8, peak, peak_src)
    stage_s = ms_max / 1e3 / (3 * args.steps)
    stage_bw = algo_bytes_per_cell_update(cfg) * local_cells / stage_s / 1e9
    kern_ms = {k: round(v[0] / v[1], 4) for k, v in kern.items()}
    roof = roof64

    # ---- FP32 perturbation form: throughput and accuracy against FP64 ----
    f32 = None
    if not args.no_fp32:
        f32 = run_fp32_form(args, opts, workload_state(args.workload), mb, cells, stream, barrier,
                            world)
        if world > 1:
            t = torch.tensor([f32["ms"]], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            f32["ms"] = t.item()
        f32["value"] = world * cells * 3 * args.steps / (f32["ms"] / 1e3) / 1e6

    adj = None
    if not args.no_adjoint:
        adj = run_adjoint_timing(args, opts, workload_state(args.workload), cells, stream,
                                 barrier)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline_block(args.workload)

    if rank == 0:
        forms = {"fp64_plain": {"value": value, "ms_per_step": ms_max / args.steps}}
        head_value, head_ms, head_dtype, head_form = value, ms_max / args.steps, "f64", "plain_fp64"
        if f32 is not None:
            forms["fp32_perturbation"] = {
                "value": f32["value"], "ms_per_step": f32["ms"] / args.steps,
                "kernel_ms_per_launch": f32["kern"],
                "accuracy_vs_fp64": f32["acc"]}
            forms["fp32_over_fp64_speedup"] = f32["value"] / value
            head_value, head_ms = f32["value"], f32["ms"] / args.steps
            head_dtype, head_form = "f32 (perturbation over f64 reference)", "fp32_perturbation"
            roof = dominant_roofline(f32["kern_raw"], cfg, cells, 4, peak, peak_src)
            forms["fp64_plain"]["roofline"] = roof64
            st32 = f32["ms"] / 1e3 / (3 * args.steps)
            bw32 = algo_bytes_per_cell_update(cfg, 4) * cells / st32 / 1e9
            forms["fp32_perturbation"]["stage_roofline"] = {
                "achieved": bw32, "peak": peak, "unit": "GB/s", "frac": bw32 / peak,
                "algorithmic_bytes_per_cell_update": algo_bytes_per_cell_update(cfg, 4)}
            e2e = f32["e2e"] if f32.get("e2e") else e2e
            h2d = f32.get("h2d", h2d)
            d2h = f32.get("d2h", d2h)
        line = {
            "metric": METRIC, "value": head_value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": head_ms, "higher_is_better": True,
            "scaling": "strong" if decomposed else "weak",
            "vs_baseline": None, "dtype": head_dtype, "data": "synthetic",
            "forms": forms,
            "config": {"workload": desc, "form": head_form,
                       "cells_per_gpu": cells, "rk_stages_per_step": 3,
                       "l2_policy": "inputs larger than L2 (state > 126 MB)",
                       "parallelism": (f"x2 slabs x{world} (ghost exchange per stage)"
                                       if decomposed else f"replicas x{world}")},
            "roofline": roof,
            "stage_roofline_fp64": {"achieved": stage_bw, "peak": peak, "unit": "GB/s",
                                    "frac": stage_bw / peak,
                                    "algorithmic_bytes_per_cell_update":
                                        algo_bytes_per_cell_update(cfg)},
            "kernel_ms_per_launch_fp64": kern_ms,
            "adjoint": adj,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e if not isinstance(e2e, dict) else e2e["value"], "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches_per_step(cfg) * args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3")
    ap.add_argument("--decomp", default="slab", choices=["slab", "replicas"],
                    help="single-domain workloads on N > 1 GPUs: x2 slabs with the ghost "
                         "exchange (total work fixed) or independent replicas")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--acc-steps", type=int, default=100)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-single-domain", action="store_true",
                    help="skip the 384 x 384 x 192 FP32/FP64 comparison of the ensemble line")
    ap.add_argument("--tuning", default="",
                    help="fixed ensemble tile shapes instead of the autotuner, "
                         "e.g. x1_columns=8,march_segment=16,vic_kernel=0,vic_block=32,vic_regs=0")
    ap.add_argument("--adj-steps", type=int, default=2)
    ap.add_argument("--adj-nsteps", type=int, default=200)
    ap.add_argument("--adj-every", type=int, default=20)
    ap.add_argument("--adj-dirs", type=int, default=64)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload in ("c3", "c3s"):
        return run_ensemble(args)
    if args.workload == "c4":
        return run_adjoint_check(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
