"""Batched ensembles of uneven mesh blocks (FP32 perturbation form).

``Ensemble`` advances many independent members (snapy MeshBlocks of
different sizes with the same physics) together through the
``snapb_ensemble_*`` entry points of include/snapb.h: every sweep of a stage
is one persistent launch over all members whose CTAs pull (member, tile)
work items from a device counter.  A step (per-member CFL + three stages) can
be captured once in a CUDA graph and replayed; ``tune()`` is the autotuner:
it times candidate tile shapes on the live ensemble (state saved and
restored around each trial) and keeps the fastest.

The reference advances one MeshBlock per call (MeshBlockImpl::forward,
src/mesh/meshblock.cpp:577-786) and has no batched form.
"""
from __future__ import annotations

import ctypes
import itertools
import time

from . import _lib
from .config import HydroConfig, MeshBlockOptions
from .mesh import MeshBlockF32


class MemberF32(ctypes.Structure):
    _fields_ = [("cfg", HydroConfig),
                ("u", ctypes.c_void_p), ("u0", ctypes.c_void_p), ("w", ctypes.c_void_p),
                ("s", ctypes.c_void_p), ("s0", ctypes.c_void_p), ("r", ctypes.c_void_p),
                ("workspace", ctypes.c_void_p), ("workspace_bytes", ctypes.c_size_t)]


class Tuning(ctypes.Structure):
    _fields_ = [("x1_columns", ctypes.c_int32), ("march_segment", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("vic_block", ctypes.c_int32),
                ("vic_regs", ctypes.c_int32), ("vic_kernel", ctypes.c_int32)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


def _vp(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class Ensemble:
    """members: list of (MeshBlockOptions, hydro_w, scalar_r) with the same physics."""

    def __init__(self, members, device=None, tuning: dict | None = None):
        import torch

        self.device = torch.device(device if device is not None else "cuda")
        self.lib = _lib.lib()
        self.blocks = []
        for opts, w, r in members:
            mb = MeshBlockF32(opts, device=self.device)
            mb.initialize(w, r)
            self.blocks.append(mb)
        self.options = self.blocks[0].options
        self.cfl = self.options.integration.cfl
        arr = (MemberF32 * len(self.blocks))()
        for k, mb in enumerate(self.blocks):
            m = arr[k]
            m.cfg = mb.cfg.copy() if hasattr(mb.cfg, "copy") else mb.cfg
            m.u, m.u0, m.w = _vp(mb.hydro_u), _vp(mb.hydro_u0), _vp(mb.hydro_w)
            m.s, m.s0, m.r = _vp(mb.scalar_s), _vp(mb.scalar_s0), _vp(mb.scalar_r)
            m.workspace = _vp(mb.workspace)
            m.workspace_bytes = mb.workspace.numel()
        self._members = arr
        self.tuning = Tuning()
        for k, v in (tuning or {}).items():
            setattr(self.tuning, k, int(v))
        h = ctypes.c_void_p()
        _lib.check(self.lib.snapb_ensemble_create(ctypes.cast(arr, ctypes.c_void_p), len(arr),
                                                  ctypes.byref(self.tuning), ctypes.byref(h)),
                   "snapb_ensemble_create")
        self.handle = h
        nbytes = self.lib.snapb_ensemble_workspace_size(h)
        # room for re-plans with other tile shapes
        self.workspace = torch.zeros(2 * nbytes + (1 << 20), dtype=torch.uint8,
                                     device=self.device)
        _lib.check(self.lib.snapb_ensemble_bind(h, _vp(self.workspace), self.workspace.numel(),
                                                _lib.stream_ptr()), "snapb_ensemble_bind")
        self.graph = None
        self.cycle = 0

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and getattr(self, "lib", None) is not None:
            self.lib.snapb_ensemble_destroy(h)
            self.handle = None

    # ---- stepping ----
    @property
    def cells(self):
        return sum(b.cfg.nx1 * b.cfg.nx2 * b.cfg.nx3 for b in self.blocks)

    def dts(self):
        """the members' dt (device tensor view, [n])"""
        import torch

        ptr = self.lib.snapb_ensemble_dt(self.handle)
        n = len(self.blocks)
        store = torch.empty(0, dtype=torch.float64, device=self.device)
        off = ptr - self.workspace.data_ptr()
        return self.workspace[off:off + 8 * n].view(torch.float64)[:n] if off >= 0 else store

    def max_time_step(self):
        _lib.check(self.lib.snapb_ensemble_max_time_step_f32(self.handle,
                                                             ctypes.c_double(self.cfl),
                                                             _lib.stream_ptr()),
                   "snapb_ensemble_max_time_step_f32")

    def stage(self, k: int):
        _lib.check(self.lib.snapb_ensemble_stage_f32(self.handle, int(k), _lib.stream_ptr()),
                   "snapb_ensemble_stage_f32")

    def step_eager(self):
        self.max_time_step()
        for k in range(3):
            self.stage(k)

    def capture(self):
        """Capture one step (CFL + three stages) in a CUDA graph."""
        import torch

        snap = self.save()
        self.step_eager()  # warm: function attributes and lazy loading happen outside
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.step_eager()
        self.restore(snap)
        self.graph = g
        return g

    def step(self):
        if self.graph is not None:
            self.graph.replay()
        else:
            self.step_eager()
        self.cycle += 1

    # ---- state ----
    def save(self):
        out = []
        for b in self.blocks:
            out.append([t.clone() if t is not None else None
                        for t in (b.hydro_u, b.hydro_u0, b.hydro_w, b.scalar_s, b.scalar_s0,
                                  b.scalar_r)])
        return out

    def restore(self, snap):
        for b, ts in zip(self.blocks, snap):
            for dst, src in zip((b.hydro_u, b.hydro_u0, b.hydro_w, b.scalar_s, b.scalar_s0,
                                 b.scalar_r), ts):
                if dst is not None:
                    dst.copy_(src)

    # ---- autotuner ----
    def set_tuning(self, **kw):
        t = Tuning()
        for k, v in self.tuning.as_dict().items():
            setattr(t, k, int(kw.get(k, v)))
        _lib.check(self.lib.snapb_ensemble_set_tuning(self.handle, ctypes.byref(t),
                                                      _lib.stream_ptr()),
                   "snapb_ensemble_set_tuning")
        self.tuning = t
        self.graph = None

    def tune(self, steps: int = 2, candidates: dict | None = None, log=None):
        """Time each candidate tile shape over `steps` eager steps on the live
        state (saved and restored), keep the fastest; returns the table."""
        import torch

        cand = candidates or {"x1_columns": [0, 4, 8], "march_segment": [16, 32, 64],
                              "ctas_per_sm": [0, 4, 8], "vic_kernel": [0, 1, 2],
                              "vic_block": [32, 64, 128], "vic_regs": [0, 1, 2]}
        snap = self.save()
        results = []
        best = None
        # coordinate descent: one parameter at a time, starting from the defaults
        current = self.tuning.as_dict()
        for key, values in cand.items():
            if key in ("vic_block", "vic_regs") and current.get("vic_kernel", 0) != 0:
                continue  # shapes of the column kernel, not in use
            for v in values:
                trial = dict(current)
                trial[key] = v
                try:
                    self.set_tuning(**trial)
                except _lib.SnapbError:
                    continue
                self.restore(snap)
                self.step_eager()  # warm
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(steps):
                    self.step_eager()
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / steps
                results.append((dict(trial), ms))
                if log:
                    log(f"tune {trial} -> {ms:.3f} ms/step")
                if best is None or ms < best[1]:
                    best = (dict(trial), ms)
            current = dict(best[0])
        self.set_tuning(**best[0])
        self.restore(snap)
        return {"best": best[0], "best_ms_per_step": best[1],
                "trials": [{"tuning": t, "ms_per_step": m} for t, m in results]}


class StreamedEnsemble:
    """An ensemble whose states live in pinned host memory: every step copies
    each member's FP32 state (``hydro_u``, ghosts included) in and its result
    back out.  The members are split into ``groups`` sub-ensembles balanced by
    cells, each an ``Ensemble`` with its own CUDA stream and step graph, so
    the host-to-device copies of one group, the device-to-host copies of
    another (the two copy directions run on separate engines) and the steps
    of a third overlap.  A group's copies and steps are ordered on its own
    stream; groups never wait for each other, so ``step()`` returns after
    queueing and ``wait()`` joins every group into the current stream.

    members: as ``Ensemble``; host: one pinned FP32 tensor per member, in
    member order, shaped like its ``hydro_u`` (``host_states()`` makes them
    from the current states)."""

    def __init__(self, members, groups: int = 4, device=None, tuning: dict | None = None):
        import torch

        self.device = torch.device(device if device is not None else "cuda")
        cells = [o.hydro.nx1 * o.hydro.nx2 * o.hydro.nx3 for o, _, _ in members]
        groups = max(1, min(groups, len(members)))
        load = [0] * groups
        self.slots = [[] for _ in range(groups)]  # member indices of each group
        for m in sorted(range(len(members)), key=lambda k: -cells[k]):
            g = min(range(groups), key=lambda k: load[k])
            self.slots[g].append(m)
            load[g] += cells[m]
        self.parts = [Ensemble([members[m] for m in idx], device=self.device, tuning=tuning)
                      for idx in self.slots]
        self.where = {}  # member -> (group, position)
        for g, idx in enumerate(self.slots):
            for k, m in enumerate(idx):
                self.where[m] = (g, k)
        self.streams = [torch.cuda.Stream(device=self.device) for _ in self.parts]
        cur = torch.cuda.current_stream(self.device)
        for s in self.streams:
            s.wait_stream(cur)

    @property
    def blocks(self):
        """the member blocks in member order"""
        return [self.parts[g].blocks[k] for g, k in (self.where[m] for m in range(len(self.where)))]

    @property
    def cells(self):
        return sum(p.cells for p in self.parts)

    def host_states(self):
        """pinned host copies of the members' current states, in member order"""
        import torch

        out = []
        for b in self.blocks:
            h = torch.empty(b.hydro_u.shape, dtype=torch.float32).pin_memory()
            h.copy_(b.hydro_u.cpu())
            out.append(h)
        return out

    def capture(self):
        """capture each group's step in its own CUDA graph"""
        import torch

        self.wait()
        for p in self.parts:
            p.capture()
        torch.cuda.synchronize(self.device)

    def step(self, host):
        """one step of every member from and back to its host state (queued
        on the groups' streams)"""
        import torch

        for g, (p, s) in enumerate(zip(self.parts, self.streams)):
            with torch.cuda.stream(s):
                for k, m in enumerate(self.slots[g]):
                    p.blocks[k].hydro_u.copy_(host[m], non_blocking=True)
                p.step()
                for k, m in enumerate(self.slots[g]):
                    host[m].copy_(p.blocks[k].hydro_u, non_blocking=True)

    def wait(self):
        """join every group's queued work into the current stream"""
        import torch

        cur = torch.cuda.current_stream(self.device)
        for s in self.streams:
            cur.wait_stream(s)
