"""Slab domain decomposition of one mesh block over several GPUs: the x2 axis
split into px blocks and the x3 axis into py blocks, whole vertical (x1)
columns on every rank, one ghost-zone exchange per RK stage and a MIN
all-reduce of dt per step.

Reference: SlabLayoutImpl (src/layout/slab_layout.cpp:10-72), the exchange of
LayoutImpl (src/layout/layout.cpp:361-634) and the internal-boundary set-up of
MeshBlockImpl (src/mesh/meshblock.cpp:69-118).  As there:

* rank r sits at (x, y) = the r-th coordinate of the px x py grid in Morton
  (Z) order: codes 0, 1, 2, ... are decoded with x from the even bits and y
  from the odd bits, and the codes that fall inside the grid are handed out
  in order (build_zorder_coords2, src/layout/connectivity.cpp:28-43);
* x runs along x2 and y along x3 (loc_of -> (lx2, lx3, lx1));
* internal faces, and both faces of a periodic decomposed axis, take no
  boundary function: here the 'custom' boundary type, which the local fill
  leaves untouched, so the exchange alone writes those ghost cells.

The exchange runs over torch.distributed point-to-point messages (NCCL between
GPUs; gloo in the CPU tests), x2 faces first and then x3 faces, each message
the ng interior layers next to a face with the full extent of the other axes
(ghosts included): the x3 messages therefore carry the x2 ghost cells just
received, which fills the corners the way the global block's fill order (x1,
x2, x3) does.  With two blocks on a periodic axis both neighbours are the same
rank; every rank posts, per axis, send-up, send-down, receive-from-below,
receive-from-above, so messages between a pair of ranks match in order.
"""
from __future__ import annotations

import copy

from .config import BC, HydroConfig

CUSTOM = BC["custom"]
PERIODIC = BC["periodic"]


def _compact1by1(v: int) -> int:
    """keep the bits of v at even positions, packed"""
    v &= 0x55555555
    v = (v ^ (v >> 1)) & 0x33333333
    v = (v ^ (v >> 2)) & 0x0F0F0F0F
    v = (v ^ (v >> 4)) & 0x00FF00FF
    v = (v ^ (v >> 8)) & 0x0000FFFF
    return v


def zorder_coords(px: int, py: int):
    """[(x, y)] of ranks 0 .. px*py-1 in Morton order"""
    out, code = [], 0
    while len(out) < px * py:
        x, y = _compact1by1(code), _compact1by1(code >> 1)
        if x < px and y < py:
            out.append((x, y))
        code += 1
    return out


class SlabLayout:
    """px x py blocks over (x2, x3); periodic flags per decomposed axis."""

    def __init__(self, px: int = 1, py: int = 1, periodic_x: bool = False,
                 periodic_y: bool = False):
        if px < 1 or py < 1:
            raise ValueError("px and py must be >= 1")
        self.px, self.py = px, py
        self.periodic = (bool(periodic_x), bool(periodic_y))
        self.coords = zorder_coords(px, py)
        self.rank_at = {xy: r for r, xy in enumerate(self.coords)}

    @staticmethod
    def from_options(options) -> "SlabLayout":
        """from MeshBlockOptions.layout (the YAML 'distribute' section)"""
        lo = options.layout
        if lo.type != "slab":
            raise ValueError(f"layout {lo.type!r} is not on this path (slab only)")
        if lo.pz != 1:
            raise ValueError("a slab layout keeps whole x1 columns: nb1 must be 1")
        return SlabLayout(lo.px, lo.py, lo.periodic_x, lo.periodic_y)

    @property
    def world_size(self) -> int:
        return self.px * self.py

    def loc_of(self, rank: int):
        """(lx2, lx3) of a rank, (-1, -1) outside the layout"""
        if rank < 0 or rank >= self.world_size:
            return (-1, -1)
        return self.coords[rank]

    def neighbor_rank(self, rank: int, dx: int, dy: int) -> int:
        """rank of the block at offset (dx, dy) in (x2, x3); -1 off a
        non-periodic edge"""
        x, y = self.loc_of(rank)
        n = [x + dx, y + dy]
        for a, (size, per) in enumerate(zip((self.px, self.py), self.periodic)):
            if per:
                n[a] %= size
            elif n[a] < 0 or n[a] >= size:
                return -1
        return self.rank_at[(n[0], n[1])]

    # ---- the local block ----
    def local_config(self, cfg: HydroConfig, rank: int) -> HydroConfig:
        """This rank's block of the global configuration: nx2 / px x nx3 / py
        interior cells, its coordinate range, and 'custom' boundaries on the
        faces the exchange fills."""
        x, y = self.loc_of(rank)
        if x < 0:
            raise ValueError(f"rank {rank} outside a {self.px} x {self.py} layout")
        c = copy.deepcopy(cfg)
        for a, (p, l, nx, lo, hi, face) in enumerate(
                ((self.px, x, cfg.nx2, cfg.x2min, cfg.x2max, 2),
                 (self.py, y, cfg.nx3, cfg.x3min, cfg.x3max, 4))):
            if p == 1:
                continue
            if nx % p:
                raise ValueError(f"x{a + 2}: {nx} cells do not split into {p} blocks")
            n = nx // p
            if n < cfg.nghost:
                raise ValueError(f"x{a + 2}: blocks of {n} cells are thinner than the ghost zone")
            # CoordinateOptionsImpl::repartition (src/coord/coordinate.cpp:167-191)
            bmin = lo + l * (hi - lo) / p
            setattr(c, f"nx{a + 2}", n)
            setattr(c, f"x{a + 2}min", bmin)
            setattr(c, f"x{a + 2}max", bmin + (hi - lo) / p)
            if self.periodic[a] or l > 0:
                c.bc[face] = CUSTOM
            if self.periodic[a] or l < p - 1:
                c.bc[face + 1] = CUSTOM
        return c

    def local_slices(self, cfg: HydroConfig, rank: int):
        """(j slice, k slice) of this rank's interior in the global block's
        arrays (ghosts of the global block excluded)"""
        x, y = self.loc_of(rank)
        ng = cfg.nghost
        out = []
        for p, l, nx in ((self.px, x, cfg.nx2), (self.py, y, cfg.nx3)):
            if nx == 1:
                out.append(slice(0, 1))
                continue
            n = nx // p
            out.append(slice(ng + l * n, ng + (l + 1) * n))
        return tuple(out)

    # ---- exchange ----
    def _face_plan(self, cfg: HydroConfig, rank: int):
        """per decomposed axis (tensor dim, [(peer, send slice, recv slice,
        tag)]) in the posting order described in the module docstring"""
        ng = cfg.nghost
        plans = []
        for a, (p, n_loc) in enumerate(((self.px, cfg.nx2), (self.py, cfg.nx3))):
            if p == 1:
                continue
            dim = 2 if a == 0 else 1  # [nv, nc3, nc2, nc1]
            lo, hi = ng, ng + n_loc  # interior [lo, hi)
            up = self.neighbor_rank(rank, 1, 0) if a == 0 else self.neighbor_rank(rank, 0, 1)
            dn = self.neighbor_rank(rank, -1, 0) if a == 0 else self.neighbor_rank(rank, 0, -1)
            sends = [(up, slice(hi - ng, hi), 2 * a), (dn, slice(lo, lo + ng), 2 * a + 1)]
            # what I receive from below is what it sent up (tag 2a) into my low ghosts
            recvs = [(dn, slice(0, ng), 2 * a), (up, slice(hi, hi + ng), 2 * a + 1)]
            plans.append((dim, sends, recvs))
        return plans

    # ---- slab buffers: the message format of the exchange ----
    @staticmethod
    def pack(cfg: HydroConfig, t, dim: int, sl: slice):
        """the slab t[:, .., sl, ..] along tensor dim (2: x2, 1: x3) as a
        contiguous buffer in row-major order; device tensors are packed by the
        snapb_pack_slab kernel, host tensors (CPU ranks) by a tensor copy of
        the same layout"""
        import torch

        shape = list(t.shape)
        shape[dim] = sl.stop - sl.start
        if not t.is_cuda:
            idx = [slice(None)] * 4
            idx[dim] = sl
            return t[tuple(idx)].contiguous()
        if t.dtype != torch.float64 or not t.is_contiguous():
            raise ValueError("device slabs are packed from contiguous float64 arrays")
        import ctypes

        from . import _lib

        buf = torch.empty(shape, dtype=t.dtype, device=t.device)
        _lib.check(_lib.lib().snapb_pack_slab(ctypes.byref(cfg), 2 if dim == 2 else 3, sl.start,
                                              sl.stop - sl.start, _lib.ptr(t), int(t.shape[0]),
                                              _lib.ptr(buf), _lib.stream_ptr()),
                   "snapb_pack_slab")
        return buf

    @staticmethod
    def unpack(cfg: HydroConfig, t, dim: int, sl: slice, buf):
        """write a buffer made by pack() into the slab t[:, .., sl, ..]"""
        if not t.is_cuda:
            idx = [slice(None)] * 4
            idx[dim] = sl
            t[tuple(idx)].copy_(buf)
            return
        import ctypes

        from . import _lib

        _lib.check(_lib.lib().snapb_unpack_slab(ctypes.byref(cfg), 2 if dim == 2 else 3,
                                                sl.start, sl.stop - sl.start, _lib.ptr(t),
                                                int(t.shape[0]), _lib.ptr(buf),
                                                _lib.stream_ptr()),
                   "snapb_unpack_slab")

    def exchange(self, cfg: HydroConfig, rank: int, tensors, group=None):
        """Fill the exchange faces' ghost cells of each [nv, nc3, nc2, nc1]
        tensor (local block, after its local boundary fill) from the
        neighbours' interiors.  `rank` and the layout's ranks are ranks of
        `group` (the default group when None); a subgroup may hold any set of
        global ranks."""
        import torch
        import torch.distributed as dist

        def peer_of(r):
            # layout ranks are ranks of `group`; P2POp names global ranks
            return r if group is None else dist.get_global_rank(group, r)

        for dim, sends, recvs in self._face_plan(cfg, rank):
            ops, keep, unpacks = [], [], []
            for ti, t in enumerate(tensors):
                for peer, sl, tag in sends:
                    if peer < 0:
                        continue
                    buf = self.pack(cfg, t, dim, sl)
                    keep.append(buf)
                    ops.append(dist.P2POp(dist.isend, buf, peer_of(peer), group, 4 * ti + tag))
                for peer, sl, tag in recvs:
                    if peer < 0:
                        continue
                    shape = list(t.shape)
                    shape[dim] = sl.stop - sl.start
                    buf = torch.empty(shape, dtype=t.dtype, device=t.device)
                    ops.append(dist.P2POp(dist.irecv, buf, peer_of(peer), group, 4 * ti + tag))
                    unpacks.append((t, sl, buf))
            if not ops:
                continue
            for req in dist.batch_isend_irecv(ops):
                req.wait()
            for t, sl, buf in unpacks:
                self.unpack(cfg, t, dim, sl, buf)
            del keep

    def exchange_local(self, cfg: HydroConfig, fields_by_rank):
        """The same exchange between blocks held by one process (a list, per
        rank, of that rank's tensors): the copies the messages would make,
        axis by axis in the same order.  Used to check the decomposition on
        one device."""
        plans = [self._face_plan(cfg, r) for r in range(self.world_size)]
        for a in range(len(plans[0])):
            moves = []
            for r in range(self.world_size):
                dim, _, recvs = plans[r][a]
                for peer, rsl, tag in recvs:
                    if peer < 0:
                        continue
                    _, psends, _ = plans[peer][a]
                    ssl = next(sl for q, sl, tg in psends if q == r and tg == tag)
                    for t_dst, t_src in zip(fields_by_rank[r], fields_by_rank[peer]):
                        # the message the sender would post, unpacked by the receiver
                        moves.append((t_dst, dim, rsl, self.pack(cfg, t_src, dim, ssl)))
            for t, dim, sl, buf in moves:
                self.unpack(cfg, t, dim, sl, buf)

    @staticmethod
    def min_dt(dt, group=None):
        """MIN all-reduce of a device dt tensor (in place) across the ranks"""
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
            dist.all_reduce(dt, op=dist.ReduceOp.MIN, group=group)
        return dt


class SlabBlock:
    """One rank's block of a decomposed domain, advanced with the same C ABI
    as MeshBlock: local CFL -> MIN all-reduce -> three stages, each followed
    by the ghost exchange (MeshBlockImpl::forward with a layout,
    src/mesh/meshblock.cpp:577-786)."""

    def __init__(self, options, layout: SlabLayout, rank: int, device=None, group=None):
        from .config import MeshBlockOptions
        from .mesh import MeshBlock

        if isinstance(options, HydroConfig):
            options = MeshBlockOptions(options)
        self.global_cfg = options.hydro
        self.layout, self.rank, self.group = layout, rank, group
        local = copy.deepcopy(options)
        local.hydro = layout.local_config(options.hydro, rank)
        self.block = MeshBlock(local, device=device)
        self.cfg = local.hydro

    def _fields(self):
        b = self.block
        return [b.hydro_u] + ([b.scalar_s] if b.scalar_s is not None else [])

    def initialize(self, w_global, r_global=None):
        """primitive state of the whole domain (global arrays, ghosts
        included); this rank takes its part and exchanges the halos"""
        j, k = self.layout.local_slices(self.global_cfg, self.rank)
        ng = self.global_cfg.nghost
        jj = slice(j.start - ng, j.stop + ng) if self.global_cfg.nx2 > 1 else j
        kk = slice(k.start - ng, k.stop + ng) if self.global_cfg.nx3 > 1 else k
        import numpy as np

        w = np.ascontiguousarray(w_global[:, kk, jj, :])
        r = np.ascontiguousarray(r_global[:, kk, jj, :]) if r_global is not None else None
        self.block.initialize(w, r)
        self.exchange()
        if self.block.scalar_r is not None:
            self.block.scalar_r.copy_(self.block.scalar_s / self.block.hydro_u[0:1])

    def exchange(self):
        self.layout.exchange(self.cfg, self.rank, self._fields(), self.group)

    def max_time_step(self):
        b = self.block
        import ctypes

        from . import _lib

        ws, nb = b._ws()
        b._call("snapb_max_time_step", ctypes.byref(b.cfg), _lib.ptr(b.hydro_w),
                _lib.ptr(b.dt_raw), ws, nb, b._stream())
        self.layout.min_dt(b.dt_raw, self.group)
        b._call("snapb_scale_dt", _lib.ptr(b.dt_raw), ctypes.c_double(
            b.options.integration.cfl), b.current_redo, _lib.ptr(b.dt), b._stream())
        return b.dt

    def step(self, dt=None):
        if dt is None:
            self.max_time_step()
        else:
            self.block.set_dt(dt)
        for s in range(3):
            self.block.forward(s)
            self.exchange()
        self.block.cycle += 1


class LocalSlabBlocks:
    """Every block of a layout held by one process on one device (the
    reference's blocks-per-process > 1): the same local blocks, CFL minimum
    and ghost exchange as SlabBlock, with the exchange done by copies."""

    def __init__(self, options, layout: SlabLayout, device=None):
        from .config import MeshBlockOptions
        from .mesh import MeshBlock

        if isinstance(options, HydroConfig):
            options = MeshBlockOptions(options)
        self.global_cfg = options.hydro
        self.layout = layout
        self.blocks = []
        for r in range(layout.world_size):
            local = copy.deepcopy(options)
            local.hydro = layout.local_config(options.hydro, r)
            self.blocks.append(MeshBlock(local, device=device))
        self.cfg = self.blocks[0].cfg

    def _fields(self):
        return [[b.hydro_u] + ([b.scalar_s] if b.scalar_s is not None else [])
                for b in self.blocks]

    def initialize(self, w_global, r_global=None):
        import numpy as np

        ng = self.global_cfg.nghost
        for r, b in enumerate(self.blocks):
            j, k = self.layout.local_slices(self.global_cfg, r)
            jj = slice(j.start - ng, j.stop + ng) if self.global_cfg.nx2 > 1 else j
            kk = slice(k.start - ng, k.stop + ng) if self.global_cfg.nx3 > 1 else k
            b.initialize(np.ascontiguousarray(w_global[:, kk, jj, :]),
                         None if r_global is None
                         else np.ascontiguousarray(r_global[:, kk, jj, :]))
        self.layout.exchange_local(self.cfg, self._fields())

    def max_time_step(self):
        import ctypes

        import torch

        from . import _lib

        raws = []
        for b in self.blocks:
            ws, nb = b._ws()
            b._call("snapb_max_time_step", ctypes.byref(b.cfg), _lib.ptr(b.hydro_w),
                    _lib.ptr(b.dt_raw), ws, nb, b._stream())
            raws.append(b.dt_raw)
        low = torch.min(torch.cat(raws))
        for b in self.blocks:
            b.dt_raw.fill_(low)
            b._call("snapb_scale_dt", _lib.ptr(b.dt_raw), ctypes.c_double(
                b.options.integration.cfl), b.current_redo, _lib.ptr(b.dt), b._stream())
        return self.blocks[0].dt

    def step(self, dt=None):
        if dt is None:
            self.max_time_step()
        else:
            for b in self.blocks:
                b.set_dt(dt)
        for s in range(3):
            for b in self.blocks:
                b.forward(s)
            self.layout.exchange_local(self.cfg, self._fields())
        for b in self.blocks:
            b.cycle += 1

    def gather(self, which="hydro_u"):
        """the blocks' interiors assembled into a global-shaped array (ghosts of
        the global block left zero)"""
        import torch

        ng = self.global_cfg.nghost
        first = getattr(self.blocks[0], which)
        out = torch.zeros((first.shape[0],) + tuple(self.global_cfg.shape[1:]),
                          dtype=first.dtype, device=first.device)
        for r, b in enumerate(self.blocks):
            j, k = self.layout.local_slices(self.global_cfg, r)
            lj = slice(ng, ng + (j.stop - j.start)) if self.global_cfg.nx2 > 1 else j
            lk = slice(ng, ng + (k.stop - k.start)) if self.global_cfg.nx3 > 1 else k
            out[:, k, j, :] = getattr(b, which)[:, lk, lj, :]
        return out
