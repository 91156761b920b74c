"""Slab decomposition host logic on CPU: the Morton rank order and neighbours
of the reference's SlabLayout, the local block configurations, and the ghost
exchange itself between gloo ranks (127.0.0.1) and between blocks held by one
process, checked against the undivided array with its periodic wraps."""
import os
import socket

import numpy as np
import pytest

from snapy_linfel_b200.config import BC, make_config
from snapy_linfel_b200.layout import SlabLayout, zorder_coords

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")


def test_zorder_order():
    # codes 0..7 decode to (x, y) = (0,0) (1,0) (0,1) (1,1) (2,0) (3,0) (2,1) (3,1)
    assert zorder_coords(2, 2) == [(0, 0), (1, 0), (0, 1), (1, 1)]
    assert zorder_coords(4, 2) == [(0, 0), (1, 0), (0, 1), (1, 1), (2, 0), (3, 0), (2, 1), (3, 1)]
    # codes outside a 3 x 2 grid are skipped
    assert zorder_coords(3, 2) == [(0, 0), (1, 0), (0, 1), (1, 1), (2, 0), (2, 1)]
    assert zorder_coords(1, 3) == [(0, 0), (0, 1), (0, 2)]


def test_neighbours():
    lay = SlabLayout(4, 2, periodic_x=True, periodic_y=False)
    r = lay.rank_at[(0, 0)]
    assert lay.neighbor_rank(r, -1, 0) == lay.rank_at[(3, 0)]  # wraps in x2
    assert lay.neighbor_rank(r, 1, 0) == lay.rank_at[(1, 0)]
    assert lay.neighbor_rank(r, 0, -1) == -1                   # x3 edge
    assert lay.neighbor_rank(r, 0, 1) == lay.rank_at[(0, 1)]
    assert lay.loc_of(8) == (-1, -1)


def test_local_config():
    cfg = make_config(nx1=8, nx2=12, nx3=8, x2=(0.0, 1200.0), x3=(0.0, 800.0),
                      bc=("reflecting", "reflecting", "reflecting", "outflow", "periodic",
                          "periodic"))
    lay = SlabLayout(3, 2, periodic_x=False, periodic_y=True)
    seen = np.zeros((cfg.nx3, cfg.nx2), dtype=int)
    for r in range(lay.world_size):
        x, y = lay.loc_of(r)
        c = lay.local_config(cfg, r)
        assert (c.nx1, c.nx2, c.nx3) == (8, 4, 4)
        assert c.x2min == pytest.approx(400.0 * x) and c.x2max == pytest.approx(400.0 * (x + 1))
        assert c.x3min == pytest.approx(400.0 * y) and c.x3max == pytest.approx(400.0 * (y + 1))
        assert c.bc[0] == BC["reflecting"] and c.bc[1] == BC["reflecting"]
        assert c.bc[2] == (BC["reflecting"] if x == 0 else BC["custom"])
        assert c.bc[3] == (BC["outflow"] if x == 2 else BC["custom"])
        assert c.bc[4] == c.bc[5] == BC["custom"]  # periodic decomposed axis
        j, k = lay.local_slices(cfg, r)
        seen[k.start - 3:k.stop - 3, j.start - 3:j.stop - 3] += 1
    assert (seen == 1).all()
    with pytest.raises(ValueError):
        SlabLayout(5, 1).local_config(cfg, 0)  # 12 cells do not split into 5


def _global_with_wraps(cfg, lay, seed):
    """a seeded global array [nv, nc3, nc2, nc1], and the same array with the
    decomposed periodic axes wrapped (x2 first, then x3)"""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((2,) + cfg.shape[1:])
    gx = g.copy()
    ng = cfg.nghost
    if lay.periodic[0] and lay.px > 1:
        n = cfg.nx2
        gx[:, :, :ng, :] = gx[:, :, n:n + ng, :]
        gx[:, :, n + ng:, :] = gx[:, :, ng:2 * ng, :]
    if lay.periodic[1] and lay.py > 1:
        n = cfg.nx3
        gx[:, :ng] = gx[:, n:n + ng]
        gx[:, n + ng:] = gx[:, ng:2 * ng]
    return g, gx


def _local(arr, cfg, lay, r):
    j, k = lay.local_slices(cfg, r)
    ng = cfg.nghost
    jj = slice(j.start - ng, j.stop + ng) if cfg.nx2 > 1 else j
    kk = slice(k.start - ng, k.stop + ng) if cfg.nx3 > 1 else k
    return np.ascontiguousarray(arr[:, kk, jj, :])


def _poison(t, cfg, lay, r):
    """NaN into the ghost cells the exchange must write"""
    c = lay.local_config(cfg, r)
    ng = cfg.nghost
    for face, dim in ((2, 2), (3, 2), (4, 1), (5, 1)):
        if c.bc[face] != BC["custom"]:
            continue
        idx = [slice(None)] * 4
        n = t.shape[dim]
        idx[dim] = slice(0, ng) if face % 2 == 0 else slice(n - ng, n)
        t[tuple(idx)] = float("nan")


CASES = [
    (dict(nx1=6, nx2=12, nx3=1), (2, 1, True, False)),
    (dict(nx1=6, nx2=12, nx3=1), (3, 1, False, False)),
    (dict(nx1=5, nx2=8, nx3=12), (2, 2, True, False)),
    (dict(nx1=5, nx2=8, nx3=12), (2, 2, False, True)),
]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, case, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        kw, (px, py, perx, pery) = CASES[case]
        cfg = make_config(**kw)
        lay = SlabLayout(px, py, perx, pery)
        g, gx = _global_with_wraps(cfg, lay, 7)
        lc = lay.local_config(cfg, rank)
        t = torch.from_numpy(_local(g, cfg, lay, rank))
        s = torch.from_numpy(_local(g, cfg, lay, rank) * 2.0)
        _poison(t, cfg, lay, rank)
        _poison(s, cfg, lay, rank)
        lay.exchange(lc, rank, [t, s])
        want = _local(gx, cfg, lay, rank)
        ok = bool(np.array_equal(t.numpy(), want)) and bool(np.array_equal(s.numpy(), 2.0 * want))
        dt = torch.tensor([1.0 + rank])
        lay.min_dt(dt)
        out.put((rank, ok, float(dt)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", range(len(CASES)))
def test_exchange_between_gloo_ranks(case):
    _, (px, py, _, _) = CASES[case]
    world = px * py
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, ok, dt in res:
        assert ok, f"rank {r}: ghost cells differ from the undivided array"
        assert dt == 1.0  # MIN over ranks


def _subgroup_worker(rank, world, port, out):
    """global ranks 1 and 2 form a subgroup holding a 2 x 1 layout; global
    rank 0 only takes part in creating the group"""
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sub = dist.new_group([1, 2])
        if rank == 0:
            out.put((rank, True, 0.0))
            return
        lrank = dist.get_group_rank(sub, rank)
        kw, (px, py, perx, pery) = CASES[0]
        cfg = make_config(**kw)
        lay = SlabLayout(px, py, perx, pery)
        g, gx = _global_with_wraps(cfg, lay, 5)
        lc = lay.local_config(cfg, lrank)
        t = torch.from_numpy(_local(g, cfg, lay, lrank))
        _poison(t, cfg, lay, lrank)
        lay.exchange(lc, lrank, [t], group=sub)
        ok = bool(np.array_equal(t.numpy(), _local(gx, cfg, lay, lrank)))
        dt = torch.tensor([3.0 + rank])
        lay.min_dt(dt, group=sub)
        out.put((rank, ok, float(dt)))
    finally:
        dist.destroy_process_group()


def test_exchange_in_a_subgroup_of_nonzero_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_subgroup_worker, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(3))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, ok, dt in res:
        assert ok, f"rank {r}: ghost cells differ from the undivided array"
        if r:
            assert dt == 4.0  # MIN over the subgroup (global ranks 1 and 2)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_exchange_in_one_process(case):
    kw, (px, py, perx, pery) = CASES[case]
    cfg = make_config(**kw)
    lay = SlabLayout(px, py, perx, pery)
    g, gx = _global_with_wraps(cfg, lay, 11)
    lc = lay.local_config(cfg, 0)
    fields = []
    for r in range(lay.world_size):
        t = torch.from_numpy(_local(g, cfg, lay, r))
        _poison(t, cfg, lay, r)
        fields.append([t])
    lay.exchange_local(lc, fields)
    for r in range(lay.world_size):
        assert np.array_equal(fields[r][0].numpy(), _local(gx, cfg, lay, r)), r


def test_yaml_distribute_section(tmp_path):
    from snapy_linfel_b200.config import MeshBlockOptions

    text = """
geometry:
  type: cartesian
  bounds: {x1min: 0., x1max: 1000., x2min: 0., x2max: 1200., x3min: 0., x3max: 800.}
  cells: {nx1: 8, nx2: 12, nx3: 8, nghost: 3}
dynamics:
  equation-of-state: {type: ideal-gas, gammad: 1.4}
  reconstruct:
    vertical: {type: weno5}
    horizontal: {type: weno5}
  riemann-solver: {type: lmars}
boundary-condition:
  external: {x1-inner: reflecting, x1-outer: reflecting, x2-inner: reflecting,
             x2-outer: reflecting, x3-inner: periodic, x3-outer: periodic}
integration: {type: rk3, cfl: 0.8}
distribute: {layout: slab, nb2: 3, nb3: 2}
"""
    p = tmp_path / "dist.yaml"
    p.write_text(text)
    o = MeshBlockOptions.from_yaml(str(p))
    lay = SlabLayout.from_options(o)
    assert (lay.px, lay.py, lay.periodic) == (3, 2, (False, True))
    c = lay.local_config(o.hydro, lay.rank_at[(2, 1)])
    assert (c.nx2, c.nx3) == (4, 4)
    assert (c.x2min, c.x2max, c.x3min, c.x3max) == (800.0, 1200.0, 400.0, 800.0)
    p.write_text(text.replace("layout: slab", "layout: cubed-sphere"))
    with pytest.raises(ValueError):
        SlabLayout.from_options(MeshBlockOptions.from_yaml(str(p)))


@pytest.mark.parametrize("split", [(2, 1, False, False), (2, 2, True, True)])
def test_oracle_blocks_reproduce_the_undivided_step(oracle, split):
    """the oracle's own stage on each block, with the exchange after every
    stage, against the oracle stepping the whole domain (CPU)"""
    from snapy_linfel_b200 import problems
    from snapy_linfel_b200.config import CONSERVED, PRIMITIVE

    px, py, perx, pery = split
    if py == 1:
        opts, w, _ = problems.straka(nx2=16, nx1=12, implicit_scheme=1)
    else:
        opts, w, _ = problems.large_3d(nx3=8, nx2=8, nx1=12, nscalar=0)
    c = opts.hydro
    lay = SlabLayout(px, py, perx, pery)

    def conserved(cfg, wp):
        wp = np.ascontiguousarray(wp)
        oracle.bc_apply(cfg, wp, PRIMITIVE)
        u = oracle.prim2cons(cfg, wp)
        oracle.bc_apply(cfg, u, CONSERVED)
        return u

    u = conserved(c, w.copy())
    parts = []
    for r in range(lay.world_size):
        lc = lay.local_config(c, r)
        parts.append((lc, conserved(lc, _local(w, c, lay, r))))
    lay.exchange_local(parts[0][0], [[torch.from_numpy(p[1])] for p in parts])
    whole = oracle.block(c)
    blocks = [oracle.block(lc) for lc, _ in parts]
    u0 = np.empty_like(u)
    u0s = [np.empty_like(p[1]) for p in parts]
    ww = np.empty_like(u)
    wws = [np.empty_like(p[1]) for p in parts]
    for _ in range(2):
        for st in range(3):
            whole.stage(st, 0.4, u, u0, ww)
            for (lc, up), b, u0p, wp in zip(parts, blocks, u0s, wws):
                b.stage(st, 0.4, up, u0p, wp)
            lay.exchange_local(parts[0][0], [[torch.from_numpy(p[1])] for p in parts])
    for r, (lc, up) in enumerate(parts):
        j, k = lay.local_slices(c, r)
        ng = c.nghost
        lj = slice(ng, ng + j.stop - j.start) if c.nx2 > 1 else j
        lk = slice(ng, ng + k.stop - k.start) if c.nx3 > 1 else k
        a = up[:, lk, lj, ng:ng + c.nx1]
        b = u[:, k, j, ng:ng + c.nx1]
        for v in range(5):
            assert np.abs(a[v] - b[v]).max() <= 1e-12 * np.abs(b[v]).max() + 1e-300, (r, v)
