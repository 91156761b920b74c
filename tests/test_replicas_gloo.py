"""The multi-rank host logic on CPU: two gloo ranks (127.0.0.1), the
max-over-ranks timing and the member sharding the multi-GPU runs use."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from snapy_linfel_b200.replicas import max_over_ranks, rank_info, shard_members, sum_over_ranks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, w, lr = rank_info()
        mx = max_over_ranks(10.0 + r)
        total = sum_over_ranks(1.0)
        sizes = [64 * 64 * 64, 128 * 128 * 128, 96 * 96 * 64, 64 * 64 * 128, 128 * 128 * 64]
        mine = shard_members(sizes, w)[r]
        cells = sum_over_ranks(sum(sizes[m] for m in mine))
        out.put((r, w, lr, mx, total, tuple(mine), cells))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sizes = [64 * 64 * 64, 128 * 128 * 128, 96 * 96 * 64, 64 * 64 * 128, 128 * 128 * 64]
    for r, (rank, w, lr, mx, total, mine, cells) in enumerate(res):
        assert (rank, w, lr) == (r, world, r)
        assert mx == 10.0 + world - 1          # the slowest rank sets the time
        assert total == world
        assert cells == sum(sizes)              # every member on exactly one rank
    assert set(res[0][5]).isdisjoint(res[1][5])
    assert sorted(res[0][5] + res[1][5]) == list(range(len(sizes)))


def test_shard_balance():
    from snapy_linfel_b200 import problems
    from snapy_linfel_b200.replicas import shard_members

    sizes = [m["nx1"] * m["nx2"] * m["nx3"] for m in problems.ensemble(48, 2024)]
    for world in (2, 4, 8):
        parts = shard_members(sizes, world)
        loads = [sum(sizes[k] for k in p) for p in parts]
        assert sorted(sum(parts, [])) == list(range(48))
        assert max(loads) / min(loads) < 1.25
