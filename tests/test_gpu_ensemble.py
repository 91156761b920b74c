"""Batched ensemble (persistent work-queue launches) against the one-block
FP32 path on the same members: the batched sweeps run the same tile code, so
every member's state must agree bit for bit with snapb_stage_f32 run on that
member alone, for every tile shape the autotuner may pick, eager or replayed
from a CUDA graph."""
import numpy as np
import pytest

from snapy_linfel_b200 import problems

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return "cuda"


def small_members(n=5, seed=9, implicit_scheme=1, riemann="lmars"):
    return problems.ensemble_members(n=n, seed=seed, horiz=(8, 12, 16), vert=(8, 16),
                                     riemann=riemann, implicit_scheme=implicit_scheme)


def singles(members, steps, dev):
    from snapy_linfel_b200.mesh import MeshBlockF32

    out = []
    for opts, w, r in members:
        mb = MeshBlockF32(opts, device=dev)
        mb.initialize(w, r)
        for _ in range(steps):
            mb.step()
        out.append(mb.hydro_u.clone())
    return out


def batched(members, steps, dev, tuning=None, graph=False):
    from snapy_linfel_b200.ensemble import Ensemble

    ens = Ensemble(members, device=dev, tuning=tuning)
    if graph:
        ens.capture()
    for _ in range(steps):
        ens.step()
    return ens, [b.hydro_u.clone() for b in ens.blocks]


@pytest.mark.parametrize("scheme,riemann", [(1, "lmars"), (9, "roe"), (0, "hllc")])
def test_batched_matches_single_blocks(dev, scheme, riemann):
    from snapy_linfel_b200 import _lib

    members = small_members(implicit_scheme=scheme, riemann=riemann)
    ref = singles(members, 3, dev)
    _, got = batched(members, 3, dev)
    for k, (a, b) in enumerate(zip(got, ref)):
        assert torch.equal(a, b), f"member {k}: max diff {float((a - b).abs().max())}"
    # the x1 sweeps' bulk copies all completed
    assert _lib.lib().snapb_bulk_copy_timeouts() == 0


def test_tile_shapes_and_graph_replay_are_exact(dev):
    members = small_members(n=4, seed=3)
    ref = singles(members, 2, dev)
    for tuning in ({"x1_columns": 1, "march_segment": 8, "ctas_per_sm": 1, "vic_block": 32},
                   {"x1_columns": 8, "march_segment": 64, "ctas_per_sm": 4, "vic_block": 128}):
        _, got = batched(members, 2, dev, tuning=tuning)
        for a, b in zip(got, ref):
            assert torch.equal(a, b)
    _, got = batched(members, 2, dev, graph=True)
    for a, b in zip(got, ref):
        assert torch.equal(a, b)


def test_x1_prefetch_across_members_of_different_heights(dev):
    """the batched x1 sweep stages the next tile (of any member) while the
    current one's faces run: with one CTA per SM every CTA takes many tiles,
    and members of 8 and 40 layers alternate, so a tile's staging follows
    rows of a longer or shorter column; every member matches its one-block
    run exactly"""
    from snapy_linfel_b200 import _lib

    members = problems.ensemble_members(n=6, seed=21, horiz=(12, 20), vert=(8, 40),
                                        riemann="lmars", implicit_scheme=1)
    ref = singles(members, 2, dev)
    for tuning in ({"x1_columns": 8, "ctas_per_sm": 1}, {"x1_columns": 2, "ctas_per_sm": 1}):
        _, got = batched(members, 2, dev, tuning=tuning)
        for k, (a, b) in enumerate(zip(got, ref)):
            assert torch.equal(a, b), f"{tuning} member {k}: {float((a - b).abs().max())}"
    assert _lib.lib().snapb_bulk_copy_timeouts() == 0


def test_streamed_ensemble_from_host_states(dev):
    """members stepped from pinned host states in groups on their own streams
    (copies of one group overlapping the steps of the others) end exactly
    where their one-block runs end"""
    from snapy_linfel_b200.ensemble import StreamedEnsemble

    members = small_members(n=5, seed=17)
    ref = singles(members, 3, dev)
    sens = StreamedEnsemble(members, groups=3, device=dev)
    sens.capture()
    host = sens.host_states()
    for _ in range(3):
        sens.step(host)
    sens.wait()
    torch.cuda.synchronize()
    for k, (h, b) in enumerate(zip(host, ref)):
        assert torch.equal(h.to(dev), b), f"member {k}: {float((h.to(dev) - b).abs().max())}"


def test_per_member_dt(dev):
    from snapy_linfel_b200.mesh import MeshBlockF32

    members = small_members(n=3, seed=5)
    ens, _ = batched(members, 0, dev)
    ens.max_time_step()
    dts = ens.dts().cpu().numpy()
    for k, (opts, w, r) in enumerate(members):
        mb = MeshBlockF32(opts, device=dev)
        mb.initialize(w, r)
        assert float(mb.max_time_step()) == dts[k]


def test_autotuner_keeps_results(dev):
    members = small_members(n=4, seed=7)
    ref = singles(members, 1, dev)
    from snapy_linfel_b200.ensemble import Ensemble

    ens = Ensemble(members, device=dev)
    table = ens.tune(steps=1, candidates={"x1_columns": [0, 2], "ctas_per_sm": [0, 2]})
    assert table["best"] and len(table["trials"]) == 4
    ens.step()
    for a, b in zip([b.hydro_u for b in ens.blocks], ref):
        assert torch.equal(a, b)


@pytest.mark.parametrize("kernel,env", [(1, "cr"), (2, "fused")])
def test_implicit_variants_batched_equal_one_block(dev, monkeypatch, kernel, env):
    """block cyclic reduction (tuning vic_kernel = 1, SNAPB_VIC_KERNEL=cr for the
    one-block path) and the fused kernel (vic_kernel = 2, SNAPB_VIC_KERNEL=fused)
    give every member exactly the one-block result"""
    monkeypatch.setenv("SNAPB_VIC_KERNEL", env)
    members = small_members(n=4, seed=11)
    ref = singles(members, 2, dev)
    _, got = batched(members, 2, dev, tuning={"vic_kernel": kernel})
    for k, (a, b) in enumerate(zip(got, ref)):
        assert torch.equal(a, b), f"member {k}: max diff {float((a - b).abs().max())}"


def test_cyclic_reduction_agrees_with_block_thomas(dev):
    """block cyclic reduction and the block-Thomas column kernel (the default)
    eliminate the same system in FP64 in different orders: the FP32 states
    after two steps agree to a few FP32 ulps"""
    members = problems.ensemble_members(n=6, seed=13, horiz=(8, 12), vert=(7, 13, 16),
                                        riemann="lmars", implicit_scheme=1)
    _, th = batched(members, 2, dev)
    _, cr = batched(members, 2, dev, tuning={"vic_kernel": 1})
    for k, (a, b) in enumerate(zip(cr, th)):
        assert torch.isfinite(a).all()
        for v in range(a.shape[0]):
            scale = float(b[v].abs().max())
            err = float((a[v] - b[v]).abs().max())
            assert err <= 1e-5 * max(scale, 1e-30), f"member {k} var {v}: {err} vs {scale}"
