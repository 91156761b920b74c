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
    members = small_members(implicit_scheme=scheme, riemann=riemann)
    ref = singles(members, 3, dev)
    _, got = batched(members, 3, dev)
    for k, (a, b) in enumerate(zip(got, ref)):
        assert torch.equal(a, b), f"member {k}: max diff {float((a - b).abs().max())}"


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


def test_fused_implicit_variant_batched_equals_one_block(dev, monkeypatch):
    """the fused implicit-solve kernel (tuning vic_regs = 3, and
    SNAPB_VIC_KERNEL=fused for the one-block path) gives every member exactly
    the one-block result"""
    monkeypatch.setenv("SNAPB_VIC_KERNEL", "fused")
    members = small_members(n=4, seed=11)
    ref = singles(members, 2, dev)
    _, got = batched(members, 2, dev, tuning={"vic_regs": 3})
    for k, (a, b) in enumerate(zip(got, ref)):
        assert torch.equal(a, b), f"member {k}: max diff {float((a - b).abs().max())}"
