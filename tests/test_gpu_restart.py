"""Restart round trip on the GPU: a block written after two steps and restored
into a fresh block continues bit for bit like the original."""
import pytest

from snapy_linfel_b200 import problems

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_restart_continues_bit_for_bit(tmp_path):
    from snapy_linfel_b200 import restart
    from snapy_linfel_b200.mesh import MeshBlock

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    opts, w, r = problems.large_3d(nx3=12, nx2=12, nx1=24, nscalar=2)
    a = MeshBlock(opts)
    a.initialize(w, r)
    for _ in range(2):
        a.step()
    p = a.write_restart(str(tmp_path), "blk", 1, current_time=3.5)
    path = restart.combine(str(tmp_path), "blk", 1)
    b = MeshBlock(opts)
    t = b.restore(restart.load_restart(path, 0))
    assert t == 3.5 and b.cycle == a.cycle == 2
    assert torch.equal(b.hydro_u, a.hydro_u) and torch.equal(b.scalar_s, a.scalar_s)
    for _ in range(2):
        a.step()
        b.step()
    assert torch.equal(b.hydro_u, a.hydro_u) and torch.equal(b.scalar_s, a.scalar_s)
    assert p.endswith("blk.block0.00001.part")
