"""Slab decomposition on one GPU: the blocks of a layout stepped side by side
(local CFL minimum, ghost exchange after every stage) reproduce the undivided
block through the C ABI.  Bound: 1e-12 of each field's largest magnitude
after 3 RK3 steps (the blocks' x2 / x3 spacing is recomputed from their own
coordinate ranges, which moves the last bit of the face areas)."""
import numpy as np
import pytest

from snapy_linfel_b200 import problems

from errnorm import assert_finite

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _compare(opts, w, r, layout, steps=3):
    from snapy_linfel_b200.layout import LocalSlabBlocks
    from snapy_linfel_b200.mesh import MeshBlock

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    whole = MeshBlock(opts)
    whole.initialize(w, r)
    parts = LocalSlabBlocks(opts, layout)
    parts.initialize(w, r)
    for _ in range(steps):
        whole.step()
        parts.step()
    torch.cuda.synchronize()
    assert abs(float(whole.dt) / float(parts.blocks[0].dt) - 1.0) < 1e-12  # the CFL minimum
    it = (slice(None),) + opts.hydro.interior()
    a = parts.gather()[it].cpu().numpy()
    b = whole.hydro_u[it].cpu().numpy()
    assert_finite(a, b)
    for v in range(a.shape[0]):
        scale = max(np.abs(b[v]).max(), 1e-300)
        assert np.abs(a[v] - b[v]).max() / scale < 1e-12, v
    if whole.scalar_s is not None:
        sa = parts.gather("scalar_s")[it].cpu().numpy()
        sb = whole.scalar_s[it].cpu().numpy()
        assert_finite(sa, sb)
        assert np.abs(sa - sb).max() / np.abs(sb).max() < 1e-12


def test_two_x2_slabs_straka_implicit():
    from snapy_linfel_b200.layout import SlabLayout

    opts, w, _ = problems.straka(nx2=64, nx1=24, implicit_scheme=1)
    _compare(opts, w, None, SlabLayout(2, 1))


def test_2x2_slabs_3d_periodic_roe_tracers():
    from snapy_linfel_b200.layout import SlabLayout

    opts, w, r = problems.large_3d(nx3=16, nx2=16, nx1=24, nscalar=2)
    _compare(opts, w, r, SlabLayout(2, 2, periodic_x=True, periodic_y=True), steps=2)
