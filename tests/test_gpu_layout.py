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


def test_pack_unpack_slab_kernels_match_tensor_slices():
    """snapb_pack_slab / snapb_unpack_slab move exactly the values of the
    tensor slices the message format is defined by (bit for bit)"""
    from snapy_linfel_b200.config import make_config
    from snapy_linfel_b200.layout import SlabLayout

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = make_config(nx1=10, nx2=12, nx3=8)
    g = torch.randn((7,) + tuple(c.shape[1:]), dtype=torch.float64, device="cuda")
    for dim, n in ((2, c.shape[2]), (1, c.shape[1])):
        for start, width in ((0, 3), (3, 3), (n - 6, 3), (n - 3, 3), (2, 5)):
            sl = slice(start, start + width)
            idx = [slice(None)] * 4
            idx[dim] = sl
            buf = SlabLayout.pack(c, g, dim, sl)
            torch.cuda.synchronize()
            assert torch.equal(buf, g[tuple(idx)].contiguous()), (dim, start)
            h = torch.zeros_like(g)
            SlabLayout.unpack(c, h, dim, sl, buf * 2.0)
            torch.cuda.synchronize()
            want = torch.zeros_like(g)
            want[tuple(idx)] = g[tuple(idx)] * 2.0
            assert torch.equal(h, want), (dim, start)
    from snapy_linfel_b200 import _lib

    bad = _lib.lib().snapb_pack_slab(__import__("ctypes").byref(c), 2, c.shape[2] - 2, 3,
                                     _lib.ptr(g), 7, _lib.ptr(g), _lib.stream_ptr())
    assert bad == 1 and b"outside" in _lib.lib().snapb_last_error()


def test_large_3d_shape_2x2_blocks_pack_path():
    """the large H2-He configuration's physics and column height (WENO5 + Roe
    + VIC, two tracers, 192 layers) on 2 x 2 blocks exchanged through the
    slab kernels reproduce the undivided block"""
    from snapy_linfel_b200.layout import SlabLayout

    opts, w, r = problems.large_3d(nx3=32, nx2=32, nx1=192, nscalar=2)
    _compare(opts, w, r, SlabLayout(2, 2, periodic_x=True, periodic_y=True), steps=2)
