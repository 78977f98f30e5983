"""The upload overlapped with the leaf min/max (mtx_upload_compute_min_max_mip).

The volume goes to the device in z-slabs and each slab's leaf pass runs as it
lands; the device volume and every min/max level must equal the oracle's and
what the two separate calls (mtx_volume_upload, mtx_compute_min_max_mip)
give, and the extraction that follows must be the oracle's mesh.  Shapes
cover slabs that do not divide the block grid, depths that are not a
multiple of the block edge, rows that are not 16-byte aligned (the load-based
leaf pass) and every dtype.
"""
import numpy as np
import pytest
import torch

from helpers import blob_volume, mid_iso, u32

pytestmark = pytest.mark.gpu


_PINNED = []  # page-locked allocations behind the arrays _pinned hands out


def _pinned(a: np.ndarray) -> np.ndarray:
    """A copy of `a` in page-locked host memory."""
    t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
    _PINNED.append(t)
    p = t.numpy().view(a.dtype).reshape(a.shape)
    p[...] = a
    return p


@pytest.mark.parametrize("shape,dtype,block", [
    ((130, 48, 64), np.uint16, 8),     # 17 block layers: slabs of 2, the last one short
    ((67, 40, 32), np.uint8, 4),       # depth not a multiple of the block edge
    ((96, 36, 64), np.float32, 16),
    ((50, 33, 41), np.uint8, 3),       # unaligned rows: the load-based leaf pass
    ((200, 32, 48), np.uint16, 4),
])
def test_upload_overlapped_minmax_matches_oracle(ctx, oracle, shape, dtype, block):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    a = blob_volume(shape, dtype, seed=sum(shape))
    host = _pinned(a)
    iso = mid_iso(a)
    pc = api.push_constants((shape[2], shape[1], shape[0]), block, iso)
    for _ in range(2):  # the second call reuses cached buffers and the context's copy stream
        v, mm = api.upload_compute_min_max_mip(ctx, host, pc)
        ctx.synchronize()
        dev = api.device_view(v.data.ptr, (a.size * a.itemsize,), torch.uint8).cpu().numpy()
        np.testing.assert_array_equal(dev, a.view(np.uint8).reshape(-1))
        grid = oracle.block_grid(a.shape, block)
        assert mm.levels == oracle.mip_levels(grid)
        np.testing.assert_array_equal(u32(mm.all_levels()), oracle.pyramid(oracle.minmax_halo(a, block), grid))
        # the rest of the drop-in sequence on the uploaded volume
        f = api.filter_active_blocks(ctx, mm, pc)
        api.read_active_block_count(ctx, f)
        x = api.extract_meshlet_descriptors(ctx, mm, f, pc)
        ctx.synchronize()
        ref = oracle.extract(a, block, iso)
        np.testing.assert_array_equal(x.vertices().cpu().numpy().view(np.uint32), ref.xyz.view(np.uint32))
        np.testing.assert_array_equal(u32(x.indices()), ref.indices)
        x.free()
        f.free()
        mm.free()
        api.free_volume(ctx, v)
        assert v.data.ptr is None or v.data.ptr == 0


def test_upload_overlapped_minmax_rejects_bad_arguments(ctx):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    import ctypes as C
    a = _pinned(np.zeros((16, 16, 16), np.uint8))
    pc = api.push_constants((16, 16, 16), 8, 1.0)
    pc.blockGridDim[0] = 5
    v, out = L.Volume(), L.MinMaxOutput()
    d = (C.c_uint32 * 3)(16, 16, 16)
    rc = L.lib().mtx_upload_compute_min_max_mip(ctx.handle, C.c_void_p(a.ctypes.data), d, L.DTYPE_U8, C.byref(pc),
                                                None, C.byref(v), C.byref(out))
    assert rc == 1  # MTX_ERR_INVALID_ARG
    rc = L.lib().mtx_upload_compute_min_max_mip(ctx.handle, None, d, L.DTYPE_U8, C.byref(pc), None, C.byref(v),
                                                C.byref(out))
    assert rc == 1
