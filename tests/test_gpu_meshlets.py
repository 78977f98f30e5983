"""Meshlet split (mtx_build_meshlets) against the oracle's restatement, bit for
bit, and the renderer's contract: every meshlet within its limits, its
triangles indexing only its own vertices, and the mesh rebuilt from the
meshlets equal to the extraction's."""
import numpy as np
import pytest

from helpers import blob_volume, mid_iso, to_cuda, u32

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,dtype,block,limits", [
    ((40, 36, 48), np.uint8, 8, (64, 126)),
    ((32, 40, 24), np.float32, 4, (64, 126)),
    ((48, 40, 48), np.uint16, 16, (64, 126)),
    ((40, 36, 48), np.uint8, 8, (12, 10)),
])
def test_meshlets_match_oracle_and_contract(ctx, oracle, shape, dtype, block, limits):
    from meshtrex_b200 import api
    a = blob_volume(shape, dtype, seed=41 + block)
    iso = mid_iso(a)
    vol = to_cuda(a)
    v = api.wrap_volume(vol)
    pc = api.push_constants((shape[2], shape[1], shape[0]), block, iso)
    mm = api.compute_min_max_mip(ctx, v, pc)
    f = api.filter_active_blocks(ctx, mm, pc)
    api.read_active_block_count(ctx, f)
    x = api.extract_meshlet_descriptors(ctx, mm, f, pc)
    ml = api.build_meshlets(ctx, x, *limits)
    ctx.synchronize()
    verts = x.vertices().cpu().numpy()
    idx = u32(x.indices())
    blocks = u32(x.meshlets())
    x.free()
    f.free()
    mm.free()

    want_d, want_v, want_i = oracle.meshlets(blocks[:, 3], idx, *limits)
    d = u32(ml.descriptors)
    np.testing.assert_array_equal(d, want_d)
    np.testing.assert_array_equal(u32(ml.vertex_ids), want_v)
    np.testing.assert_array_equal(u32(ml.indices), want_i)

    max_v, max_p = limits
    assert (d[:, 2] <= max_v).all() and (d[:, 3] <= max_p).all() and (d[:, 3] > 0).all()
    # triangles are covered in order, each meshlet's indices inside its own vertex range
    np.testing.assert_array_equal(d[:, 1] // 3, np.concatenate([[0], np.cumsum(d[:-1, 3])]))
    tri_meshlet = np.repeat(np.arange(len(d)), d[:, 3])
    mi = u32(ml.indices)
    lo = d[tri_meshlet, 0][:, None]
    hi = lo + d[tri_meshlet, 2][:, None]
    assert ((mi >= lo) & (mi < hi)).all()
    # the mesh rebuilt from the meshlets is the extraction's, vertex records gathered bit for bit
    np.testing.assert_array_equal(u32(ml.vertex_ids)[mi], idx)
    np.testing.assert_array_equal(ml.vertices.cpu().numpy().view(np.uint32),
                                  verts.view(np.uint32)[u32(ml.vertex_ids)])


def test_meshlet_limits_are_checked(ctx):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    a = blob_volume((24, 24, 24), np.uint8, seed=3)
    x_mesh = api.extract(to_cuda(a), 8, mid_iso(a), ctx=ctx)
    assert x_mesh.indices.shape[0] > 0
    out = L.MeshletOutput()
    ext = L.ExtractionOutput()
    import ctypes as C
    assert L.lib().mtx_build_meshlets(ctx.handle, C.byref(ext), 65, 126, C.byref(out)) == 1
    assert L.lib().mtx_build_meshlets(ctx.handle, C.byref(ext), 64, 0, C.byref(out)) == 1
    assert L.lib().mtx_build_meshlets(ctx.handle, C.byref(ext), 64, 126, C.byref(out)) == 0  # empty mesh
    assert out.meshletCount == 0
