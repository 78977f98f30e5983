"""Parity of the CUDA path with the CPU oracle on the same seeded volumes.

Every stage is compared bit for bit: block min/max keys (every mip level),
the compacted active-block list, per-block vertex/triangle counts (meshlet
descriptors), per-cell case indices, vertex positions (FP32 bits) and the
index buffer.
"""
import numpy as np
import pytest
import torch

from helpers import blob_volume, mid_iso, to_cuda, u32

pytestmark = pytest.mark.gpu

CASES = [
    # shape (z, y, x), dtype, block edge, staging
    ((32, 32, 32), np.uint8, 8, "tma"),
    ((32, 32, 32), np.uint8, 8, "ldg"),
    ((37, 29, 48), np.uint8, 4, "tma"),
    ((37, 29, 41), np.uint8, 4, "ldg"),      # rows not 16-byte aligned: generic min/max, plain loads
    ((48, 40, 64), np.uint16, 8, "tma"),
    ((33, 31, 30), np.uint16, 3, "ldg"),     # the block edge meshtrex's main uses
    ((40, 36, 32), np.float32, 8, "tma"),
    ((64, 48, 64), np.float32, 16, "tma"),
    ((50, 47, 64), np.uint16, 16, "tma"),
    ((21, 19, 32), np.uint8, 2, "ldg"),
    ((17, 16, 16), np.float32, 8, "ldg"),
]


def _staging(name):
    from meshtrex_b200 import _lib as L
    return {"tma": L.STAGING_TMA, "ldg": L.STAGING_LDG, "auto": L.STAGING_AUTO}[name]


@pytest.mark.parametrize("shape,dtype,block,staging", CASES)
def test_plain_path_matches_oracle(ctx, oracle, shape, dtype, block, staging):
    from meshtrex_b200 import api
    a = blob_volume(shape, dtype, seed=sum(shape) + block)
    iso = mid_iso(a)
    vol = to_cuda(a)
    B = block
    ncell = B ** 3
    pc = api.push_constants((shape[2], shape[1], shape[0]), B, iso)
    v = api.wrap_volume(vol)
    mm = api.compute_min_max_mip(ctx, v, pc)
    f = api.filter_active_blocks(ctx, mm, pc)
    n = api.read_active_block_count(ctx, f)

    # stage 1: every level of the min/max octree
    leaf = oracle.minmax_halo(a, B)
    grid = oracle.block_grid(a.shape, B)
    pyr = oracle.pyramid(leaf, grid)
    assert mm.levels == oracle.mip_levels(grid)
    got = u32(mm.all_levels())
    np.testing.assert_array_equal(got, pyr)

    # stage 2: ordered compaction
    ids = oracle.compact(leaf, oracle.dtype_code(a), iso)
    assert n == len(ids)
    np.testing.assert_array_equal(u32(f.ids()), ids)

    # stage 3
    cases = torch.zeros(max(n, 1) * ncell, dtype=torch.uint8, device="cuda")
    opts = api.extract_options(staging=_staging(staging), cell_cases=cases)
    x = api.extract_meshlet_descriptors(ctx, mm, f, pc, opts)
    ctx.synchronize()
    ref = oracle.mc_extract(a, B, iso, ids, want_xyz64=True)
    assert x.vertex_count == ref.n_vertices
    assert x.index_count == 3 * ref.n_triangles
    assert x.meshlet_count == n
    if n:
        ml = u32(x.meshlets())
        np.testing.assert_array_equal(ml[:, 2], ref.nvert_per_block)
        np.testing.assert_array_equal(ml[:, 3], ref.ntri_per_block)
        np.testing.assert_array_equal(ml[:, 0], np.concatenate([[0], np.cumsum(ref.nvert_per_block)[:-1]]))
        np.testing.assert_array_equal(cases.cpu().numpy()[: n * ncell].reshape(n, ncell),
                                      oracle.cell_cases(a, B, iso, ids))
    xyz = x.vertices().cpu().numpy()
    np.testing.assert_array_equal(xyz.view(np.uint32), ref.xyz.view(np.uint32))
    np.testing.assert_array_equal(u32(x.indices()), ref.indices)
    if ref.n_vertices:
        rel = np.abs(xyz.astype(np.float64) - ref.xyz64) / np.maximum(np.abs(ref.xyz64), 1.0)
        assert rel.max() <= 1e-6
    cnt = u32(x.counters())
    assert list(cnt) == [ref.n_vertices, 3 * ref.n_triangles, n]
    x.free()
    f.free()
    mm.free()
