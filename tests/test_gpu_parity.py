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


def _mesh_via_async(ctx, vol, block, iso, vcap, tcap, **kw):
    from meshtrex_b200 import api
    ex = api.AsyncExtractor(ctx, vol, block, iso, vcap, tcap, **kw)
    ex.run()
    ctx.synchronize()
    c = u32(ex.counters)
    V, T = int(c[0]), int(c[1]) // 3
    return ex.vertices[:V].cpu().numpy(), u32(ex.indices[:T]), c


@pytest.mark.parametrize("shape,dtype,block", [((40, 36, 48), np.uint8, 8), ((33, 40, 32), np.uint16, 4),
                                               ((48, 48, 48), np.float32, 16), ((30, 27, 26), np.uint16, 5)])
def test_async_whole_path_matches_oracle(ctx, oracle, shape, dtype, block):
    a = blob_volume(shape, dtype, seed=7)
    iso = mid_iso(a)
    ref = oracle.extract(a, block, iso)
    xyz, idx, c = _mesh_via_async(ctx, to_cuda(a), block, iso, ref.n_vertices + 7, ref.n_triangles + 3)
    assert c[4] == 0 and c[2] == len(ref.ids) and c[3] == len(ref.ids)
    np.testing.assert_array_equal(xyz.view(np.uint32), ref.xyz.view(np.uint32))
    np.testing.assert_array_equal(idx, ref.indices)


@pytest.mark.parametrize("slices", [1, 2, 4])
@pytest.mark.parametrize("warps", [1, 2, 8])
def test_tuning_variants_match_oracle(ctx, oracle, slices, warps):
    from meshtrex_b200 import api
    a = blob_volume((36, 40, 64), np.uint16, seed=11)
    iso = mid_iso(a)
    ref = oracle.extract(a, 8, iso)
    ctx.set_tuning(minmax_slices=slices, extract_warps=warps, minmax_zchunk=1 + slices % 3)
    try:
        m = api.extract(to_cuda(a), 8, iso, ctx=ctx)
        np.testing.assert_array_equal(u32(m.leaf).reshape(-1, 2), oracle.minmax_halo(a, 8))
        np.testing.assert_array_equal(m.vertices.cpu().numpy().view(np.uint32), ref.xyz.view(np.uint32))
        np.testing.assert_array_equal(u32(m.indices), ref.indices)
        xyz, idx, c = _mesh_via_async(ctx, to_cuda(a), 8, iso, ref.n_vertices, ref.n_triangles)
        np.testing.assert_array_equal(xyz.view(np.uint32), ref.xyz.view(np.uint32))
        np.testing.assert_array_equal(idx, ref.indices)
    finally:
        ctx.set_tuning()


@pytest.mark.parametrize("dtype", [np.uint8, np.float32])
def test_vertexdata_normals_and_ndc(ctx, oracle, dtype):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    a = blob_volume((34, 30, 32), dtype, seed=5)
    iso = mid_iso(a)
    ref = oracle.extract(a, 8, iso, frame=oracle.FRAME_NDC, want_normals=True)
    opts = api.extract_options(vertex_format=L.VERTEX_DATA, frame=L.FRAME_NDC, normals=True)
    m = api.extract(to_cuda(a), 8, iso, ctx=ctx, options=opts)
    v = m.vertices.cpu().numpy()
    assert v.shape == (ref.n_vertices, 8)
    np.testing.assert_array_equal(v[:, :3].view(np.uint32), ref.xyz.view(np.uint32))
    np.testing.assert_array_equal(v[:, 4:7].view(np.uint32), ref.normals.view(np.uint32))
    assert (v[:, 3] == 1.0).all() and (v[:, 7] == 0.0).all()
    # the same record written by the count pass (async path)
    xyz, idx, c = _mesh_via_async(ctx, to_cuda(a), 8, iso, ref.n_vertices, ref.n_triangles, options=opts)
    np.testing.assert_array_equal(xyz[:, 4:7].view(np.uint32), ref.normals.view(np.uint32))
    np.testing.assert_array_equal(idx, ref.indices)


def test_capacity_overflow_is_reported(ctx, oracle):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    a = blob_volume((40, 40, 48), np.uint8, seed=3)
    iso = mid_iso(a)
    ref = oracle.extract(a, 8, iso)
    ex = api.AsyncExtractor(ctx, to_cuda(a), 8, iso, ref.n_vertices // 2, ref.n_triangles // 2)
    ex.run()
    with pytest.raises(L.MtxError) as e:
        ctx.synchronize()
    assert e.value.status == 4  # MTX_ERR_CAPACITY
    c = u32(ex.counters)
    assert c[0] == ref.n_vertices and c[1] == 3 * ref.n_triangles and c[4] == 4
    ctx.synchronize()  # the error word was cleared
    # a bound on active blocks that is too small is reported the same way
    ex = api.AsyncExtractor(ctx, to_cuda(a), 8, iso, ref.n_vertices, ref.n_triangles,
                            max_active_blocks=max(1, len(ref.ids) // 2))
    ex.run()
    with pytest.raises(L.MtxError):
        ctx.synchronize()
    assert u32(ex.counters)[3] == len(ref.ids)
    ctx.synchronize()


def test_injected_allocation_failure(oracle):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    a = blob_volume((24, 24, 32), np.uint8, seed=1)
    c = api.Context(0)
    try:
        pc = api.push_constants((32, 24, 24), 8, 120.0)
        v = api.wrap_volume(to_cuda(a))
        c.fail_allocation(1)
        with pytest.raises(L.MtxError) as e:
            api.compute_min_max_mip(c, v, pc)
        assert e.value.status == 3  # MTX_ERR_OOM
        mm = api.compute_min_max_mip(c, v, pc)  # the next call allocates normally
        mm.free()
    finally:
        c.close()


def test_profiler_stage_names(ctx):
    from meshtrex_b200 import api
    a = blob_volume((32, 32, 32), np.uint8, seed=2)
    prof = api.Profiler(ctx)
    prof.begin_frame()
    api.extract(to_cuda(a), 8, 128.5, ctx=ctx, profiler=prof)
    prof.end_frame()
    r = prof.regions()
    for name in ("MinMax_Leaf_Pass", "MinMax_Octree_Reduction", "Active_Block_Filtering", "Mesh_Extraction"):
        assert name in r and r[name][0] > 0.0
    prof.close()


def test_invalid_arguments_are_rejected(ctx):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    a = blob_volume((16, 16, 16), np.uint8, seed=2)
    v = api.wrap_volume(to_cuda(a))
    pc = api.push_constants((16, 16, 16), 8, 100.0)
    pc.blockGridDim[0] = 3
    with pytest.raises(L.MtxError) as e:
        api.compute_min_max_mip(ctx, v, pc)
    assert e.value.status == 1
    pc = api.push_constants((16, 16, 16), 32, 100.0)
    with pytest.raises(L.MtxError) as e:
        api.compute_min_max_mip(ctx, v, pc)
    assert e.value.status == 2


def test_extraction_stream_overlaps_and_matches_oracle(oracle):
    """With an extraction stream (mtx_context_set_extract_stream), the whole-path
    call queues count, scan and emit there; back-to-back calls on the same
    context reuse its scratch only after the previous extraction, and a drop-in
    call afterwards joins it.  Every output must still be the oracle's, with the
    count and emit passes capped to two CTAs an SM."""
    from meshtrex_b200 import api
    a = blob_volume((48, 40, 64), np.uint16, seed=41)
    b = blob_volume((40, 48, 32), np.uint8, seed=42)
    isos_a = [mid_iso(a), float(np.percentile(a, 30))]
    refs = [oracle.extract(a, 8, iso) for iso in isos_a]
    va, vb = to_cuda(a), to_cuda(b)
    ls, xs = torch.cuda.Stream(), torch.cuda.Stream()
    c = api.Context(0, stream=ls)
    try:
        c.set_extract_stream(xs)
        c.set_tuning(extract_ctas_per_sm=2)
        exts = [api.AsyncExtractor(c, va, 8, iso, r.n_vertices + 5, r.n_triangles + 5) for iso, r in zip(isos_a, refs)]
        for _ in range(3):
            for e in exts:
                e.run()
        c.synchronize()
        for e, r in zip(exts, refs):
            cnt = u32(e.counters)
            assert cnt[4] == 0 and cnt[0] == r.n_vertices and cnt[1] == 3 * r.n_triangles
            np.testing.assert_array_equal(e.vertices[: r.n_vertices].cpu().numpy().view(np.uint32),
                                          r.xyz.view(np.uint32))
            np.testing.assert_array_equal(u32(e.indices[: r.n_triangles]), r.indices)
        # a drop-in call on the same context after an asynchronous one
        exts[0].run()
        iso_b = mid_iso(b)
        m = api.extract(vb, 4, iso_b, ctx=c)
        rb = oracle.extract(b, 4, iso_b)
        np.testing.assert_array_equal(m.vertices.cpu().numpy().view(np.uint32), rb.xyz.view(np.uint32))
        np.testing.assert_array_equal(u32(m.indices), rb.indices)
        c.set_extract_stream(None)
        exts[1].run()
        c.synchronize()
        assert u32(exts[1].counters)[0] == refs[1].n_vertices
    finally:
        c.close()
