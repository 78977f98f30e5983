"""The batched path against the plain drop-in path, job by job.

A batch of volumes of mixed sizes, dtypes and block edges, each extracted at
several isovalues, must give for every job exactly what the plain sequence
(compute_min_max_mip, filter_active_blocks, extract_meshlet_descriptors) gives
for that volume, block edge and isovalue: the same vertex bits, the same
indices (counted from the job's first vertex) and the same meshlet
descriptors.
"""
import numpy as np
import pytest
import torch

from helpers import blob_volume, to_cuda, u32

pytestmark = pytest.mark.gpu

MIX = [
    # shape (z, y, x), dtype, block edge
    ((24, 40, 32), np.uint8, 8),
    ((40, 16, 48), np.uint16, 8),
    ((32, 32, 64), np.float32, 4),
    ((17, 33, 29), np.uint8, 4),     # rows not 16-byte aligned: one-thread-per-block min/max
    ((48, 24, 16), np.uint16, 3),    # block edge outside the vector min/max set
    ((16, 16, 16), np.float32, 8),
]


def _isos(a, k, rng):
    qs = np.sort(rng.uniform(10, 90, size=k))
    out = [float(np.float32(np.percentile(a.astype(np.float64), q))) for q in qs]
    if a.dtype != np.float32:
        out = [float(round(v)) + (0.5 if a.dtype == np.uint8 else 0.0) for v in out]
    return out


def _mix(seed=5, with_big_block=False):
    rng = np.random.default_rng(seed)
    mix = list(MIX) + ([((40, 36, 48), np.uint16, 16)] if with_big_block else [])
    arrays, blocks, jobs = [], [], []
    for v, (shape, dt, B) in enumerate(mix):
        a = blob_volume(shape, dt, seed=100 + v)
        arrays.append(a)
        blocks.append(B)
        for iso in _isos(a, 1 + v % 4, rng):
            jobs.append((v, iso))
    # a job whose isovalue lies outside the volume's values: no active block
    jobs.append((0, 1000.0))
    return arrays, blocks, jobs


def _plain(ctx, vol, B, iso, options=None):
    from meshtrex_b200 import api
    m = api.extract(vol, B, iso, ctx=ctx, options=options)
    return (m.vertices.cpu().numpy().view(np.uint32), u32(m.indices), u32(m.meshlets))


def _check_batch(ctx, arrays, blocks, jobs, options=None, use_graph=True, runs=2):
    from meshtrex_b200 import api
    vols = [to_cuda(a) for a in arrays]
    b = api.Batch(ctx, vols, blocks, jobs, options=options, use_graph=use_graph)
    try:
        for _ in range(runs):  # a second run resets every counter and gives the same bits
            b.run()
        res, tot = b.results()
        assert tot["status"] == 0
        assert tot["activeBlocks"] == sum(r["meshletCount"] for r in res)
        assert tot["vertexCount"] == sum(r["vertexCount"] for r in res)
        assert 3 * tot["triangleCount"] == sum(r["indexCount"] for r in res)
        for (v, iso), r in zip(jobs, res):
            want_v, want_i, want_m = _plain(ctx, vols[v], blocks[v], iso, options)
            got_v, got_i, got_m = b.mesh(r)
            assert r["vertexCount"] == want_v.shape[0], (v, iso)
            assert r["indexCount"] == 3 * want_i.shape[0], (v, iso)
            assert r["meshletCount"] == want_m.shape[0], (v, iso)
            np.testing.assert_array_equal(got_v.cpu().numpy().view(np.uint32).reshape(-1), want_v.reshape(-1))
            np.testing.assert_array_equal(u32(got_i), want_i)
            np.testing.assert_array_equal(u32(got_m), want_m)
        # jobs are laid out back to back in job order
        assert res[0]["vertexOffset"] == 0 and res[0]["indexOffset"] == 0
        for p, q in zip(res, res[1:]):
            assert q["vertexOffset"] == p["vertexOffset"] + p["vertexCount"]
            assert q["indexOffset"] == p["indexOffset"] + p["indexCount"]
            assert q["meshletOffset"] == p["meshletOffset"] + p["meshletCount"]
        assert res[-1]["meshletCount"] == 0 and res[-1]["vertexCount"] == 0
        return res
    finally:
        b.close()


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_matches_plain_per_job(ctx, use_graph):
    arrays, blocks, jobs = _mix()
    _check_batch(ctx, arrays, blocks, jobs, use_graph=use_graph)


def test_batch_with_16_edge_blocks(ctx):
    arrays, blocks, jobs = _mix(seed=9, with_big_block=True)
    _check_batch(ctx, arrays, blocks, jobs)


def test_batch_vertex_data_ndc_normals(ctx):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    arrays, blocks, jobs = _mix(seed=11)
    opts = api.extract_options(vertex_format=L.VERTEX_DATA, frame=L.FRAME_NDC, normals=True)
    _check_batch(ctx, arrays, blocks, jobs, options=opts, runs=1)


@pytest.mark.parametrize("generic", [False, True])
def test_batch_all_edge_8(ctx, generic):
    """Every volume at block edge 8: the kernel instantiated with the edge at
    compile time."""
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    arrays, _, jobs = _mix(seed=17)
    opts = api.extract_options(vertex_format=L.VERTEX_DATA, frame=L.FRAME_NDC, normals=True) if generic else None
    _check_batch(ctx, arrays, [8] * len(arrays), jobs, options=opts, runs=2 - generic)


def test_batch_reports_capacity_with_needed_sizes(ctx):
    from meshtrex_b200 import api
    arrays, blocks, jobs = _mix(seed=13)
    vols = [to_cuda(a) for a in arrays]
    full = api.Batch(ctx, vols, blocks, jobs)
    full.run()
    _, need = full.results()
    full.close()
    assert need["status"] == 0 and need["activeBlocks"] > 8

    short_blocks = api.Batch(ctx, vols, blocks, jobs, max_active_blocks=need["activeBlocks"] - 1)
    short_blocks.run()
    _, tot = short_blocks.results(check=False)
    short_blocks.close()
    assert tot["status"] == 4  # MTX_ERR_CAPACITY
    assert tot["activeBlocks"] == need["activeBlocks"]

    short_verts = api.Batch(ctx, vols, blocks, jobs, vertex_capacity=need["vertexCount"] - 1,
                            triangle_capacity=need["triangleCount"])
    short_verts.run()
    _, tot = short_verts.results(check=False)
    short_verts.close()
    assert tot["status"] == 4
    assert tot["vertexCount"] == need["vertexCount"]
    assert tot["triangleCount"] == need["triangleCount"]

    exact = api.Batch(ctx, vols, blocks, jobs, max_active_blocks=need["activeBlocks"],
                      vertex_capacity=need["vertexCount"], triangle_capacity=need["triangleCount"])
    exact.run()
    _, tot = exact.results()
    exact.close()
    assert tot == need


def test_batch_rejects_bad_descriptions(ctx):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    vol = to_cuda(blob_volume((16, 16, 16), np.uint8, seed=1))
    with pytest.raises(L.MtxError):
        api.Batch(ctx, [vol], [8], [(1, 10.0)])  # job names no volume
    with pytest.raises(L.MtxError):
        api.Batch(ctx, [vol], [17], [(0, 10.0)])  # block edge outside 2..16
    with pytest.raises(L.MtxError):
        api.Batch(ctx, [vol], [8], [])
