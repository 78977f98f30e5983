"""mtx_autotune: it times the candidates once per (dims, dtype, device) and
caches the choice in the process and in a file; the extraction it picks is
the same surface, bit-exact with the oracle for that block edge, and its
vertices are within 1e-6 relative of an FP64 recomputation of the
interpolation (the check of the gyroid workload)."""
import numpy as np
import pytest
import torch

from helpers import u32

pytestmark = pytest.mark.gpu


def _gyroid(shape):
    from meshtrex_b200 import synth
    return synth.gyroid(shape_zyx=shape, seed=2, device="cuda")


def test_autotune_picks_caches_and_reuses(ctx, oracle, tmp_path):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    vol = _gyroid((80, 72, 96))
    cache = str(tmp_path / "tune.txt")
    r1 = api.autotune(ctx, vol, 0.0, cache_path=cache, flags=L.AUTOTUNE_QUICK)
    # block edge x warps x staging, then the load-based min/max pass with 1, 2, 4 slices
    assert r1["fromCache"] == 0 and r1["candidates"] == 3 * 3 * 2 + 3
    assert r1["blockEdge"] in (4, 8, 16) and r1["ms"] > 0
    assert r1["tuning"]["extractWarps"] in (2, 4, 8) and r1["tuning"]["staging"] in (1, 2)
    lines = open(cache).read().splitlines()
    assert len(lines) == 1 and lines[0].startswith("96 72 80 2 ")
    before = ctx.get_tuning()
    r2 = api.autotune(ctx, vol, 0.0, cache_path=cache)
    assert r2["fromCache"] == 1 and r2["blockEdge"] == r1["blockEdge"] and r2["tuning"] == r1["tuning"]
    assert ctx.get_tuning() == before  # the context's tuning is left alone
    r3 = api.autotune(ctx, vol, 0.0, flags=L.AUTOTUNE_IGNORE_CACHE | L.AUTOTUNE_QUICK)
    assert r3["fromCache"] == 0

    # the chosen shape extracts the same mesh as the oracle for that block edge
    t = r1["tuning"]
    ctx.set_tuning(t["minmaxZChunk"], t["minmaxSlices"], t["extractWarps"], t["staging"])
    try:
        B = r1["blockEdge"]
        m = api.extract(vol, B, 0.0, ctx=ctx)
        a = vol.cpu().numpy()
        ids = oracle.compact(oracle.minmax_halo(a, B), oracle.F32, 0.0)
        np.testing.assert_array_equal(u32(m.active_ids), ids)
        ref = oracle.mc_extract(a, B, 0.0, ids, want_xyz64=True)
        xyz = m.vertices.cpu().numpy()
        np.testing.assert_array_equal(xyz.view(np.uint32), ref.xyz.view(np.uint32))
        np.testing.assert_array_equal(u32(m.indices), ref.indices)
        rel = np.abs(xyz.astype(np.float64) - ref.xyz64) / np.maximum(np.abs(ref.xyz64), 1.0)
        assert rel.max() <= 1e-6
    finally:
        ctx.set_tuning(0, 0, 0, 0)


def test_autotune_reads_a_cache_file_written_before(ctx, tmp_path):
    from meshtrex_b200 import api
    vol = torch.zeros((20, 24, 28), dtype=torch.float32, device="cuda")
    name = torch.cuda.get_device_name(0)
    cache = tmp_path / "tune.txt"
    cache.write_text(f"28 24 20 2 16 0 4 8 2 1.250000 {name}\n28 24 20 1 4 0 1 2 1 9.0 {name}\n")
    r = api.autotune(ctx, vol, 0.0, cache_path=str(cache))
    assert r["fromCache"] == 1 and r["blockEdge"] == 16 and r["ms"] == 1.25
    assert r["tuning"] == {"minmaxZChunk": 0, "minmaxSlices": 4, "extractWarps": 8, "staging": 2,
                           "extractCtasPerSm": 0}


def test_batch_autotune_picks_edges_caches_them_and_matches_oracle(ctx, oracle, tmp_path):
    """mtx_autotune_batch times the batched run for one edge for all volumes
    (4, 8, 16) and per-dtype changes; the choice is cached per the batch's
    (dims, dtype) list, read back from the file by a later call that ignores
    nothing, and the batch with those edges gives the oracle's meshes."""
    from helpers import blob_volume, mid_iso, to_cuda
    from meshtrex_b200 import api
    arrays = [blob_volume((24, 40, 32), np.uint8, seed=71), blob_volume((32, 24, 48), np.uint16, seed=72),
              blob_volume((40, 32, 24), np.float32, seed=73)]
    vols = [to_cuda(a) for a in arrays]
    jobs = [(v, mid_iso(a)) for v, a in enumerate(arrays)] + [(0, float(np.percentile(arrays[0], 30)))]
    cache = tmp_path / "batch_tune.txt"
    r1 = api.autotune_batch(ctx, vols, jobs, cache_path=str(cache), flags=1)  # ignore any cached choice
    assert r1["fromCache"] == 0 and r1["candidates"] >= 6 and r1["ms"] > 0
    assert all(e in (4, 8, 16) for e in r1["blockEdges"]) and len(r1["blockEdges"]) == 3
    assert r1["blockWarps"] in (0, 6)
    r2 = api.autotune_batch(ctx, vols, jobs, cache_path=str(cache))
    assert r2["fromCache"] == 1 and r2["blockEdges"] == r1["blockEdges"] and r2["blockWarps"] == r1["blockWarps"]
    assert "batch " in cache.read_text()
    b = api.Batch(ctx, vols, r1["blockEdges"], jobs, block_warps=r1["blockWarps"])
    try:
        b.run()
        res, tot = b.results()
        for (v, iso), r in zip(jobs, res):
            ref = oracle.extract(arrays[v], r1["blockEdges"][v], iso)
            gv, gi, _ = b.mesh(r)
            np.testing.assert_array_equal(gv.cpu().numpy().view(np.uint32), ref.xyz.view(np.uint32))
            np.testing.assert_array_equal(u32(gi), ref.indices)
    finally:
        b.close()
