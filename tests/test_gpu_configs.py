"""The CUDA path against the oracle where the numbers are quoted.

Every workload the bench reports on is checked bit for bit against the CPU
oracle on the same bytes -- at full size where the oracle finishes in
seconds on all host threads, else on stated crops -- together with
meshtrex's own fixtures:

  - 256^3 uint8 Gaussian blobs (seed 0), block 8, isovalue 128;
  - the 1024^3 uint16 fBm ball (seed 1), block 8, at 16384, 32768 and 49152;
  - the 2048^3 float32 gyroid (seed 2), isovalue 0: 256^3 crops at block 4,
    8 and 16 and a 2048 x 2048 x 64 z-slab at block 8, with vertices also
    within 1e-6 of the oracle's FP64 interpolation;
  - the 64-volume batched mix (seed 3): every job of the mix with edges
    divided by 4, and the first volumes' jobs at full size;
  - generateSphereVolume(64, 64, 64) at isovalue 128 (src/meshtrex.cpp:23-52,
    72-73) at main's block edge 3, and at 4 and 8;
  - main's shape, 1024 x 1024 x 314 uint8 at block 3 and isovalue 80
    (src/meshtrex.cpp:56-84: a 342 x 342 x 105 block grid);
  - the committed 256^3 golden volume at block 4 and 8.

Volumes too large to generate on the CPU are generated on the device and
copied to the host, so both sides read the same bytes.
"""
import os

import numpy as np
import pytest
import torch

from helpers import to_cuda, to_numpy, u32

pytestmark = pytest.mark.gpu


def _threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _check_plain(ctx, oracle, a, block, iso, fp64=False, vol=None):
    """The drop-in sequence on the device against oracle.extract on the host:
    leaf min/max keys, active ids, per-block counts, vertex bits, indices."""
    from meshtrex_b200 import api
    vol = to_cuda(a) if vol is None else vol
    m = api.extract(vol, block, iso, ctx=ctx)
    ref = oracle.extract(a, block, iso, nthreads=_threads(), want_xyz64=fp64)
    np.testing.assert_array_equal(u32(m.leaf).reshape(-1, 2), oracle.minmax_halo(a, block, _threads()))
    np.testing.assert_array_equal(u32(m.active_ids), ref.ids)
    ml = u32(m.meshlets)
    assert ml.shape[0] == len(ref.ids)
    np.testing.assert_array_equal(ml[:, 2], ref.nvert_per_block)
    np.testing.assert_array_equal(ml[:, 3], ref.ntri_per_block)
    xyz = m.vertices.cpu().numpy()
    assert xyz.shape == ref.xyz.shape
    np.testing.assert_array_equal(xyz.view(np.uint32), ref.xyz.view(np.uint32))
    np.testing.assert_array_equal(u32(m.indices), ref.indices)
    if fp64 and ref.n_vertices:
        rel = np.abs(xyz.astype(np.float64) - ref.xyz64) / np.maximum(np.abs(ref.xyz64), 1.0)
        assert rel.max() <= 1e-6
    return ref.n_vertices, ref.n_triangles


# ------------------------------------------------------------ 256^3 blobs
def test_blobs_256_u8_block8_iso128(ctx, oracle):
    from meshtrex_b200 import synth
    a = to_numpy(synth.blobs(256, seed=0))
    V, T = _check_plain(ctx, oracle, a, 8, 128.0, fp64=True)
    assert V > 10000 and T > 10000


# ------------------------------------------------------- 1024^3 fBm ball
@pytest.fixture(scope="module")
def fbm_ball():
    from meshtrex_b200 import synth
    vol = synth.fbm_ball(1024, seed=1, device="cuda")
    torch.cuda.synchronize()
    yield vol, to_numpy(vol)
    del vol
    torch.cuda.empty_cache()


@pytest.mark.parametrize("iso", [16384.0, 32768.0, 49152.0])
def test_fbm_ball_1024_u16_block8(ctx, oracle, fbm_ball, iso):
    vol, a = fbm_ball
    V, T = _check_plain(ctx, oracle, a, 8, iso, vol=vol)
    assert T > 1_000_000


def test_fbm_ball_1024_async_path_matches_oracle(ctx, oracle, fbm_ball):
    """The asynchronous whole-path call the bench times, at the bench's size."""
    from meshtrex_b200 import api
    vol, a = fbm_ball
    iso = 32768.0
    ref = oracle.extract(a, 8, iso, nthreads=_threads())
    ex = api.AsyncExtractor(ctx, vol, 8, iso, ref.n_vertices, ref.n_triangles, max_active_blocks=len(ref.ids))
    ex.run()
    ctx.synchronize()
    c = u32(ex.counters)
    assert list(c[:5]) == [ref.n_vertices, 3 * ref.n_triangles, len(ref.ids), len(ref.ids), 0]
    np.testing.assert_array_equal(ex.vertices.cpu().numpy().view(np.uint32), ref.xyz.view(np.uint32))
    np.testing.assert_array_equal(u32(ex.indices), ref.indices)


# -------------------------------------------------------- 2048^3 gyroid
@pytest.fixture(scope="module")
def gyroid_2048():
    from meshtrex_b200 import synth
    vol = synth.gyroid(2048, seed=2, device="cuda")
    torch.cuda.synchronize()
    yield vol
    del vol
    torch.cuda.empty_cache()


@pytest.mark.parametrize("z0,y0,x0", [(0, 0, 0), (896, 1000, 1536)])
@pytest.mark.parametrize("block", [4, 8, 16])
def test_gyroid_crop_256_f32(ctx, oracle, gyroid_2048, z0, y0, x0, block):
    crop = gyroid_2048[z0:z0 + 256, y0:y0 + 256, x0:x0 + 256].contiguous()
    a = to_numpy(crop)
    V, T = _check_plain(ctx, oracle, a, block, 0.0, fp64=True, vol=crop)
    assert T > 100_000


def test_gyroid_zslab_2048x2048x64_f32(ctx, oracle, gyroid_2048):
    slab = gyroid_2048[1000:1064].contiguous()
    a = to_numpy(slab)
    _check_plain(ctx, oracle, a, 8, 0.0, fp64=True, vol=slab)


# ------------------------------------------------------- batched mix
def _batch_vs_oracle(ctx, oracle, items, block=8):
    from meshtrex_b200 import api
    vols = [it.volume for it in items]
    jobs = [(v, iso) for v, it in enumerate(items) for iso in it.isovalues]
    b = api.Batch(ctx, vols, [block] * len(vols), jobs, use_graph=True)
    try:
        b.run()
        res, tot = b.results()
        assert tot["status"] == 0
        hosts = [to_numpy(v) for v in vols]
        for (v, iso), r in zip(jobs, res):
            ref = oracle.extract(hosts[v], block, iso, nthreads=_threads())
            gv, gi, gm = b.mesh(r)
            assert (r["meshletCount"], r["vertexCount"], r["indexCount"]) == \
                (len(ref.ids), ref.n_vertices, 3 * ref.n_triangles), (v, iso)
            np.testing.assert_array_equal(gv.cpu().numpy().view(np.uint32), ref.xyz.view(np.uint32))
            np.testing.assert_array_equal(u32(gi), ref.indices)
            ml = u32(gm)
            np.testing.assert_array_equal(ml[:, 2], ref.nvert_per_block)
            np.testing.assert_array_equal(ml[:, 3], ref.ntri_per_block)
        return len(jobs)
    finally:
        b.close()


def test_batch_mix_quarter_every_job(ctx, oracle):
    from meshtrex_b200 import synth
    items = synth.batch(seed=3, n=64, device="cuda", scale_down=4)
    assert _batch_vs_oracle(ctx, oracle, items) > 400


def test_batch_mix_full_size_first_volumes(ctx, oracle):
    from meshtrex_b200 import synth
    items = synth.batch(seed=3, n=64, device="cuda")
    items = items[:4] + items[5:8]  # uint8, uint16 and float32 volumes, 68 jobs
    assert _batch_vs_oracle(ctx, oracle, items) >= 60


# -------------------------------------------------- meshtrex's fixtures
@pytest.mark.parametrize("block", [3, 4, 8])
def test_sphere_fixture_64_iso128(ctx, oracle, block):
    from golden.fixtures import sphere_volume
    a = sphere_volume(64, 64, 64)
    V, T = _check_plain(ctx, oracle, a, block, 128.0, fp64=True)
    assert T > 1000


def test_main_shape_1024x1024x314_u8_block3_iso80(ctx, oracle):
    from meshtrex_b200 import synth
    vol = synth.blob_field((314, 1024, 1024), seed=5, device="cuda")
    torch.cuda.synchronize()
    a = to_numpy(vol)
    from meshtrex_b200 import api
    pc = api.push_constants((1024, 1024, 314), 3, 80.0)
    assert tuple(pc.blockGridDim[:3]) == (342, 342, 105)
    V, T = _check_plain(ctx, oracle, a, 3, 80.0, vol=vol)
    assert T > 100_000


@pytest.mark.parametrize("block", [4, 8])
@pytest.mark.parametrize("iso", [40.0, 80.0, 128.0, 200.0])
def test_golden_volume_256(ctx, oracle, block, iso):
    from golden.make_golden import golden_volume
    _check_plain(ctx, oracle, golden_volume(), block, iso)
