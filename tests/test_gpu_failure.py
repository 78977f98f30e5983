"""Failure detection of the bounded device waits, without a GPU fault.

The compaction and the count scan resolve their offsets with decoupled
look-back: a tile waits for the tiles before it.  mtx_debug_set_waits makes
those waits give up after a few thousand polls and makes the next launch skip
the ticket of its first tile, so that the tiles after it wait for a
predecessor that never publishes (a flag that nothing sets).  They must give
up, report MTX_ERR_TIMEOUT through mtx_synchronize, leave the context usable,
and the next call without the injection must be the oracle's mesh again.
"""
import numpy as np
import pytest

from helpers import blob_volume, mid_iso, to_cuda, u32

pytestmark = pytest.mark.gpu

TIMEOUT = 5  # MTX_ERR_TIMEOUT


def _volume():
    # 40^3 blocks of edge 4: 16 compaction tiles of 4096 blocks, and more than
    # 1024 active blocks, so the count scan has several tiles too
    a = blob_volume((160, 160, 160), np.uint8, seed=61)
    return a, mid_iso(a)


@pytest.mark.parametrize("withhold,what", [(1, "compaction"), (2, "count scan")])
def test_withheld_lookback_tile_times_out_and_the_context_recovers(oracle, withhold, what):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    a, iso = _volume()
    ref = oracle.extract(a, 4, iso)
    assert len(ref.ids) > 2048
    vol = to_cuda(a)
    c = api.Context(0)
    try:
        ex = api.AsyncExtractor(c, vol, 4, iso, ref.n_vertices, ref.n_triangles)
        ex.run()
        c.synchronize()  # a clean run first: every tile takes part
        c.set_waits(max_polls=4096, withhold=withhold)
        ex.run()
        with pytest.raises(L.MtxError) as e:
            c.synchronize()
        assert e.value.status == TIMEOUT, what
        assert u32(ex.counters)[4] == TIMEOUT
        c.synchronize()  # the error word was read and cleared
        c.set_waits()
        ex.counters.zero_()
        ex.run()
        c.synchronize()
        cnt = u32(ex.counters)
        assert list(cnt[:5]) == [ref.n_vertices, 3 * ref.n_triangles, len(ref.ids), len(ref.ids), 0]
        np.testing.assert_array_equal(ex.vertices.cpu().numpy().view(np.uint32), ref.xyz.view(np.uint32))
        np.testing.assert_array_equal(u32(ex.indices), ref.indices)
    finally:
        c.close()


def test_withheld_compaction_tile_fails_the_drop_in_count_read(oracle):
    """The drop-in sequence reads the active count back: the timeout surfaces
    there, as readActiveBlockCount's error, and the next sequence succeeds."""
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    a, iso = _volume()
    vol = to_cuda(a)
    c = api.Context(0)
    try:
        v = api.wrap_volume(vol)
        pc = api.push_constants((a.shape[2], a.shape[1], a.shape[0]), 4, iso)
        mm = api.compute_min_max_mip(c, v, pc)
        c.set_waits(max_polls=4096, withhold=1)
        f = api.filter_active_blocks(c, mm, pc)
        with pytest.raises(L.MtxError) as e:
            api.read_active_block_count(c, f)
        assert e.value.status == TIMEOUT
        f.free()
        c.set_waits()
        f = api.filter_active_blocks(c, mm, pc)
        n = api.read_active_block_count(c, f)
        assert n == len(oracle.compact(oracle.minmax_halo(a, 4), oracle.U8, iso))
        f.free()
        mm.free()
    finally:
        c.close()


def test_wait_injection_rejects_unknown_bits():
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    c = api.Context(0)
    try:
        with pytest.raises(L.MtxError) as e:
            c.set_waits(withhold=4)
        assert e.value.status == 1
    finally:
        c.close()
