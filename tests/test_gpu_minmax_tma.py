"""The TMA-fed leaf min/max pass (the default for 2- and 4-byte voxels whose
rows are 16-byte aligned) against the oracle's (B+1)^3 block min/max, bit for
bit, and against the load-based pass (min/max slices 1, 2, 4) on the same
volume.  Shapes cover partial x-strips (X not a multiple of the 512-byte
strip), partial groups of four block rows, partial runs of z slabs, volumes
smaller than one strip, and every block edge the pass takes.  With one block
per lane and even z runs the pass also writes octree level 1; odd block-grid
extents give level-1 texels with missing children in x, y and z."""
import numpy as np
import pytest

from helpers import blob_volume, mid_iso, to_cuda, u32

pytestmark = pytest.mark.gpu

CASES = [
    # shape (z, y, x), dtype, block edge, z-chunk override (0: default)
    ((40, 36, 264), np.uint16, 8, 0),    # two strips, the second 8 voxels wide
    ((67, 45, 24), np.uint16, 8, 0),     # one narrow strip, partial row group, partial z slab
    ((33, 40, 256), np.uint16, 4, 0),    # one full strip, halo column outside the volume
    ((50, 47, 520), np.uint16, 16, 0),   # three strips, block rows past Y
    ((90, 17, 16), np.uint16, 8, 3),     # tall volume, runs of 3 slabs
    ((40, 36, 132), np.float32, 8, 0),   # float: 128-voxel strips
    ((31, 29, 20), np.float32, 4, 0),
    ((48, 48, 136), np.float32, 16, 1),  # runs of one slab
    ((72, 40, 264), np.uint16, 8, 2),    # level 1 in the pass: grid 33 x 5 x 9, the last slab unpaired
    ((56, 24, 136), np.float32, 8, 4),   # level 1, two lanes a block: grid 17 x 3 x 7
    ((40, 40, 264), np.uint16, 16, 2),   # level 1, block 16: grid 17 x 3 x 3
    # strip-start column records merged into the previous strip's last block (and its level-1 texel)
    ((24, 20, 600), np.uint16, 4, 0),    # two blocks a lane, three strips, the last one partial
    ((40, 24, 384), np.float32, 4, 2),   # level 1, one block a lane: three full strips of 128 voxels
    ((34, 41, 1024), np.uint16, 8, 0),   # four full strips: the 1024-voxel rows of the bench volume
]


@pytest.mark.parametrize("shape,dtype,block,zchunk", CASES)
def test_tma_leaf_matches_oracle(ctx, oracle, shape, dtype, block, zchunk):
    from meshtrex_b200 import api
    a = blob_volume(shape, dtype, seed=sum(shape) * 3 + block)
    iso = mid_iso(a)
    pc = api.push_constants((shape[2], shape[1], shape[0]), block, iso)
    ctx.set_tuning(minmax_zchunk=zchunk)
    try:
        mm = api.compute_min_max_mip(ctx, api.wrap_volume(to_cuda(a)), pc)
        ctx.synchronize()
        leaf = oracle.minmax_halo(a, block)
        grid = oracle.block_grid(a.shape, block)
        np.testing.assert_array_equal(u32(mm.all_levels()), oracle.pyramid(leaf, grid))
        mm.free()
    finally:
        ctx.set_tuning()


@pytest.mark.parametrize("dtype", [np.uint16, np.float32])
def test_tma_leaf_equals_load_based_pass(ctx, dtype):
    from meshtrex_b200 import api
    a = blob_volume((137, 129, 392), dtype, seed=23)
    vol = to_cuda(a)
    pc = api.push_constants((a.shape[2], a.shape[1], a.shape[0]), 8, mid_iso(a))
    got = {}
    for slices in (0, 1, 2, 4):
        ctx.set_tuning(minmax_slices=slices)
        try:
            mm = api.compute_min_max_mip(ctx, api.wrap_volume(vol), pc)
            ctx.synchronize()
            got[slices] = u32(mm.all_levels()).copy()
            mm.free()
        finally:
            ctx.set_tuning()
    for slices in (1, 2, 4):
        np.testing.assert_array_equal(got[0], got[slices])
