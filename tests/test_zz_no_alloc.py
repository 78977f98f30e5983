"""The compaction entry point that allocates no memory.

mtx_filter_active_blocks_noalloc serves callers that cannot allocate device
memory while they run (a fixed device-memory budget, or code where cudaMalloc
is not allowed): it keeps its scratch in a fixed array inside the library.
These tests call it through the C ABI and check that it gives exactly what
the ordinary, allocating mtx_filter_active_blocks gives, on consecutive calls
that share that array.  The file sorts last so that a run stopping at the
first failure has run every other test already.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import blob_volume, to_cuda, u32

pytestmark = pytest.mark.gpu


def _noalloc(leaf_ptr, nblocks, dtype, iso):
    from meshtrex_b200 import _lib as L
    ids = torch.full((nblocks,), -1, dtype=torch.int32, device="cuda")
    rank = torch.full((nblocks,), -7, dtype=torch.int32, device="cuda")
    count = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    status = torch.full((4,), -1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    rc = L.lib().mtx_filter_active_blocks_noalloc(C.c_void_p(leaf_ptr), nblocks, dtype, float(iso),
                                                  C.c_void_p(ids.data_ptr()), C.c_void_p(rank.data_ptr()),
                                                  C.c_void_p(count.data_ptr()), C.c_void_p(status.data_ptr()),
                                                  C.c_void_p(s.cuda_stream))
    assert rc == 0, L.STATUS.get(rc, rc)
    torch.cuda.synchronize()
    assert int(status[0].item()) == 0
    n = int(count.item())
    return n, u32(ids[:n]), u32(rank)


def _allocating(ctx, mm, pc):
    from meshtrex_b200 import api
    f = api.filter_active_blocks(ctx, mm, pc)
    n = api.read_active_block_count(ctx, f)
    ids = u32(f.ids())
    rank = api.device_view(f.out.blockRankBuffer.ptr, (f.out.totalBlocks,), torch.int32).cpu().numpy().view(np.uint32)
    f.free()
    return n, ids, rank


@pytest.mark.parametrize("dtype,block", [(np.uint8, 4), (np.uint16, 8), (np.float32, 8)])
def test_noalloc_compaction_matches_allocating_path(dtype, block):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    a = blob_volume((40, 56, 64), dtype, seed=21)
    vol = to_cuda(a)
    ctx = api.Context(0)
    try:
        isos = [float(np.float32(np.percentile(a, q))) for q in (35, 65)]
        if dtype != np.float32:
            isos = [float(round(i)) for i in isos]
        dcode = {np.uint8: L.DTYPE_U8, np.uint16: L.DTYPE_U16, np.float32: L.DTYPE_F32}[dtype]
        v = api.wrap_volume(vol)
        for iso in isos + isos[:1]:  # consecutive calls reuse the same scratch array
            pc = api.push_constants((a.shape[2], a.shape[1], a.shape[0]), block, iso)
            mm = api.compute_min_max_mip(ctx, v, pc)
            ctx.synchronize()
            nb = int(mm.out.blockGridDim[0] * mm.out.blockGridDim[1] * mm.out.blockGridDim[2])
            want_n, want_ids, want_rank = _allocating(ctx, mm, pc)
            got_n, got_ids, got_rank = _noalloc(mm.out.minMaxImage.ptr, nb, dcode, iso)
            assert got_n == want_n > 0
            np.testing.assert_array_equal(got_ids, want_ids)
            np.testing.assert_array_equal(got_rank, want_rank)
            mm.free()
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_its_array():
    from meshtrex_b200 import _lib as L
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    p = C.c_void_p(dummy.data_ptr())
    rc = L.lib().mtx_filter_active_blocks_noalloc(p, 65536 * 1024 + 1, L.DTYPE_U8, 1.0, p, p, p, p, None)
    assert rc == 4  # MTX_ERR_CAPACITY, before any GPU work
    rc = L.lib().mtx_filter_active_blocks_noalloc(None, 16, L.DTYPE_U8, 1.0, p, p, p, p, None)
    assert rc == 1  # MTX_ERR_INVALID_ARG


def _build_context_program(out_dir):
    """tests/cpp/noalloc_contexts.cpp, linked against the library and the CUDA
    driver (the link-time stub; the driver itself is loaded at run time)."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib_dir = os.path.join(root, "meshtrex_b200")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    exe = os.path.join(str(out_dir), "noalloc_contexts")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(root, "include"),
           "-I", os.path.join(cuda, "include"), os.path.join(root, "tests", "cpp", "noalloc_contexts.cpp"),
           "-L", lib_dir, "-lmeshtrex_b200", f"-Wl,-rpath,{lib_dir}", "-L", os.path.join(cuda, "lib64", "stubs"),
           "-lcuda", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_noalloc_in_a_second_cuda_context(tmp_path, oracle):
    """The scratch array's device address belongs to a CUDA context: a call in
    a second context on the same device must look it up there, and a later
    call in the first context must still use the first one's."""
    import json
    import subprocess
    a = blob_volume((40, 56, 64), np.uint8, seed=23)
    keys = oracle.minmax_halo(a, 4)  # 10 x 14 x 16 = 2240 blocks: three 1024-block tiles
    iso = 128.5
    path = tmp_path / "keys.bin"
    keys.astype(np.uint32).tofile(path)
    exe = _build_context_program(tmp_path)
    r = subprocess.run([exe, str(path), "0", repr(iso)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    calls = json.loads(r.stdout.strip().splitlines()[-1])["calls"]
    ids = oracle.compact(keys, oracle.U8, iso)
    rank = np.full(keys.shape[0], 0xFFFFFFFF, np.uint32)
    rank[ids] = np.arange(len(ids), dtype=np.uint32)
    from test_gpu_facade import _fnv1a
    want = {"status": 0, "count": len(ids), "device_status": 0, "ids": _fnv1a(ids.astype(np.uint32).tobytes()),
            "rank": _fnv1a(rank.tobytes())}
    assert len(ids) > 0
    for c in calls:
        assert c == want
