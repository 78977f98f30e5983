"""Small extraction cases run against the bounds-check build of the library.

Run by tests/test_gpu_bounds_check.py in a child process whose
MESHTREX_B200_LIB names libmeshtrex_b200_check.so: every checked shared- and
global-memory index of the kernels is tested, and mtx_synchronize reports the
first one out of range as MTX_ERR_INTERNAL.  Each case must raise nothing and
give the oracle's mesh.  Prints one line per case and "all cases passed".
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402
import torch  # noqa: E402

from helpers import blob_volume, mid_iso, to_cuda, u32  # noqa: E402


def main():
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    from oracle import oracle as O
    lib_path = os.path.realpath(L.LIB_PATH)
    L.lib()
    maps = open("/proc/self/maps").read()
    assert lib_path in maps and lib_path.endswith("_check.so"), lib_path
    print("library", lib_path)
    ctx = api.Context(0)
    cases = [((32, 32, 32), np.uint8, 8, "tma"), ((37, 29, 41), np.uint8, 4, "ldg"), ((48, 40, 64), np.uint16, 8, "tma"),
             ((33, 31, 30), np.uint16, 3, "ldg"), ((40, 36, 32), np.float32, 8, "tma"),
             ((50, 47, 64), np.uint16, 16, "tma"), ((21, 19, 32), np.uint8, 2, "ldg"), ((17, 16, 16), np.float32, 8, "ldg"),
             # several x-strips of the leaf pass: strip-start column records and their patch
             ((24, 20, 600), np.uint16, 8, "tma"), ((20, 18, 300), np.float32, 4, "tma")]
    for shape, dt, B, staging in cases:
        a = blob_volume(shape, dt, seed=sum(shape) + B)
        iso = mid_iso(a)
        st = L.STAGING_TMA if staging == "tma" else L.STAGING_LDG
        m = api.extract(to_cuda(a), B, iso, ctx=ctx, options=api.extract_options(staging=st))
        ref = O.extract(a, B, iso)
        assert np.array_equal(m.vertices.cpu().numpy().view(np.uint32), ref.xyz.view(np.uint32)), (shape, dt, B)
        assert np.array_equal(u32(m.indices), ref.indices), (shape, dt, B)
        ex = api.AsyncExtractor(ctx, to_cuda(a), B, iso, ref.n_vertices, ref.n_triangles)
        ex.run()
        ctx.synchronize()
        assert np.array_equal(u32(ex.indices), ref.indices)
        print("plain and asynchronous", shape, np.dtype(dt).name, B, staging, "ok", flush=True)
    # VertexData with normals in the NDC frame
    a = blob_volume((34, 30, 32), np.uint8, seed=5)
    iso = mid_iso(a)
    opts = api.extract_options(vertex_format=L.VERTEX_DATA, frame=L.FRAME_NDC, normals=True)
    m = api.extract(to_cuda(a), 8, iso, ctx=ctx, options=opts)
    ref = O.extract(a, 8, iso, frame=O.FRAME_NDC, want_normals=True)
    assert np.array_equal(m.vertices.cpu().numpy()[:, 4:7].view(np.uint32), ref.normals.view(np.uint32))
    print("VertexData, normals, NDC ok", flush=True)
    # a small batch of mixed dtypes and block edges
    vols = [blob_volume((24, 40, 32), np.uint8, seed=3), blob_volume((32, 24, 16), np.uint16, seed=4),
            blob_volume((20, 20, 36), np.float32, seed=5)]
    blocks = [8, 4, 8]
    jobs = [(v, mid_iso(a)) for v, a in enumerate(vols)]
    b = api.Batch(ctx, [to_cuda(a) for a in vols], blocks, jobs)
    b.run()
    res, tot = b.results()
    assert tot["status"] == 0
    for (v, iso), r in zip(jobs, res):
        ref = O.extract(vols[v], blocks[v], iso)
        gv, gi, _ = b.mesh(r)
        assert np.array_equal(gv.cpu().numpy().view(np.uint32), ref.xyz.view(np.uint32))
        assert np.array_equal(u32(gi), ref.indices)
    b.close()
    print("batch ok", flush=True)
    ctx.synchronize()
    ctx.close()
    print("all cases passed", flush=True)


if __name__ == "__main__":
    main()
