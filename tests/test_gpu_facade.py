"""The C++ drop-in facade on the GPU: a program written like meshtrex's main
(tests/cpp/drop_in_main.cpp) gives the same mesh bits as the Python drop-in
path, its OBJ passes the weld check, and mtx_volume_load streams raw files to
the device byte for byte."""
import ctypes as C
import json
import subprocess

import numpy as np
import pytest
import torch

from helpers import blob_volume, mid_iso, to_cuda
from test_facade import build_program

pytestmark = pytest.mark.gpu


def _fnv1a(b: bytes) -> str:
    h = 1469598103934665603
    for c in b:
        h = ((h ^ c) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return f"{h:016x}"


@pytest.mark.parametrize("dtype,tname", [(np.uint16, "uint16"), (np.uint8, "uint8"), (np.float32, "float32")])
def test_facade_program_matches_python_drop_in(ctx, tmp_path, dtype, tname):
    from meshtrex_b200 import api
    a = blob_volume((30, 36, 40), dtype, seed=31)
    iso = mid_iso(a)
    raw = tmp_path / f"blob_{a.shape[2]}x{a.shape[1]}x{a.shape[0]}_{tname}.raw"
    a.tofile(raw)
    exe = build_program(tmp_path)
    obj = tmp_path / "mesh.obj"
    r = subprocess.run([exe, str(raw), "8", repr(iso), str(obj)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    got = json.loads(r.stdout.strip().splitlines()[-1])

    m = api.extract(to_cuda(a), 8, iso, ctx=ctx)
    V, T = m.vertices.shape[0], m.indices.shape[0]
    assert got["vertices"] == V and got["indices"] == 3 * T
    assert got["activeBlocks"] == got["meshlets"] == m.active_ids.shape[0]
    assert got["vertexHash"] == _fnv1a(m.vertices.cpu().numpy().tobytes())
    assert got["indexHash"] == _fnv1a(m.indices.cpu().numpy().tobytes())
    assert got["leafMs"] > 0
    # weld check: PMB writes every cut edge's vertex once, so positions repeat
    # only where a voxel equals the isovalue (t = 0 on one edge, 1 on another)
    vb = m.vertices.cpu().numpy().view(np.uint32)
    uniq, inv = np.unique(vb, axis=0, return_inverse=True)
    t = inv.reshape(-1)[m.indices.cpu().numpy().astype(np.int64)]
    degenerate = int(((t[:, 0] == t[:, 1]) | (t[:, 1] == t[:, 2]) | (t[:, 0] == t[:, 2])).sum())
    assert got["uniqueVertices"] == len(uniq)
    assert got["degenerateTriangles"] == degenerate
    if not (a == np.asarray(iso, a.dtype)).any() or dtype == np.uint8:
        assert len(uniq) == V
    lines = obj.read_text().splitlines()
    vs = np.array([[float(x) for x in l.split()[1:]] for l in lines if l.startswith("v ")], np.float32)
    np.testing.assert_array_equal(vs.view(np.uint32), m.vertices.cpu().numpy().view(np.uint32))


def test_volume_load_streams_the_file(ctx, tmp_path):
    from meshtrex_b200 import _lib as L
    a = blob_volume((70, 64, 48), np.uint16, seed=2)
    raw = tmp_path / f"vol_{a.shape[2]}x{a.shape[1]}x{a.shape[0]}_uint16.raw"
    a.tofile(raw)
    v = L.Volume()
    assert L.lib().mtx_volume_load(ctx.handle, str(raw).encode(), C.byref(v)) == 0
    assert tuple(v.dims) == (48, 64, 70) and v.dtype == L.DTYPE_U16 and v.owned == 1
    back = np.empty(a.size, np.uint16)
    assert L.lib().mtx_read_buffer(ctx.handle, C.byref(v.data), 0, back.ctypes.data, back.nbytes) == 0
    np.testing.assert_array_equal(back.reshape(a.shape), a)
    L.lib().mtx_volume_free(ctx.handle, C.byref(v))

    short = tmp_path / "cut_48x64x71_uint16.raw"
    a.tofile(short)  # one slice short of its name
    assert L.lib().mtx_volume_load(ctx.handle, str(short).encode(), C.byref(v)) == 1
    assert L.lib().mtx_volume_load(ctx.handle, str(tmp_path / "x_1x1x1_uint8.raw").encode(), C.byref(v)) == 1


def test_volume_load_of_several_staging_chunks(ctx, tmp_path):
    from meshtrex_b200 import _lib as L
    a = np.random.default_rng(5).integers(0, 65536, size=(160, 512, 512), dtype=np.uint16)  # 80 MiB: two chunks
    raw = tmp_path / "big_512x512x160_uint16.raw"
    a.tofile(raw)
    v = L.Volume()
    assert L.lib().mtx_volume_load(ctx.handle, str(raw).encode(), C.byref(v)) == 0
    back = np.empty(a.size, np.uint16)
    assert L.lib().mtx_read_buffer(ctx.handle, C.byref(v.data), 0, back.ctypes.data, back.nbytes) == 0
    assert np.array_equal(back, a.reshape(-1))
    L.lib().mtx_volume_free(ctx.handle, C.byref(v))
