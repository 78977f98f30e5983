"""The C++ drop-in facade (include/meshtrex/*.h) and the host-only ingest and
export calls, without a GPU: the facade compiles against the library with a
program written like meshtrex's main, raw-volume names parse as loadVolume's
scheme does, and the OBJ writer writes what it is given with its weld check."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROGRAM = os.path.join(ROOT, "tests", "cpp", "drop_in_main.cpp")


def build_program(out_dir):
    """Compiles tests/cpp/drop_in_main.cpp against the facade and the library."""
    lib_dir = os.path.join(ROOT, "meshtrex_b200")
    exe = os.path.join(str(out_dir), "drop_in_main")
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), PROGRAM,
           "-L", lib_dir, "-lmeshtrex_b200", f"-Wl,-rpath,{lib_dir}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_facade_program_compiles_and_links(tmp_path):
    exe = build_program(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def test_facade_headers_compile_as_cpp17(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text('#include "meshtrex/meshtrex.hpp"\nint main() { return 0; }\n')
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I",
                        os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("name,dims,dtype", [
    ("aneurism_256x256x256_uint8.raw", (256, 256, 256), 0),
    ("/some/dir/bonsai_ct_64x48x32_uint16.raw", (64, 48, 32), 1),
    ("field_7x5x3_float32.raw", (7, 5, 3), 2),
    ("field_7x5x3_float.raw", (7, 5, 3), 2),
])
def test_volume_names_parse_like_load_volume(name, dims, dtype):
    from meshtrex_b200 import _lib as L
    d = (C.c_uint32 * 3)()
    t = C.c_uint32()
    assert L.lib().mtx_parse_volume_name(name.encode(), d, C.byref(t)) == 0
    assert tuple(d) == dims and t.value == dtype


@pytest.mark.parametrize("name,status", [
    ("vol_64x64x64_int32.raw", 2),    # a type this library does not read
    ("vol_64x64_uint8.raw", 1),       # not the scheme
    ("vol_64x64x64_uint8.bin", 1),
    ("vol_0x64x64_uint8.raw", 1),
])
def test_bad_volume_names_are_rejected(name, status):
    from meshtrex_b200 import _lib as L
    d = (C.c_uint32 * 3)()
    t = C.c_uint32()
    assert L.lib().mtx_parse_volume_name(name.encode(), d, C.byref(t)) == status


def _write(path, v, idx, stride):
    from meshtrex_b200 import _lib as L
    st = L.ObjStats()
    v = np.ascontiguousarray(v, np.float32)
    idx = np.ascontiguousarray(idx, np.uint32)
    rc = L.lib().mtx_write_obj(str(path).encode(), v.ctypes.data, v.shape[0], stride, idx.ctypes.data, idx.size,
                               C.byref(st))
    return rc, st


def test_obj_writer_format_and_weld_check(tmp_path):
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 0, 0], [0.1, 0.2, 0.30000001]], np.float32)
    idx = np.array([[0, 1, 2], [0, 3, 2], [1, 3, 4]], np.uint32)  # vertex 3 repeats vertex 1's position
    rc, st = _write(tmp_path / "m.obj", v, idx, 3)
    assert rc == 0
    assert (st.vertexCount, st.triangleCount, st.uniqueVertexCount, st.degenerateTriangleCount) == (5, 3, 4, 1)
    lines = (tmp_path / "m.obj").read_text().splitlines()
    vs = np.array([[float(x) for x in l.split()[1:]] for l in lines if l.startswith("v ")], np.float32)
    fs = np.array([[int(x) for x in l.split()[1:]] for l in lines if l.startswith("f ")])
    np.testing.assert_array_equal(vs.view(np.uint32), v.view(np.uint32))  # 9 digits read back to the same bits
    np.testing.assert_array_equal(fs, idx + 1)


def test_obj_writer_vertex_data_layout(tmp_path):
    v = np.zeros((3, 8), np.float32)
    v[:, :3] = [[0, 0, 0], [1, 0, 0], [0, 1, 0]]
    v[:, 3] = 1
    v[:, 4:7] = [[0, 0, 1]] * 3
    rc, st = _write(tmp_path / "d.obj", v, np.array([0, 1, 2]), 8)
    assert rc == 0 and st.uniqueVertexCount == 3
    text = (tmp_path / "d.obj").read_text()
    assert text.count("\nvn ") == 3 and "f 1//1 2//2 3//3" in text


def test_obj_writer_rejects_bad_input(tmp_path):
    rc, _ = _write(tmp_path / "x.obj", np.zeros((2, 3)), np.array([0, 1, 2]), 3)  # index out of range
    assert rc == 1
    rc, _ = _write(tmp_path / "x.obj", np.zeros((3, 3)), np.array([0, 1]), 3)  # not whole triangles
    assert rc == 1
