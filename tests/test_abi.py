"""The C ABI library without a GPU: it loads, exports every declared entry
point, and its host-only calls behave."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "meshtrex", "mtx.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mtx_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_entry_point():
    from meshtrex_b200 import _lib as L
    lib = L.lib()
    names = declared()
    assert len(names) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mtx_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    bound = {n for n, _, _ in L.SIGNATURES}
    assert set(names) == bound, (set(names) - bound, bound - set(names))
    for n in names:
        getattr(lib, n)


def test_status_strings_and_version():
    from meshtrex_b200 import _lib as L
    for code, name in L.STATUS.items():
        assert L.lib().mtx_status_string(code).decode() == name
    assert L.lib().mtx_abi_version() == 1


def test_push_constants_follow_meshtrex():
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    assert C.sizeof(L.PushConstants) == 64  # alignas(16) struct of 3 uvec4 + float (common.h:29-34)
    pc = api.push_constants((1024, 1024, 314), 3, 80.0)  # meshtrex.cpp:56-84
    assert list(pc.blockGridDim)[:3] == [342, 342, 105]
    assert pc.isovalue == 80.0 and list(pc.blockDim)[:3] == [3, 3, 3]


def test_key_decoding_matches_oracle(oracle):
    from meshtrex_b200 import _lib as L
    for f in (-3.5, -0.0, 0.0, 1e-30, 7.25, 3.0e38):
        k = oracle.key_of_f32(f)
        assert L.lib().mtx_key_to_float(L.DTYPE_F32, k) == C.c_float(f).value
    assert L.lib().mtx_key_to_float(L.DTYPE_U16, 65535) == 65535.0


def test_host_side_argument_checks():
    from meshtrex_b200 import _lib as L
    lib = L.lib()
    assert lib.mtx_context_create(0, None, None) == 1
    assert lib.mtx_push_constants_init(None, 8, 1.0, None) == 1


def test_no_device_is_reported():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from meshtrex_b200 import _lib as L
    h = C.c_void_p()
    assert L.lib().mtx_context_create(0, None, C.byref(h)) == 7  # MTX_ERR_NO_DEVICE


def test_tensor_map_plan_alignment():
    """Every TMA tile plan keeps 16-byte aligned x coordinates and rows."""
    for esz in (1, 2, 4):
        A = 16 // esz
        for B in range(2, 17):
            g = 1
            for d in range(1, A + 1):
                if B % d == 0 and A % d == 0:
                    g = d
            xoff_max = 0 if B % A == 0 else A - g
            PX = -(-(xoff_max + B + 1) // A) * A
            assert (PX * esz) % 16 == 0 and PX <= 256
            for bx in range(64):
                ox = bx * B
                assert ox % A <= xoff_max and ox % A + B + 1 <= PX


def test_noalloc_compaction_rejects_bad_pointers_before_any_work():
    """mtx_filter_active_blocks_noalloc checks its arguments before it touches
    the GPU: the status record is required, and the keys and the rank map are
    read and written as 16-byte words, so they must be 16-byte aligned.  The
    pointers below are never dereferenced."""
    from meshtrex_b200 import _lib as L
    f = L.lib().mtx_filter_active_blocks_noalloc
    ok = C.c_void_p(0x10000)
    off8 = C.c_void_p(0x10008)
    assert f(ok, 16, L.DTYPE_U8, 1.0, ok, ok, ok, None, None) == 1      # no status record
    assert f(off8, 16, L.DTYPE_U8, 1.0, ok, ok, ok, ok, None) == 1      # keys not 16-byte aligned
    assert f(ok, 16, L.DTYPE_U8, 1.0, ok, off8, ok, ok, None) == 1      # rank map not 16-byte aligned
    assert f(ok, 16, 3, 1.0, ok, ok, ok, ok, None) == 1                 # unknown dtype
    assert f(ok, 0, L.DTYPE_U8, 1.0, ok, ok, ok, ok, None) == 1         # no blocks
    assert f(ok, 65536 * 1024 + 1, L.DTYPE_U8, 1.0, ok, ok, ok, ok, None) == 4  # beyond the array
