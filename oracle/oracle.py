"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (``mtx_oracle.c``) restates meshtrex's CPU path for the
isosurface-extraction hot path; see ``mtx_oracle.h`` for which reference lines
each function follows and what it is pinned against.  Only the tests,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
module, as the checker; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_HARNESS = os.path.join(HERE, "_ref", "ref_harness")

U8, U16, F32, F64 = 0, 1, 2, 3
FRAME_VOXEL, FRAME_NDC = 0, 1
_DTYPES = {np.dtype(np.uint8): U8, np.dtype(np.uint16): U16, np.dtype(np.float32): F32,
           np.dtype(np.float64): F64}


class _Vol(C.Structure):
    _fields_ = [("data", C.c_void_p), ("dims", C.c_uint32 * 3), ("dtype", C.c_int)]


class _Counts(C.Structure):
    _fields_ = [("n_vertices", C.c_uint64), ("n_triangles", C.c_uint64)]


_lib = None


def reference_src() -> str | None:
    """meshtrex's src directory: $REFERENCE_SRC, else a meshtrex checkout named
    "reference" beside this repository; None when neither holds testMinMax.h."""
    cand = os.environ.get("REFERENCE_SRC") or os.path.join(HERE, "..", "..", "reference", "src")
    cand = os.path.abspath(cand)
    return cand if os.path.isfile(os.path.join(cand, "testMinMax.h")) else None


def build() -> None:
    """Compile liboracle.so (and the reference harness when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    src = reference_src()
    if src:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE_SRC={src}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P, U32P, U64, F = C.c_void_p, C.POINTER(C.c_uint32), C.c_uint64, C.c_float
        L.orc_minmax_halo.argtypes = [C.POINTER(_Vol), U32P, P, C.c_int]
        L.orc_minmax_core.argtypes = [C.POINTER(_Vol), U32P, P]
        L.orc_mip_levels.argtypes = [U32P]
        L.orc_mip_levels.restype = C.c_int
        L.orc_mip_offset.argtypes = [U32P, C.c_int]
        L.orc_mip_offset.restype = C.c_uint64
        L.orc_mip_extent.argtypes = [U32P, C.c_int, U32P]
        L.orc_pyramid.argtypes = [P, U32P, P]
        L.orc_block_active.argtypes = [C.c_int, C.c_uint32, C.c_uint32, F]
        L.orc_block_active.restype = C.c_int
        L.orc_compact.argtypes = [P, U64, C.c_int, F, P]
        L.orc_compact.restype = C.c_uint32
        L.orc_cell_cases.argtypes = [C.POINTER(_Vol), U32P, F, P, C.c_uint32, P]
        L.orc_mc_extract.argtypes = [C.POINTER(_Vol), U32P, F, P, C.c_uint32, C.c_int, C.c_int,
                                     C.POINTER(_Counts), P, P, P, P, P, P]
        L.orc_mc_extract.restype = C.c_int
        L.orc_mc_adjoint.argtypes = [C.POINTER(_Vol), U32P, F, P, C.c_uint32, P, P, P]
        L.orc_mc_adjoint.restype = C.c_int
        L.orc_pipeline.argtypes = [C.POINTER(_Vol), U32P, F, C.c_int, C.POINTER(_Counts),
                                   U32P, P, P]
        L.orc_pipeline.restype = C.c_int
        L.orc_meshlets.argtypes = [P, C.c_uint32, P, C.c_uint32, C.c_uint32, P, P, P, C.POINTER(U64)]
        L.orc_meshlets.restype = U64
        L.orc_key_of_f32.argtypes = [F]
        L.orc_key_of_f32.restype = C.c_uint32
        L.orc_f32_of_key.argtypes = [C.c_uint32]
        L.orc_f32_of_key.restype = F
        _lib = L
    return _lib


def _vol(v: np.ndarray) -> _Vol:
    """Volume arrays are indexed [z, y, x] (x fastest in memory)."""
    assert v.flags.c_contiguous and v.ndim == 3
    d = _Vol()
    d.data = v.ctypes.data
    d.dims[0], d.dims[1], d.dims[2] = v.shape[2], v.shape[1], v.shape[0]
    d.dtype = _DTYPES[v.dtype]
    return d


def _u3(t):
    a = (C.c_uint32 * 3)(*[int(x) for x in t])
    return a


def block_grid(shape_zyx, block):
    """Block grid (gx, gy, gz) = ceil(dims / block) for a [z,y,x] volume shape."""
    X, Y, Z = shape_zyx[2], shape_zyx[1], shape_zyx[0]
    bx, by, bz = _block3(block)
    return ((X + bx - 1) // bx, (Y + by - 1) // by, (Z + bz - 1) // bz)


def _block3(block):
    return (block, block, block) if np.isscalar(block) else tuple(block)


def minmax_halo(v: np.ndarray, block, nthreads: int = 1) -> np.ndarray:
    """uint32 [nblocks, 2] keys over the (B+1)^3 overlapped blocks."""
    g = block_grid(v.shape, block)
    out = np.empty((g[0] * g[1] * g[2], 2), np.uint32)
    d = _vol(v)
    lib().orc_minmax_halo(C.byref(d), _u3(_block3(block)), out.ctypes.data, nthreads)
    return out


def minmax_core(v: np.ndarray, block) -> np.ndarray:
    g = block_grid(v.shape, block)
    out = np.empty((g[0] * g[1] * g[2], 2), np.uint32)
    d = _vol(v)
    lib().orc_minmax_core(C.byref(d), _u3(_block3(block)), out.ctypes.data)
    return out


def mip_levels(grid) -> int:
    return lib().orc_mip_levels(_u3(grid))


def mip_extent(grid, level):
    e = (C.c_uint32 * 3)()
    lib().orc_mip_extent(_u3(grid), level, e)
    return tuple(e)


def pyramid(leaf: np.ndarray, grid) -> np.ndarray:
    """All levels, concatenated, uint32 [texels, 2]."""
    L = mip_levels(grid)
    total = lib().orc_mip_offset(_u3(grid), L)
    out = np.empty((total, 2), np.uint32)
    leaf = np.ascontiguousarray(leaf, np.uint32)
    lib().orc_pyramid(leaf.ctypes.data, _u3(grid), out.ctypes.data)
    return out


def mip_offset(grid, level) -> int:
    return int(lib().orc_mip_offset(_u3(grid), level))


def compact(leaf: np.ndarray, dtype_code: int, iso: float) -> np.ndarray:
    leaf = np.ascontiguousarray(leaf, np.uint32)
    n = leaf.shape[0]
    ids = np.empty(max(n, 1), np.uint32)
    k = lib().orc_compact(leaf.ctypes.data, n, dtype_code, float(iso), ids.ctypes.data)
    return ids[:k].copy()


def block_active(dtype_code: int, kmin: int, kmax: int, iso: float) -> bool:
    return bool(lib().orc_block_active(dtype_code, kmin, kmax, float(iso)))


def dtype_code(v: np.ndarray) -> int:
    return _DTYPES[v.dtype]


def key_of_f32(f: float) -> int:
    return int(lib().orc_key_of_f32(float(f)))


def cell_cases(v: np.ndarray, block, iso: float, ids: np.ndarray) -> np.ndarray:
    b = _block3(block)
    ids = np.ascontiguousarray(ids, np.uint32)
    out = np.zeros((len(ids), b[0] * b[1] * b[2]), np.uint8)
    d = _vol(v)
    lib().orc_cell_cases(C.byref(d), _u3(b), float(iso), ids.ctypes.data, len(ids),
                         out.ctypes.data)
    return out


@dataclass
class Mesh:
    ids: np.ndarray            # active block ids, ascending
    nvert_per_block: np.ndarray
    ntri_per_block: np.ndarray
    xyz: np.ndarray | None     # float32 [V, 3]
    xyz64: np.ndarray | None   # float64 [V, 3]
    normals: np.ndarray | None  # float32 [V, 3]
    indices: np.ndarray | None  # uint32 [T, 3]

    @property
    def n_vertices(self):
        return int(self.nvert_per_block.sum())

    @property
    def n_triangles(self):
        return int(self.ntri_per_block.sum())


def mc_extract(v: np.ndarray, block, iso: float, ids: np.ndarray, frame: int = FRAME_VOXEL,
               nthreads: int = 1, want_xyz=True, want_xyz64=False, want_normals=False,
               want_indices=True) -> Mesh:
    b = _block3(block)
    ids = np.ascontiguousarray(ids, np.uint32)
    n = len(ids)
    d = _vol(v)
    cnt = _Counts()
    nv = np.zeros(max(n, 1), np.uint32)
    nt = np.zeros(max(n, 1), np.uint32)
    rc = lib().orc_mc_extract(C.byref(d), _u3(b), float(iso), ids.ctypes.data, n, frame, nthreads,
                              C.byref(cnt), nv.ctypes.data, nt.ctypes.data, None, None, None, None)
    if rc != 0:
        raise RuntimeError(f"oracle extract failed ({rc})")
    V, T = int(cnt.n_vertices), int(cnt.n_triangles)
    xyz = np.empty((V, 3), np.float32) if want_xyz else None
    xyz64 = np.empty((V, 3), np.float64) if want_xyz64 else None
    nrm = np.empty((V, 3), np.float32) if want_normals else None
    idx = np.empty((T, 3), np.uint32) if want_indices else None
    ptr = lambda a: a.ctypes.data if a is not None and a.size else None  # noqa: E731
    if any(a is not None for a in (xyz, xyz64, nrm, idx)) and (V or T):
        rc = lib().orc_mc_extract(C.byref(d), _u3(b), float(iso), ids.ctypes.data, n, frame,
                                  nthreads, C.byref(cnt), None, None, ptr(xyz), ptr(xyz64),
                                  ptr(nrm), ptr(idx))
        if rc != 0:
            raise RuntimeError(f"oracle extract failed ({rc})")
    return Mesh(ids, nv[:n], nt[:n], xyz, xyz64, nrm, idx)


def meshlets(ntri_per_block: np.ndarray, indices: np.ndarray, max_v: int = 64, max_p: int = 126):
    """(descriptors uint32 [M, 4], meshlet vertex ids [MV], indices into them [T, 3])."""
    nt = np.ascontiguousarray(ntri_per_block, np.uint32)
    idx = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    mv = C.c_uint64(0)
    m = lib().orc_meshlets(nt.ctypes.data, len(nt), idx.ctypes.data, max_v, max_p, None, None, None, C.byref(mv))
    desc = np.zeros((m, 4), np.uint32)
    mverts = np.zeros(mv.value, np.uint32)
    midx = np.zeros(idx.size, np.uint32)
    lib().orc_meshlets(nt.ctypes.data, len(nt), idx.ctypes.data, max_v, max_p, desc.ctypes.data,
                       mverts.ctypes.data, midx.ctypes.data, C.byref(mv))
    return desc, mverts, midx.reshape(-1, 3)


def mc_adjoint(v: np.ndarray, block, iso: float, ids: np.ndarray, dl_dxyz: np.ndarray):
    """(dL/dfield FP64 [z,y,x], dL/diso) for dL/dxyz given in the voxel frame."""
    b = _block3(block)
    ids = np.ascontiguousarray(ids, np.uint32)
    g = np.ascontiguousarray(dl_dxyz, np.float32)
    out = np.zeros(v.shape, np.float64)
    diso = C.c_double(0.0)
    d = _vol(v)
    lib().orc_mc_adjoint(C.byref(d), _u3(b), float(iso), ids.ctypes.data, len(ids),
                         g.ctypes.data if g.size else None, out.ctypes.data, C.byref(diso))
    return out, float(diso.value)


def pipeline(v: np.ndarray, block, iso: float, nthreads: int = 1, want_mesh=False):
    """Full plain path (min/max -> compaction -> extraction); counts, optionally the mesh."""
    d = _vol(v)
    cnt = _Counts()
    na = C.c_uint32(0)
    b = _block3(block)
    rc = lib().orc_pipeline(C.byref(d), _u3(b), float(iso), nthreads, C.byref(cnt), C.byref(na),
                            None, None)
    if rc != 0:
        raise RuntimeError(f"oracle pipeline failed ({rc})")
    if not want_mesh:
        return int(na.value), int(cnt.n_vertices), int(cnt.n_triangles)
    leaf = minmax_halo(v, block, nthreads)
    ids = compact(leaf, dtype_code(v), iso)
    return mc_extract(v, block, iso, ids, nthreads=nthreads)


def extract(v: np.ndarray, block, iso: float, frame: int = FRAME_VOXEL, nthreads: int = 1,
            **kw) -> Mesh:
    """Min/max (B+1 halo) -> compaction -> PMB marching cubes, all on the CPU."""
    leaf = minmax_halo(v, block, nthreads)
    ids = compact(leaf, dtype_code(v), iso)
    return mc_extract(v, block, iso, ids, frame=frame, nthreads=nthreads, **kw)


# --------------------------------------------------------------- reference
def have_reference_harness() -> bool:
    return os.path.exists(REF_HARNESS)


def ref_minmax_256_u8_b4(raw_path: str) -> np.ndarray:
    """meshtrex's own computeMinMaxFromFile (256^3 uint8, B=4) via the harness."""
    out = raw_path + ".ref_minmax.bin"
    subprocess.run([REF_HARNESS, "minmax", raw_path, out], check=True)
    r = np.fromfile(out, np.uint32).reshape(-1, 2)
    os.remove(out)
    return r


def ref_active_count(raw_path: str, iso: float) -> int:
    p = subprocess.run([REF_HARNESS, "count", raw_path, repr(float(iso))], check=True,
                       capture_output=True, text=True)
    return int(p.stdout.strip())


def ref_tables():
    """(triTable int32 [256,16], edgeTable int32 [256]) read from meshtrex's mc_tables.h."""
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "t.bin")
        subprocess.run([REF_HARNESS, "tables", out], check=True)
        a = np.fromfile(out, np.int32)
    return a[:4096].reshape(256, 16), a[4096:4352]


def decoded_tables():
    """This project's packed case table decoded to (triTable, edgeTable) form."""
    import re
    src = open(os.path.join(HERE, "..", "meshtrex_b200", "csrc", "mc_case_table.h")).read()
    body = src[src.index("MTX_MC_CASES[256]"):]
    words = [int(w, 16) for w in re.findall(r"0x([0-9a-fA-F]{16})ull", body)][:256]
    corners = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5),
               (2, 6), (3, 7)]
    tri = -np.ones((256, 16), np.int32)
    edge = np.zeros(256, np.int32)
    for c, w in enumerate(words):
        n = w & 0xF
        for k in range(3 * n):
            tri[c, k] = (w >> (4 + 4 * k)) & 0xF
        m = 0
        for e, (a, b) in enumerate(corners):
            m |= (((c >> a) ^ (c >> b)) & 1) << e
        edge[c] = m
    return tri, edge
