"""ctypes binding of libmeshtrex_b200.so (declarations mirror include/meshtrex/mtx.h).

There is no fallback: importing this module raises if the CUDA library has
not been built (``python -c "import __graft_entry__ as g; g.build()"`` or
``make -C meshtrex_b200/csrc``).
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# MESHTREX_B200_LIB selects another build of the library, such as the
# bounds-check build libmeshtrex_b200_check.so (`make -C meshtrex_b200/csrc check`).
LIB_PATH = os.environ.get("MESHTREX_B200_LIB") or os.path.join(HERE, "libmeshtrex_b200.so")

MTX_OK = 0
STATUS = {0: "MTX_OK", 1: "MTX_ERR_INVALID_ARG", 2: "MTX_ERR_UNSUPPORTED", 3: "MTX_ERR_OOM",
          4: "MTX_ERR_CAPACITY", 5: "MTX_ERR_TIMEOUT", 6: "MTX_ERR_CUDA", 7: "MTX_ERR_NO_DEVICE",
          8: "MTX_ERR_INTERNAL"}
DTYPE_U8, DTYPE_U16, DTYPE_F32 = 0, 1, 2
VERTEX_XYZ, VERTEX_DATA = 0, 1
FRAME_VOXEL, FRAME_NDC = 0, 1
STAGING_AUTO, STAGING_TMA, STAGING_LDG = 0, 1, 2
ADJOINT_ATOMIC, ADJOINT_DETERMINISTIC = 0, 1
MAX_MIP_LEVELS = 32


class MtxError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        name = STATUS.get(status, f"status {status}")
        super().__init__(f"{where}: {name}" + (f" ({detail})" if detail else ""))


class Buffer(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("size", C.c_uint64)]


class PushConstants(C.Structure):
    _fields_ = [("volumeDim", C.c_uint32 * 4), ("blockDim", C.c_uint32 * 4),
                ("blockGridDim", C.c_uint32 * 4), ("isovalue", C.c_float), ("_pad", C.c_uint32 * 3)]


class Volume(C.Structure):
    _fields_ = [("data", Buffer), ("dims", C.c_uint32 * 3), ("dtype", C.c_uint32),
                ("owned", C.c_uint32), ("_pad", C.c_uint32)]


class MinMaxOutput(C.Structure):
    _fields_ = [("volumeImage", Volume), ("minMaxImage", Buffer), ("mipLevels", C.c_uint32),
                ("blockDim", C.c_uint32 * 3), ("blockGridDim", C.c_uint32 * 3),
                ("levelExtent", (C.c_uint32 * 3) * MAX_MIP_LEVELS),
                ("levelOffset", C.c_uint64 * MAX_MIP_LEVELS)]


class FilteringOutput(C.Structure):
    _fields_ = [("compactedBlockIdBuffer", Buffer), ("activeBlockCountBuffer", Buffer),
                ("blockRankBuffer", Buffer), ("activeBlockCount", C.c_uint32),
                ("totalBlocks", C.c_uint32), ("isovalue", C.c_float), ("_pad", C.c_uint32)]


class ExtractOptions(C.Structure):
    _fields_ = [("vertexFormat", C.c_uint32), ("frame", C.c_uint32), ("normals", C.c_uint32),
                ("staging", C.c_uint32), ("threads", C.c_uint32), ("_pad", C.c_uint32),
                ("cellCases", C.c_void_p)]


class MeshletDescriptor(C.Structure):
    _fields_ = [("vertexOffset", C.c_uint32), ("indexOffset", C.c_uint32),
                ("vertexCount", C.c_uint32), ("primitiveCount", C.c_uint32)]


class ExtractionOutput(C.Structure):
    _fields_ = [("vertexBuffer", Buffer), ("vertexCountBuffer", Buffer), ("indexBuffer", Buffer),
                ("indexCountBuffer", Buffer), ("meshletDescriptorBuffer", Buffer),
                ("meshletDescriptorCountBuffer", Buffer), ("meshletCount", C.c_uint32),
                ("vertexCount", C.c_uint32), ("indexCount", C.c_uint32),
                ("vertexStride", C.c_uint32)]


class Tuning(C.Structure):
    _fields_ = [("minmaxZChunk", C.c_uint32), ("minmaxSlices", C.c_uint32),
                ("extractWarps", C.c_uint32), ("staging", C.c_uint32), ("extractCtasPerSm", C.c_uint32)]


class BatchAutotuneResult(C.Structure):
    _fields_ = [("blockWarps", C.c_uint32), ("fromCache", C.c_uint32), ("candidates", C.c_uint32),
                ("_pad", C.c_uint32), ("ms", C.c_double)]


class MeshBuffers(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("vertexCapacity", C.c_uint64),
                ("indices", C.c_void_p), ("triangleCapacity", C.c_uint64),
                ("meshlets", C.c_void_p), ("meshletCapacity", C.c_uint64),
                ("counters", C.c_void_p), ("maxActiveBlocks", C.c_uint64)]


class MeshletOutput(C.Structure):
    _fields_ = [("meshletDescriptorBuffer", Buffer), ("meshletVertexBuffer", Buffer), ("vertexBuffer", Buffer),
                ("indexBuffer", Buffer), ("meshletCount", C.c_uint32), ("vertexCount", C.c_uint32),
                ("indexCount", C.c_uint32), ("vertexStride", C.c_uint32)]


class BatchJob(C.Structure):
    _fields_ = [("volume", C.c_uint32), ("isovalue", C.c_float)]


class BatchDesc(C.Structure):
    _fields_ = [("volumeCount", C.c_uint32), ("jobCount", C.c_uint32),
                ("volumes", C.POINTER(Volume)), ("blockEdges", C.POINTER(C.c_uint32)),
                ("jobs", C.POINTER(BatchJob)), ("maxActiveBlocks", C.c_uint64),
                ("vertexCapacity", C.c_uint64), ("triangleCapacity", C.c_uint64),
                ("vertexFormat", C.c_uint32), ("frame", C.c_uint32), ("normals", C.c_uint32),
                ("useGraph", C.c_uint32), ("blockWarps", C.c_uint32)]


class BatchJobResult(C.Structure):
    _fields_ = [("meshletOffset", C.c_uint32), ("meshletCount", C.c_uint32),
                ("vertexCount", C.c_uint32), ("indexCount", C.c_uint32),
                ("vertexOffset", C.c_uint64), ("indexOffset", C.c_uint64)]


class BatchTotals(C.Structure):
    _fields_ = [("status", C.c_int32), ("activeBlocks", C.c_uint32),
                ("vertexCount", C.c_uint64), ("triangleCount", C.c_uint64)]


class BatchOutputs(C.Structure):
    _fields_ = [("vertexBuffer", Buffer), ("indexBuffer", Buffer), ("meshletDescriptorBuffer", Buffer),
                ("jobResultBuffer", Buffer), ("vertexStride", C.c_uint32), ("_pad", C.c_uint32)]


class AutotuneResult(C.Structure):
    _fields_ = [("blockEdge", C.c_uint32), ("tuning", Tuning), ("ms", C.c_double),
                ("fromCache", C.c_uint32), ("candidates", C.c_uint32)]


AUTOTUNE_IGNORE_CACHE, AUTOTUNE_QUICK = 1, 2


class ObjStats(C.Structure):
    _fields_ = [("vertexCount", C.c_uint32), ("triangleCount", C.c_uint32),
                ("uniqueVertexCount", C.c_uint32), ("degenerateTriangleCount", C.c_uint32)]


# (name, restype, argtypes) of every exported entry point
_P = C.c_void_p
_ST = C.c_int
SIGNATURES = [
    ("mtx_status_string", C.c_char_p, [_ST]),
    ("mtx_abi_version", C.c_uint32, []),
    ("mtx_context_create", _ST, [C.c_int, _P, C.POINTER(_P)]),
    ("mtx_context_destroy", _ST, [_P]),
    ("mtx_context_set_stream", _ST, [_P, _P]),
    ("mtx_context_set_extract_stream", _ST, [_P, _P]),
    ("mtx_context_last_error", C.c_char_p, [_P]),
    ("mtx_synchronize", _ST, [_P]),
    ("mtx_debug_fail_allocation", _ST, [_P, C.c_uint32]),
    ("mtx_debug_set_waits", _ST, [_P, C.c_uint32, C.c_uint32]),
    ("mtx_volume_upload", _ST, [_P, _P, C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(Volume)]),
    ("mtx_volume_wrap", _ST, [_P, C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(Volume)]),
    ("mtx_volume_free", _ST, [_P, C.POINTER(Volume)]),
    ("mtx_parse_volume_name", _ST, [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    ("mtx_volume_load", _ST, [_P, C.c_char_p, C.POINTER(Volume)]),
    ("mtx_read_buffer", _ST, [_P, C.POINTER(Buffer), C.c_uint64, _P, C.c_uint64]),
    ("mtx_write_obj", _ST, [C.c_char_p, _P, C.c_uint32, C.c_uint32, _P, C.c_uint32, C.POINTER(ObjStats)]),
    ("mtx_push_constants_init", _ST, [C.POINTER(C.c_uint32), C.c_uint32, C.c_float,
                                      C.POINTER(PushConstants)]),
    ("mtx_key_to_float", C.c_float, [C.c_uint32, C.c_uint32]),
    ("mtx_compute_min_max_mip", _ST, [_P, C.POINTER(Volume), C.POINTER(PushConstants), _P,
                                      C.POINTER(MinMaxOutput)]),
    ("mtx_upload_compute_min_max_mip", _ST, [_P, _P, C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(PushConstants),
                                             _P, C.POINTER(Volume), C.POINTER(MinMaxOutput)]),
    ("mtx_minmax_free", _ST, [_P, C.POINTER(MinMaxOutput)]),
    ("mtx_filter_active_blocks", _ST, [_P, C.POINTER(MinMaxOutput), C.POINTER(PushConstants), _P,
                                       C.POINTER(FilteringOutput)]),
    ("mtx_read_active_block_count", _ST, [_P, C.POINTER(FilteringOutput)]),
    ("mtx_filtering_free", _ST, [_P, C.POINTER(FilteringOutput)]),
    ("mtx_filter_active_blocks_noalloc", _ST, [_P, C.c_uint64, C.c_uint32, C.c_float, _P, _P, _P, _P, _P]),
    ("mtx_extract_meshlet_descriptors", _ST, [_P, C.POINTER(MinMaxOutput),
                                              C.POINTER(FilteringOutput),
                                              C.POINTER(PushConstants), C.POINTER(ExtractOptions),
                                              _P, C.POINTER(ExtractionOutput)]),
    ("mtx_extraction_free", _ST, [_P, C.POINTER(ExtractionOutput)]),
    ("mtx_build_meshlets", _ST, [_P, C.POINTER(ExtractionOutput), C.c_uint32, C.c_uint32, C.POINTER(MeshletOutput)]),
    ("mtx_meshlet_output_free", _ST, [_P, C.POINTER(MeshletOutput)]),
    ("mtx_extract_plain_async", _ST, [_P, C.POINTER(Volume), C.POINTER(PushConstants),
                                      C.POINTER(ExtractOptions), C.POINTER(MeshBuffers)]),
    ("mtx_extract_backward", _ST, [_P, C.POINTER(Volume), C.POINTER(PushConstants), C.POINTER(FilteringOutput),
                                   _P, C.c_uint32, _P, C.c_uint32, C.c_uint32, _P, _P, C.c_uint32]),
    ("mtx_batch_create", _ST, [_P, C.POINTER(BatchDesc), C.POINTER(_P)]),
    ("mtx_batch_run", _ST, [_P]),
    ("mtx_batch_get_outputs", _ST, [_P, C.POINTER(BatchOutputs)]),
    ("mtx_batch_read_results", _ST, [_P, _P, C.POINTER(BatchTotals)]),
    ("mtx_batch_destroy", _ST, [_P]),
    ("mtx_profiler_create", _ST, [_P, C.POINTER(_P)]),
    ("mtx_context_set_profiler", _ST, [_P, _P]),
    ("mtx_context_set_tuning", _ST, [_P, C.POINTER(Tuning)]),
    ("mtx_context_get_tuning", _ST, [_P, C.POINTER(Tuning)]),
    ("mtx_autotune", _ST, [_P, C.POINTER(Volume), C.c_float, C.c_char_p, C.c_uint32, C.POINTER(AutotuneResult)]),
    ("mtx_autotune_batch", _ST, [_P, C.POINTER(BatchDesc), C.c_char_p, C.c_uint32, C.POINTER(C.c_uint32),
                                 C.POINTER(BatchAutotuneResult)]),
    ("mtx_profiler_destroy", _ST, [_P]),
    ("mtx_profiler_begin_frame", _ST, [_P]),
    ("mtx_profiler_end_frame", _ST, [_P]),
    ("mtx_profiler_region_count", C.c_uint32, [_P]),
    ("mtx_profiler_region", _ST, [_P, C.c_uint32, C.c_char_p, C.POINTER(C.c_double),
                                  C.POINTER(C.c_double), C.POINTER(C.c_uint32)]),
    ("mtx_profiler_export_csv", _ST, [_P, C.c_char_p]),
]

_lib = None


def lib():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C meshtrex_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str, ctx=None) -> None:
    if status != MTX_OK:
        detail = ""
        if ctx:
            msg = lib().mtx_context_last_error(ctx)
            detail = msg.decode() if msg else ""
        raise MtxError(status, where, detail)
