"""Python front end of the C ABI, mirroring meshtrex's stage managers.

  compute_min_max_mip        src/minMaxManager.h:20-21
  filter_active_blocks       src/filteringManager.h:9-10
  read_active_block_count    src/filteringManager.h:13
  extract_meshlet_descriptors src/extractionManager.h:10-11

Torch is used only for device memory and streams: volumes are CUDA tensors
indexed [z, y, x] and outputs are handed back as views or copies of the
library's device buffers.  All work runs in libmeshtrex_b200.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L

_DT = {torch.uint8: L.DTYPE_U8, torch.uint16: L.DTYPE_U16, torch.float32: L.DTYPE_F32}
_NP = {np.dtype(np.uint8): L.DTYPE_U8, np.dtype(np.uint16): L.DTYPE_U16,
       np.dtype(np.float32): L.DTYPE_F32}


class _Dev:
    """Wraps a device pointer so torch can view it without copying."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr or 0), False), "version": 3,
                                         "strides": None}


def device_view(ptr: int, shape, dtype: torch.dtype) -> torch.Tensor:
    typestr = {torch.uint8: "|u1", torch.uint16: "<u2", torch.uint32: "<u4",
               torch.float32: "<f4", torch.int32: "<i4"}[dtype]
    n = int(np.prod(shape))
    if n == 0 or not ptr:
        return torch.empty(shape, dtype=dtype, device="cuda")
    return torch.as_tensor(_Dev(ptr, shape, typestr), device="cuda")


def _stream_ptr(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


class Context:
    """VulkanContext's compute role: device, stream, scratch arena."""

    def __init__(self, device: int = 0, stream=None):
        self.handle = C.c_void_p()
        self.stream_ptr = _stream_ptr(stream)
        L.check(L.lib().mtx_context_create(device, C.c_void_p(self.stream_ptr),
                                           C.byref(self.handle)), "mtx_context_create")

    def set_stream(self, stream=None):
        self.stream_ptr = _stream_ptr(stream)
        L.check(L.lib().mtx_context_set_stream(self.handle, C.c_void_p(self.stream_ptr)),
                "mtx_context_set_stream", self.handle)

    def fence(self):
        """Orders the context's stream after torch's current stream.  The
        library frees in the order of its own stream, so work queued on the
        current stream that reads a library buffer (the copies the accessors
        below make) must come first; the *.free() methods call this."""
        cur = torch.cuda.current_stream()
        if int(cur.cuda_stream) != self.stream_ptr:
            ev = torch.cuda.Event()
            ev.record(cur)
            torch.cuda.ExternalStream(self.stream_ptr).wait_event(ev)

    def synchronize(self):
        L.check(L.lib().mtx_synchronize(self.handle), "mtx_synchronize", self.handle)

    def set_profiler(self, prof):
        L.check(L.lib().mtx_context_set_profiler(self.handle, prof.handle if prof else None),
                "mtx_context_set_profiler")

    def set_extract_stream(self, stream=None):
        """Count, scan and emit of AsyncExtractor.run on `stream` (None: the
        context's own stream), so that the next work on the context's stream
        overlaps them (mtx_context_set_extract_stream)."""
        ptr = int(stream.cuda_stream) if stream is not None else 0
        L.check(L.lib().mtx_context_set_extract_stream(self.handle, C.c_void_p(ptr)),
                "mtx_context_set_extract_stream", self.handle)

    def set_tuning(self, minmax_zchunk=0, minmax_slices=0, extract_warps=0, staging=0, extract_ctas_per_sm=0):
        t = L.Tuning(minmax_zchunk, minmax_slices, extract_warps, staging, extract_ctas_per_sm)
        L.check(L.lib().mtx_context_set_tuning(self.handle, C.byref(t)), "mtx_context_set_tuning",
                self.handle)

    def get_tuning(self) -> dict:
        t = L.Tuning()
        L.check(L.lib().mtx_context_get_tuning(self.handle, C.byref(t)), "mtx_context_get_tuning")
        return {f: getattr(t, f) for f, _ in L.Tuning._fields_}

    def set_waits(self, max_polls: int = 0, withhold: int = 0):
        """Failure injection of the bounded waits (mtx_debug_set_waits)."""
        L.check(L.lib().mtx_debug_set_waits(self.handle, max_polls, withhold), "mtx_debug_set_waits")

    def fail_allocation(self, k: int):
        L.check(L.lib().mtx_debug_fail_allocation(self.handle, k), "mtx_debug_fail_allocation")

    def close(self):
        if self.handle:
            L.lib().mtx_context_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def push_constants(dims_xyz, block: int, iso: float) -> L.PushConstants:
    pc = L.PushConstants()
    d = (C.c_uint32 * 3)(*[int(x) for x in dims_xyz])
    L.check(L.lib().mtx_push_constants_init(d, int(block), float(iso), C.byref(pc)),
            "mtx_push_constants_init")
    return pc


def wrap_volume(t: torch.Tensor) -> L.Volume:
    """Describe a contiguous CUDA tensor [z, y, x] as a volume (no copy)."""
    assert t.is_cuda and t.is_contiguous() and t.dim() == 3, "volume must be a contiguous CUDA [z,y,x] tensor"
    v = L.Volume()
    d = (C.c_uint32 * 3)(t.shape[2], t.shape[1], t.shape[0])
    L.check(L.lib().mtx_volume_wrap(C.c_void_p(t.data_ptr()), d, _DT[t.dtype], C.byref(v)),
            "mtx_volume_wrap")
    return v


def upload_volume(ctx: Context, a: np.ndarray) -> L.Volume:
    """Host array [z, y, x] -> new device volume (meshtrex's staging upload)."""
    a = np.ascontiguousarray(a)
    v = L.Volume()
    d = (C.c_uint32 * 3)(a.shape[2], a.shape[1], a.shape[0])
    L.check(L.lib().mtx_volume_upload(ctx.handle, C.c_void_p(a.ctypes.data), d, _NP[a.dtype],
                                      C.byref(v)), "mtx_volume_upload", ctx.handle)
    return v


def free_volume(ctx: Context, v: L.Volume):
    ctx.fence()
    L.lib().mtx_volume_free(ctx.handle, C.byref(v))


@dataclass
class MinMax:
    ctx: Context
    out: L.MinMaxOutput

    @property
    def levels(self) -> int:
        return int(self.out.mipLevels)

    def level(self, l: int) -> torch.Tensor:
        """uint32 [gz, gy, gx, 2] {min,max} keys of mip level l (a copy)."""
        e = self.out.levelExtent[l]
        base = self.out.minMaxImage.ptr + 8 * int(self.out.levelOffset[l])
        return device_view(base, (e[2], e[1], e[0], 2), torch.int32).clone().view(torch.int32)

    def all_levels(self) -> torch.Tensor:
        n = self.out.minMaxImage.size // 8
        return device_view(self.out.minMaxImage.ptr, (n, 2), torch.int32).clone()

    def free(self):
        if self.out.minMaxImage.ptr:
            self.ctx.fence()
            L.lib().mtx_minmax_free(self.ctx.handle, C.byref(self.out))


@dataclass
class Filtering:
    ctx: Context
    out: L.FilteringOutput

    @property
    def active_block_count(self) -> int:
        return int(self.out.activeBlockCount)

    def ids(self) -> torch.Tensor:
        n = self.out.activeBlockCount
        return device_view(self.out.compactedBlockIdBuffer.ptr, (n,), torch.int32).clone()

    def device_count(self) -> int:
        return int(device_view(self.out.activeBlockCountBuffer.ptr, (1,), torch.int32).item())

    def free(self):
        if self.out.compactedBlockIdBuffer.ptr:
            self.ctx.fence()
            L.lib().mtx_filtering_free(self.ctx.handle, C.byref(self.out))


@dataclass
class Extraction:
    ctx: Context
    out: L.ExtractionOutput

    @property
    def vertex_count(self):
        return int(self.out.vertexCount)

    @property
    def index_count(self):
        return int(self.out.indexCount)

    @property
    def meshlet_count(self):
        return int(self.out.meshletCount)

    def vertices(self) -> torch.Tensor:
        """float32 [V, 3] (xyz format) or [V, 8] (VertexData)."""
        w = self.out.vertexStride // 4
        return device_view(self.out.vertexBuffer.ptr, (self.out.vertexCount, w), torch.float32).clone()

    def indices(self) -> torch.Tensor:
        return device_view(self.out.indexBuffer.ptr, (self.out.indexCount // 3, 3), torch.int32).clone()

    def meshlets(self) -> torch.Tensor:
        return device_view(self.out.meshletDescriptorBuffer.ptr, (self.out.meshletCount, 4),
                           torch.int32).clone()

    def counters(self) -> torch.Tensor:
        return device_view(self.out.vertexCountBuffer.ptr, (3,), torch.int32).clone()

    def free(self):
        if self.out.vertexCountBuffer.ptr or self.out.meshletDescriptorBuffer.ptr:
            self.ctx.fence()
            L.lib().mtx_extraction_free(self.ctx.handle, C.byref(self.out))


class Profiler:
    """GPUProfiler analogue: per-stage CUDA-event times under meshtrex's stage names."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.handle = C.c_void_p()
        L.check(L.lib().mtx_profiler_create(ctx.handle, C.byref(self.handle)), "mtx_profiler_create")

    def begin_frame(self):
        L.lib().mtx_profiler_begin_frame(self.handle)

    def end_frame(self):
        L.check(L.lib().mtx_profiler_end_frame(self.handle), "mtx_profiler_end_frame")

    def regions(self):
        out = {}
        for i in range(L.lib().mtx_profiler_region_count(self.handle)):
            name = C.create_string_buffer(64)
            last, avg, fr = C.c_double(), C.c_double(), C.c_uint32()
            L.lib().mtx_profiler_region(self.handle, i, name, C.byref(last), C.byref(avg), C.byref(fr))
            out[name.value.decode()] = (last.value, avg.value, fr.value)
        return out

    def export_csv(self, path: str):
        L.check(L.lib().mtx_profiler_export_csv(self.handle, path.encode()), "mtx_profiler_export_csv")

    def close(self):
        if self.handle:
            L.lib().mtx_profiler_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _prof(p):
    return p.handle if p is not None else None


def compute_min_max_mip(ctx: Context, volume: L.Volume, pc: L.PushConstants, profiler=None) -> MinMax:
    out = L.MinMaxOutput()
    L.check(L.lib().mtx_compute_min_max_mip(ctx.handle, C.byref(volume), C.byref(pc), _prof(profiler),
                                            C.byref(out)), "computeMinMaxMip", ctx.handle)
    return MinMax(ctx, out)


def upload_compute_min_max_mip(ctx: Context, host: np.ndarray, pc: L.PushConstants, profiler=None):
    """mtx_upload_compute_min_max_mip: a host array [z, y, x] (pinned for the
    copies to overlap) uploaded in z-slabs with the leaf min/max of each slab
    running as it lands.  Returns (device volume, MinMax); the volume is owned:
    release it with free_volume.  `host` must stay alive and unchanged until the
    context's stream has done the work."""
    a = host
    assert a.flags.c_contiguous and a.ndim == 3
    v = L.Volume()
    out = L.MinMaxOutput()
    d = (C.c_uint32 * 3)(a.shape[2], a.shape[1], a.shape[0])
    L.check(L.lib().mtx_upload_compute_min_max_mip(ctx.handle, C.c_void_p(a.ctypes.data), d, _NP[a.dtype],
                                                   C.byref(pc), _prof(profiler), C.byref(v), C.byref(out)),
            "mtx_upload_compute_min_max_mip", ctx.handle)
    return v, MinMax(ctx, out)


def filter_active_blocks(ctx: Context, mm: MinMax, pc: L.PushConstants, profiler=None) -> Filtering:
    out = L.FilteringOutput()
    L.check(L.lib().mtx_filter_active_blocks(ctx.handle, C.byref(mm.out), C.byref(pc),
                                             _prof(profiler), C.byref(out)),
            "filterActiveBlocks", ctx.handle)
    return Filtering(ctx, out)


def read_active_block_count(ctx: Context, f: Filtering) -> int:
    L.check(L.lib().mtx_read_active_block_count(ctx.handle, C.byref(f.out)), "readActiveBlockCount",
            ctx.handle)
    return f.active_block_count


def extract_options(vertex_format=L.VERTEX_XYZ, frame=L.FRAME_VOXEL, normals=False,
                    staging=L.STAGING_AUTO, threads=0, cell_cases: torch.Tensor | None = None):
    o = L.ExtractOptions()
    o.vertexFormat, o.frame, o.normals = vertex_format, frame, int(bool(normals))
    o.staging, o.threads = staging, threads
    o.cellCases = cell_cases.data_ptr() if cell_cases is not None else None
    return o


def extract_meshlet_descriptors(ctx: Context, mm: MinMax, f: Filtering, pc: L.PushConstants,
                                options: L.ExtractOptions | None = None, profiler=None) -> Extraction:
    out = L.ExtractionOutput()
    opts = options if options is not None else extract_options()
    L.check(L.lib().mtx_extract_meshlet_descriptors(ctx.handle, C.byref(mm.out), C.byref(f.out),
                                                    C.byref(pc), C.byref(opts), _prof(profiler),
                                                    C.byref(out)),
            "extractMeshletDescriptors", ctx.handle)
    return Extraction(ctx, out)


def extract_backward(ctx: Context, volume: L.Volume, pc: L.PushConstants, f: Filtering, meshlets_ptr: int,
                     vertex_count: int, dl_dvertex: torch.Tensor, frame=L.FRAME_VOXEL,
                     mode=L.ADJOINT_ATOMIC):
    """mtx_extract_backward: dL/dvertex (float32 [V, 3] or [V, 8], the forward's
    frame) -> (dL/dfield as a float32 [z, y, x] tensor, dL/diso as a float32 [1])."""
    X, Y, Z = volume.dims[0], volume.dims[1], volume.dims[2]
    dfield = torch.empty((Z, Y, X), dtype=torch.float32, device="cuda")
    diso = torch.empty(1, dtype=torch.float32, device="cuda")
    g = dl_dvertex.contiguous()
    L.check(L.lib().mtx_extract_backward(ctx.handle, C.byref(volume), C.byref(pc), C.byref(f.out),
                                         C.c_void_p(meshlets_ptr or 0), int(vertex_count),
                                         C.c_void_p(g.data_ptr() if g.numel() else 0), int(g.shape[1]),
                                         int(frame), C.c_void_p(dfield.data_ptr()), C.c_void_p(diso.data_ptr()),
                                         int(mode)),
            "mtx_extract_backward", ctx.handle)
    return dfield, diso


@dataclass
class Meshlets:
    descriptors: torch.Tensor      # int32 [M, 4] {vertexOffset, indexOffset, vertexCount, primitiveCount}
    vertex_ids: torch.Tensor       # int32 [MV]: mesh vertex id of each meshlet vertex
    vertices: torch.Tensor         # float32 [MV, 3|8]: the mesh's vertex records in meshlet order
    indices: torch.Tensor          # int32 [T, 3]: ids into vertices


def build_meshlets(ctx: Context, x: Extraction, max_vertices: int = 64, max_primitives: int = 126) -> Meshlets:
    """mtx_build_meshlets on a drop-in extraction; copies the results out."""
    o = L.MeshletOutput()
    L.check(L.lib().mtx_build_meshlets(ctx.handle, C.byref(x.out), max_vertices, max_primitives, C.byref(o)),
            "mtx_build_meshlets", ctx.handle)
    w = max(o.vertexStride // 4, 1)
    m = Meshlets(device_view(o.meshletDescriptorBuffer.ptr, (o.meshletCount, 4), torch.int32).clone(),
                 device_view(o.meshletVertexBuffer.ptr, (o.vertexCount,), torch.int32).clone(),
                 device_view(o.vertexBuffer.ptr, (o.vertexCount, w), torch.float32).clone(),
                 device_view(o.indexBuffer.ptr, (o.indexCount // 3, 3), torch.int32).clone())
    ctx.fence()
    L.lib().mtx_meshlet_output_free(ctx.handle, C.byref(o))
    return m


@dataclass
class Mesh:
    vertices: torch.Tensor   # float32 [V, 3] or [V, 8]
    indices: torch.Tensor    # int32 [T, 3] (uint32 bit pattern)
    meshlets: torch.Tensor   # int32 [M, 4]
    active_ids: torch.Tensor
    leaf: torch.Tensor


def extract(volume: torch.Tensor, block: int, iso: float, ctx: Context | None = None,
            options: L.ExtractOptions | None = None, profiler=None) -> Mesh:
    """The plain drop-in path, stage by stage, on a CUDA volume tensor [z, y, x]."""
    own = ctx is None
    ctx = ctx or Context()
    v = wrap_volume(volume)
    pc = push_constants((volume.shape[2], volume.shape[1], volume.shape[0]), block, iso)
    mm = compute_min_max_mip(ctx, v, pc, profiler)
    f = filter_active_blocks(ctx, mm, pc, profiler)
    read_active_block_count(ctx, f)
    x = extract_meshlet_descriptors(ctx, mm, f, pc, options, profiler)
    ctx.synchronize()
    m = Mesh(x.vertices(), x.indices(), x.meshlets(), f.ids(), mm.level(0))
    x.free()
    f.free()
    mm.free()
    if own:
        ctx.close()
    return m


class AsyncExtractor:
    """The whole plain path with preallocated outputs and no host sync
    (mtx_extract_plain_async); capturable in a CUDA graph once warmed up."""

    def __init__(self, ctx: Context, volume: torch.Tensor, block: int, iso: float,
                 vertex_capacity: int, triangle_capacity: int, max_active_blocks: int = 0,
                 options: L.ExtractOptions | None = None):
        self.ctx = ctx
        self.volume = volume
        self.vol = wrap_volume(volume)
        self.pc = push_constants((volume.shape[2], volume.shape[1], volume.shape[0]), block, iso)
        self.opts = options if options is not None else extract_options()
        w = 3 if self.opts.vertexFormat == L.VERTEX_XYZ else 8
        self.vertices = torch.empty((vertex_capacity, w), dtype=torch.float32, device="cuda")
        self.indices = torch.empty((triangle_capacity, 3), dtype=torch.int32, device="cuda")
        self.counters = torch.zeros(8, dtype=torch.int32, device="cuda")
        self.bufs = L.MeshBuffers()
        self.bufs.vertices = self.vertices.data_ptr()
        self.bufs.vertexCapacity = vertex_capacity
        self.bufs.indices = self.indices.data_ptr()
        self.bufs.triangleCapacity = triangle_capacity
        self.bufs.meshlets = None
        self.bufs.meshletCapacity = 0
        self.bufs.counters = self.counters.data_ptr()
        self.bufs.maxActiveBlocks = max_active_blocks

    def set_iso(self, iso: float):
        self.pc.isovalue = float(iso)

    def run(self):
        L.check(L.lib().mtx_extract_plain_async(self.ctx.handle, C.byref(self.vol), C.byref(self.pc),
                                                C.byref(self.opts), C.byref(self.bufs)),
                "mtx_extract_plain_async", self.ctx.handle)


class Batch:
    """Many (volume, isovalue) jobs in one run (mtx_batch_*): a batched min/max
    launch and one persistent extraction kernel, recorded into a CUDA graph when
    use_graph is set.  volumes are CUDA tensors [z, y, x] of any supported
    dtype; blocks gives each volume's block edge; jobs is a list of
    (volume index, isovalue)."""

    def __init__(self, ctx: Context, volumes, blocks, jobs, max_active_blocks: int = 0,
                 vertex_capacity: int = 0, triangle_capacity: int = 0,
                 options: L.ExtractOptions | None = None, use_graph: bool = True, block_warps: int = 0):
        self.ctx = ctx
        self.volumes = list(volumes)  # keeps the tensors alive
        self._vols = (L.Volume * len(self.volumes))(*[wrap_volume(v) for v in self.volumes])
        self._blocks = (C.c_uint32 * len(self.volumes))(*[int(b) for b in blocks])
        self._jobs = (L.BatchJob * len(jobs))(*[L.BatchJob(int(v), float(i)) for v, i in jobs])
        self.njobs = len(jobs)
        opts = options if options is not None else extract_options()
        d = L.BatchDesc()
        d.volumeCount = len(self.volumes)
        d.jobCount = self.njobs
        d.volumes = self._vols
        d.blockEdges = self._blocks
        d.jobs = self._jobs
        d.maxActiveBlocks = max_active_blocks
        d.vertexCapacity = vertex_capacity
        d.triangleCapacity = triangle_capacity
        d.vertexFormat = opts.vertexFormat
        d.frame = opts.frame
        d.normals = opts.normals
        d.useGraph = 1 if use_graph else 0
        d.blockWarps = int(block_warps)
        self.handle = C.c_void_p()
        L.check(L.lib().mtx_batch_create(ctx.handle, C.byref(d), C.byref(self.handle)), "mtx_batch_create",
                ctx.handle)
        self.out = L.BatchOutputs()
        L.check(L.lib().mtx_batch_get_outputs(self.handle, C.byref(self.out)), "mtx_batch_get_outputs")

    def run(self):
        L.check(L.lib().mtx_batch_run(self.handle), "mtx_batch_run", self.ctx.handle)

    def results(self, check: bool = True):
        """(per-job results as dicts, totals dict); waits for the last run."""
        res = (L.BatchJobResult * self.njobs)()
        tot = L.BatchTotals()
        st = L.lib().mtx_batch_read_results(self.handle, C.cast(res, C.c_void_p), C.byref(tot))
        if check:
            L.check(st, "mtx_batch_read_results", self.ctx.handle)
        jobs = [{f: getattr(r, f) for f, _ in L.BatchJobResult._fields_} for r in res]
        totals = {f: getattr(tot, f) for f, _ in L.BatchTotals._fields_}
        return jobs, totals

    def mesh(self, r: dict):
        """Views of one job's vertices [V, 3|8], indices [T, 3] (relative to the
        job's first vertex) and meshlet descriptors [M, 4]."""
        w = self.out.vertexStride // 4
        v = device_view(self.out.vertexBuffer.ptr + 4 * w * r["vertexOffset"], (r["vertexCount"], w), torch.float32)
        i = device_view(self.out.indexBuffer.ptr + 4 * r["indexOffset"], (r["indexCount"] // 3, 3), torch.int32)
        m = device_view(self.out.meshletDescriptorBuffer.ptr + 16 * r["meshletOffset"], (r["meshletCount"], 4),
                        torch.int32)
        return v, i, m

    def close(self):
        if self.handle:
            self.ctx.fence()
            L.lib().mtx_batch_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(ctx: Context, volume: torch.Tensor, iso: float, cache_path: str | None = None, flags: int = 0) -> dict:
    """mtx_autotune on a CUDA volume tensor [z, y, x]: the block edge and the
    tuning to use for it ({blockEdge, tuning: {...}, ms, fromCache, candidates})."""
    r = L.AutotuneResult()
    v = wrap_volume(volume)
    L.check(L.lib().mtx_autotune(ctx.handle, C.byref(v), float(iso),
                                 cache_path.encode() if cache_path else None, int(flags), C.byref(r)),
            "mtx_autotune", ctx.handle)
    t = {f: getattr(r.tuning, f) for f, _ in L.Tuning._fields_}
    return {"blockEdge": r.blockEdge, "tuning": t, "ms": r.ms, "fromCache": r.fromCache, "candidates": r.candidates}


def autotune_batch(ctx: Context, volumes, jobs, cache_path: str | None = None, flags: int = 0) -> dict:
    """mtx_autotune_batch: the block edge of every volume and the batched
    kernel's block warps for the batch (volumes: CUDA tensors [z, y, x]; jobs:
    (volume index, isovalue)), timed on the batched run itself.  Returns
    {blockEdges: [...], blockWarps, ms, fromCache, candidates}."""
    vols = list(volumes)
    nv = len(vols)
    d = L.BatchDesc()
    arr = (L.Volume * nv)(*[wrap_volume(v) for v in vols])
    edges = (C.c_uint32 * nv)(*([8] * nv))
    jarr = (L.BatchJob * len(jobs))(*[L.BatchJob(int(v), float(i)) for v, i in jobs])
    d.volumeCount = nv
    d.jobCount = len(jobs)
    d.volumes = arr
    d.blockEdges = edges
    d.jobs = jarr
    out_edges = (C.c_uint32 * nv)()
    r = L.BatchAutotuneResult()
    L.check(L.lib().mtx_autotune_batch(ctx.handle, C.byref(d), cache_path.encode() if cache_path else None,
                                       int(flags), out_edges, C.byref(r)), "mtx_autotune_batch", ctx.handle)
    return {"blockEdges": list(out_edges), "blockWarps": r.blockWarps, "ms": r.ms, "fromCache": r.fromCache,
            "candidates": r.candidates}
