/*
 * meshtrex-b200 C ABI: the isosurface-extraction path of meshtrex (block
 * min/max -> active-block filtering + compaction -> PMB marching cubes) on
 * one NVIDIA B200, behind plain C entry points.
 *
 * These calls replace, for compute only, what meshtrex does through its
 * Vulkan runtime (src/vulkan_context.*, src/device.*, src/buffer.*,
 * src/image.*) and its three stage managers.  Each declaration names the
 * meshtrex interface it stands in for.  The C++ drop-in facade with the
 * reference's own names (computeMinMaxMip, filterActiveBlocks,
 * readActiveBlockCount, extractMeshletDescriptors) is in the other headers
 * of this directory and is written on top of this ABI.
 *
 * Conventions
 *  - Every entry point returns mtx_status and never throws or aborts.
 *  - Pointers named "device" are CUDA device pointers on the context's
 *    device; everything else is host memory.
 *  - Work is issued on the context's stream (mtx_context_set_stream, the
 *    analogue of meshtrex's externalCmd command buffer).  Calls that need a
 *    host value from the GPU (counts) synchronise that stream; the *_async
 *    calls never do and can be captured in a CUDA graph.
 *  - Volumes are x fastest, then y, then z: voxel (x,y,z) is element
 *    z*X*Y + y*X + x (src/volume.h:8-12, src/testMinMax.h:97-101).
 *  - The *_free calls release device memory in the order of the context's
 *    stream, as cudaFreeAsync does, and do not wait: work queued on other
 *    streams that still reads an output must finish (or be ordered before
 *    the context's stream) before the output is freed.
 */
#ifndef MESHTREX_MTX_H
#define MESHTREX_MTX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MTX_ABI_VERSION 1
#define MTX_MAX_MIP_LEVELS 32
#define MTX_MAX_BLOCK_EDGE 16

typedef enum mtx_status {
    MTX_OK = 0,
    MTX_ERR_INVALID_ARG = 1, /* bad pointer, size, dims or option */
    MTX_ERR_UNSUPPORTED = 2, /* valid but not implemented (e.g. block edge > 16) */
    MTX_ERR_OOM = 3,         /* a device or host allocation failed */
    MTX_ERR_CAPACITY = 4,    /* caller buffers too small; counters hold the needed sizes */
    MTX_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up (error word set) */
    MTX_ERR_CUDA = 6,        /* a CUDA runtime call failed */
    MTX_ERR_NO_DEVICE = 7,   /* no usable CUDA device */
    MTX_ERR_INTERNAL = 8     /* an invariant check inside a kernel failed */
} mtx_status;

typedef enum mtx_dtype {
    MTX_DTYPE_U8 = 0,  /* meshtrex's only type on the GPU (R8_UINT, minMaxManager.cpp:117) */
    MTX_DTYPE_U16 = 1, /* loadVolume's 2-byte type (volume.h:29-30) */
    MTX_DTYPE_F32 = 2
} mtx_dtype;

/* PushConstants (src/common.h:29-34): same fields, order and 16-byte
 * alignment.  blockGridDim = ceil(volumeDim / blockDim) (src/meshtrex.cpp:79-83). */
typedef struct mtx_push_constants {
    uint32_t volumeDim[4];
    uint32_t blockDim[4];
    uint32_t blockGridDim[4];
    float isovalue;
    uint32_t _pad[3];
} mtx_push_constants;

/* A span of device memory: meshtrex's Buffer (src/resources.h, buffer.h:10-18)
 * reduced to what compute needs. */
typedef struct mtx_buffer {
    void *ptr;
    uint64_t size; /* bytes */
} mtx_buffer;

typedef struct mtx_context *mtx_context_t;
typedef struct mtx_profiler *mtx_profiler_t;

/* Device-resident scalar volume: meshtrex's Volume (src/volume.h:8-12) once
 * uploaded (MinMaxOutput::volumeImage, src/minMaxOutput.h:11). */
typedef struct mtx_volume {
    mtx_buffer data;
    uint32_t dims[3];
    uint32_t dtype; /* mtx_dtype */
    uint32_t owned; /* 1 if mtx_volume_free releases data.ptr */
    uint32_t _pad;
} mtx_volume;

/* MinMaxOutput (src/minMaxOutput.h:10-65).  minMaxImage holds every mip
 * level back to back as {min,max} uint32 keys (R32G32_UINT in meshtrex);
 * levelOffset/levelExtent play the part of minMaxMipViews.  Keys are the
 * voxel values for u8/u16 and an order-preserving transform for f32
 * (mtx_key_to_float). */
typedef struct mtx_minmax_output {
    mtx_volume volumeImage; /* borrowed copy of the input descriptor */
    mtx_buffer minMaxImage;
    uint32_t mipLevels;
    uint32_t blockDim[3];
    uint32_t blockGridDim[3];
    uint32_t levelExtent[MTX_MAX_MIP_LEVELS][3];
    uint64_t levelOffset[MTX_MAX_MIP_LEVELS]; /* in texels (8 bytes each) */
} mtx_minmax_output;

/* FilteringOutput (src/filteringOutput.h:11-74) plus the dense rank map the
 * extraction uses to find a neighbouring block's vertices. */
typedef struct mtx_filtering_output {
    mtx_buffer compactedBlockIdBuffer; /* uint32[totalBlocks]; the first count are valid, ascending */
    mtx_buffer activeBlockCountBuffer; /* uint32 */
    mtx_buffer blockRankBuffer;        /* uint32[totalBlocks]; rank of block id b, valid where b is active */
    uint32_t activeBlockCount;         /* host copy: 0 until mtx_read_active_block_count */
    uint32_t totalBlocks;
    float isovalue;
    uint32_t _pad;
} mtx_filtering_output;

typedef enum mtx_vertex_format {
    MTX_VERTEX_XYZ = 0, /* 12 bytes: float x, y, z */
    MTX_VERTEX_DATA = 1 /* 32 bytes: VertexData{vec4 position; vec4 normal} (extractionOutput.h:131-134) */
} mtx_vertex_format;

typedef enum mtx_frame {
    MTX_FRAME_VOXEL = 0, /* positions in voxel units (the exact parity frame) */
    MTX_FRAME_NDC = 1    /* (pos / volumeDim) * 2 - 1, as meshtrex writes (marching_cubes_pmb.mesh.glsl:138) */
} mtx_frame;

typedef enum mtx_staging {
    MTX_STAGING_AUTO = 0, /* TMA when the volume's layout allows it */
    MTX_STAGING_TMA = 1,  /* cp.async.bulk.tensor 3D tile of the block + halo */
    MTX_STAGING_LDG = 2   /* plain coalesced loads */
} mtx_staging;

typedef struct mtx_extract_options {
    uint32_t vertexFormat; /* mtx_vertex_format */
    uint32_t frame;        /* mtx_frame */
    uint32_t normals;      /* MTX_VERTEX_DATA only: 1 = fill the normal (pmb.mesh.glsl:111-137) */
    uint32_t staging;      /* mtx_staging */
    uint32_t threads;      /* threads per CTA of the extraction kernels; 0 = auto */
    uint32_t _pad;
    uint8_t *cellCases;    /* optional device output: B^3 case bytes per active block, rank order */
} mtx_extract_options;

/* MeshletDescriptor (extractionOutput.h:124-129).  One per active block, in
 * rank order: its own vertices and its triangles (indexOffset counts uint32s). */
typedef struct mtx_meshlet_descriptor {
    uint32_t vertexOffset;
    uint32_t indexOffset;
    uint32_t vertexCount;
    uint32_t primitiveCount;
} mtx_meshlet_descriptor;

/* ExtractionOutput (src/extractionOutput.h:10-122).  Buffers are sized
 * exactly, not for the worst case; meshletCount is the true count. */
typedef struct mtx_extraction_output {
    mtx_buffer vertexBuffer;
    mtx_buffer vertexCountBuffer; /* uint32 */
    mtx_buffer indexBuffer;       /* uint32, 3 per triangle, global vertex ids */
    mtx_buffer indexCountBuffer;  /* uint32 */
    mtx_buffer meshletDescriptorBuffer;
    mtx_buffer meshletDescriptorCountBuffer; /* uint32 */
    uint32_t meshletCount;
    uint32_t vertexCount;
    uint32_t indexCount;
    uint32_t vertexStride; /* 12 or 32 bytes */
} mtx_extraction_output;

/* Caller-owned outputs of the asynchronous whole-path call.  counters (device,
 * uint32[8]) receive {vertexCount, indexCount, meshletCount, activeBlockCount,
 * status, 0, 0, 0}; they hold the full sizes even when a capacity was short. */
typedef struct mtx_mesh_buffers {
    void *vertices;
    uint64_t vertexCapacity; /* vertices */
    uint32_t *indices;
    uint64_t triangleCapacity; /* triangles */
    mtx_meshlet_descriptor *meshlets; /* optional */
    uint64_t meshletCapacity;
    uint32_t *counters;
    /* Upper bound on active blocks, sizing the scratch of the extraction
     * (0 = every block of the grid); more active blocks -> MTX_ERR_CAPACITY.
     * The scratch per active block is 12 B^2 bytes of face records, 16 B of
     * descriptor and, for B <= 8, the block state the count pass hands to the
     * emit pass (1920 B at B = 8): about 2.7 KB at B = 8, so a bound well
     * under the grid's block count saves gigabytes on large volumes. */
    uint64_t maxActiveBlocks;
} mtx_mesh_buffers;

/* ------------------------------------------------------------ context */

/* Human-readable name of a status code. */
const char *mtx_status_string(mtx_status s);
uint32_t mtx_abi_version(void);

/* VulkanContext (src/vulkan_context.h:7-45), compute only: binds a CUDA
 * device, a stream (NULL = the legacy default stream) and a grow-only
 * scratch arena. */
mtx_status mtx_context_create(int device, void *stream, mtx_context_t *out);
mtx_status mtx_context_destroy(mtx_context_t ctx);
mtx_status mtx_context_set_stream(mtx_context_t ctx, void *stream);
/* A second stream for the count, scan and emit passes of
 * mtx_extract_plain_async (NULL: none, everything on the context's stream).
 * With it, the call queues the leaf min/max, octree and filter on the
 * context's stream and the extraction passes on this one behind an event, so
 * that work queued next on the context's stream -- the min/max of the next
 * volume or isovalue, for one -- runs while this extraction is still being
 * emitted.  The context's scratch is reused by its next call, so that call's
 * filter waits for this extraction first, and every other call on the context
 * joins the extraction stream before it starts.  mtx_synchronize waits for
 * both streams.  Meant for eager use: a stream capture must not span calls on
 * such a context.  No meshtrex counterpart (one queue, vulkan_context.cpp:94-109). */
mtx_status mtx_context_set_extract_stream(mtx_context_t ctx, void *stream);
/* Last error text of this context ("" if none). */
const char *mtx_context_last_error(mtx_context_t ctx);
/* Wait for the stream, then report (and clear) any error a kernel recorded. */
mtx_status mtx_synchronize(mtx_context_t ctx);
/* Host-side fault injection for tests: the k-th device allocation from now
 * fails with MTX_ERR_OOM (k = 0 disables). */
mtx_status mtx_debug_fail_allocation(mtx_context_t ctx, uint32_t k);
/* Failure injection for tests of the bounded waits, on the host: the
 * look-back waits of this context's compaction and count scans give up after
 * max_polls polls (0: the built-in bound of about a second), and withhold
 * bit 0 (compaction) / bit 1 (count scan) makes the next launches skip the
 * ticket of their first tile, so that every later tile waits for a
 * predecessor that never publishes.  Those tiles give up, record
 * MTX_ERR_TIMEOUT (reported by mtx_synchronize) and abort their successors;
 * the context stays usable.  mtx_debug_set_waits(ctx, 0, 0) restores normal
 * operation.  No meshtrex counterpart. */
mtx_status mtx_debug_set_waits(mtx_context_t ctx, uint32_t max_polls, uint32_t withhold);

/* ------------------------------------------------------------- volume */

/* loadVolume's in-memory result + the staging upload of computeMinMaxMip
 * (src/volume.h:14-43, src/minMaxManager.cpp:115-125): copies host voxels
 * into a new device volume. */
mtx_status mtx_volume_upload(mtx_context_t ctx, const void *host, const uint32_t dims[3],
                             uint32_t dtype, mtx_volume *out);
/* Describes existing device memory as a volume (no copy, not owned). */
mtx_status mtx_volume_wrap(void *device_ptr, const uint32_t dims[3], uint32_t dtype,
                           mtx_volume *out);
mtx_status mtx_volume_free(mtx_context_t ctx, mtx_volume *vol);

/* The file-name scheme of loadVolume (src/volume.h:14-30):
 * "<name>_<X>x<Y>x<Z>_<type>.raw" with type uint8, uint16 or float32 (also
 * "float").  meshtrex reads every type other than uint8 as 16-bit; here an
 * unknown type is MTX_ERR_UNSUPPORTED and a name that does not match is
 * MTX_ERR_INVALID_ARG.  Host only. */
mtx_status mtx_parse_volume_name(const char *path, uint32_t dims[3], uint32_t *dtype);
/* loadVolume (src/volume.h:14-43) and the staging upload of computeMinMaxMip
 * (src/minMaxManager.cpp:115-125) in one call: the raw file is streamed to a
 * new device volume through two 64 MiB pinned buffers, reading one chunk
 * while the previous one is copied.  Returns when the volume is on the
 * device.  A file shorter than its name says is MTX_ERR_INVALID_ARG. */
mtx_status mtx_volume_load(mtx_context_t ctx, const char *path, mtx_volume *out);

/* PushConstants as src/meshtrex.cpp:76-84 fills them, for a cubic block. */
mtx_status mtx_push_constants_init(const uint32_t dims[3], uint32_t block_edge, float isovalue,
                                   mtx_push_constants *out);
/* Decode a min/max key back to the voxel value (u8/u16: the value). */
float mtx_key_to_float(uint32_t dtype, uint32_t key);

/* ------------------------------------------------------------ stage 1 */

/* computeMinMaxMip (src/minMaxManager.h:20-21, minMaxManager.cpp:63-225):
 * per-block min/max over (B+1)^3 voxels, then the min/max octree with
 * 1 + floor(log2(max grid extent)) levels of ceil extents. */
mtx_status mtx_compute_min_max_mip(mtx_context_t ctx, const mtx_volume *vol,
                                   const mtx_push_constants *pc, mtx_profiler_t prof,
                                   mtx_minmax_output *out);
/* loadVolume's staging upload and computeMinMaxMip in one call, overlapped
 * (src/volume.h:14-43, src/minMaxManager.cpp:63-225; meshtrex copies the
 * whole volume, then dispatches, minMaxManager.cpp:115-133).  The host voxels
 * go to a new device volume in z-slabs on a copy stream of the context; the
 * leaf min/max of each slab of block layers runs on the context's stream as
 * soon as its voxels and the one-voxel halo above them are on the device, so
 * when the last slab lands only its own leaf pass and the octree remain.  The
 * outputs equal mtx_volume_upload followed by mtx_compute_min_max_mip.  Does
 * not wait: `host` must stay unchanged until the context's stream has done
 * this work.  Pinned host memory (cudaHostAlloc, cudaHostRegister) is needed
 * for the copies to overlap anything.  vol_out is owned by the caller (free it
 * with mtx_volume_free), out as from mtx_compute_min_max_mip. */
mtx_status mtx_upload_compute_min_max_mip(mtx_context_t ctx, const void *host, const uint32_t dims[3],
                                          uint32_t dtype, const mtx_push_constants *pc, mtx_profiler_t prof,
                                          mtx_volume *vol_out, mtx_minmax_output *out);
mtx_status mtx_minmax_free(mtx_context_t ctx, mtx_minmax_output *mm);

/* ------------------------------------------------------------ stage 2 */

/* filterActiveBlocks (src/filteringManager.h:9-10, filteringManager.cpp:20-141):
 * active = min != max and the isovalue in [min, max] (round(iso) for integer
 * volumes, blockFilteringTestUtils.h:456-469); compacted in ascending block
 * order by a single-pass decoupled look-back scan. */
mtx_status mtx_filter_active_blocks(mtx_context_t ctx, const mtx_minmax_output *mm,
                                    const mtx_push_constants *pc, mtx_profiler_t prof,
                                    mtx_filtering_output *out);
/* readActiveBlockCount (src/filteringManager.h:13, filteringManager.cpp:144-164). */
mtx_status mtx_read_active_block_count(mtx_context_t ctx, mtx_filtering_output *filt);
mtx_status mtx_filtering_free(mtx_context_t ctx, mtx_filtering_output *filt);

/* Active-block filtering and ordered compaction that allocates no memory.
 * No counterpart in meshtrex: it is for callers that cannot allocate device
 * memory while they run -- an application that owns a fixed device-memory
 * budget, or code running where cudaMalloc is not allowed -- and that also
 * cannot hold an mtx context (creating one allocates).  It runs the same
 * compaction as mtx_filter_active_blocks on the current device and the given
 * stream, with its scratch in a fixed 256 KiB array inside the library
 * (every GPU that loads the library keeps it until the process exits), and
 * calls no allocator.
 *   leaf_minmax   device, 16-byte aligned: {min,max} keys of total_blocks blocks (mip level 0)
 *   compacted_ids device, total_blocks words: the active block ids, ascending
 *   block_rank    device, 16-byte aligned, total_blocks words: rank of each block, 0xffffffff if inactive
 *   active_count  device, one word
 *   device_status device, 4 words (required): {mtx_status, site, info, info} of an
 *                 error a kernel met (a look-back wait that gave up), zero otherwise;
 *                 read it after the stream is done, before trusting the outputs
 * A missing or misaligned pointer is MTX_ERR_INVALID_ARG before any work.
 * Limit: total_blocks <= 67,108,864 (65,536 tiles of 1024 blocks), else
 * MTX_ERR_CAPACITY before any work.  The first call in a CUDA context looks
 * up the array's device address in that context (again after
 * cudaDeviceReset); make that first call before any stream capture.
 * Every call reuses the same array, so calls that overlap on the GPU race:
 * issue them one after the other. */
mtx_status mtx_filter_active_blocks_noalloc(const uint32_t *leaf_minmax, uint64_t total_blocks, uint32_t dtype,
                                            float isovalue, uint32_t *compacted_ids, uint32_t *block_rank,
                                            uint32_t *active_count, uint32_t *device_status, void *stream);

/* ------------------------------------------------------------ stage 3 */

/* extractMeshletDescriptors (src/extractionManager.h:10-11,
 * extractionManager.cpp:250-717): PMB marching cubes over the active blocks.
 * Like meshtrex, returns an empty output when filt->activeBlockCount is 0
 * (the host count must have been read).  Counts, then allocates the outputs
 * exactly, then emits; each vertex is written once, by its owning block. */
mtx_status mtx_extract_meshlet_descriptors(mtx_context_t ctx, const mtx_minmax_output *mm,
                                           const mtx_filtering_output *filt,
                                           const mtx_push_constants *pc,
                                           const mtx_extract_options *opts, mtx_profiler_t prof,
                                           mtx_extraction_output *out);
mtx_status mtx_extraction_free(mtx_context_t ctx, mtx_extraction_output *ext);

/* The three stages in one call with caller-owned outputs and no host
 * synchronisation (main's sequence, src/meshtrex.cpp:107-141, without the
 * blocking count readback).  Capacity overflow is reported through
 * counters[4] and mtx_synchronize as MTX_ERR_CAPACITY. */
mtx_status mtx_extract_plain_async(mtx_context_t ctx, const mtx_volume *vol,
                                   const mtx_push_constants *pc, const mtx_extract_options *opts,
                                   const mtx_mesh_buffers *out);

/* ------------------------------------------------------------ meshlets */

/* Meshlets in the form meshtrex's renderer reads (render.task.glsl:55-250):
 * each meshlet's triangles index only its own vertices,
 * [vertexOffset, vertexOffset + vertexCount) of vertexBuffer. */
typedef struct mtx_meshlet_output {
    mtx_buffer meshletDescriptorBuffer; /* mtx_meshlet_descriptor per meshlet; indexOffset counts uint32s */
    mtx_buffer meshletVertexBuffer;     /* uint32 per meshlet vertex: its vertex id in the extraction's mesh */
    mtx_buffer vertexBuffer;            /* the extraction's vertex records, gathered in meshlet order */
    mtx_buffer indexBuffer;             /* uint32, 3 per triangle (the mesh's triangle order), ids into vertexBuffer */
    uint32_t meshletCount;
    uint32_t vertexCount; /* meshlet vertices: shared vertices appear once per meshlet that uses them */
    uint32_t indexCount;
    uint32_t vertexStride; /* bytes, as the extraction's */
} mtx_meshlet_output;

/* Splits the mesh of an extraction into meshlets of at most maxVertices
 * (3..64; 64 in meshtrex) vertices and maxPrimitives (1..1024; 126 in
 * meshtrex) triangles (the limits of marching_cubes_pmb.task.glsl:24-25).
 * Each block's triangles are taken in their canonical order and a new
 * meshlet starts when the next triangle's new vertices or the triangle count
 * would pass a limit, so meshlets never span blocks and the result does not
 * depend on the run.  Allocates the outputs; free them with
 * mtx_meshlet_output_free.  meshtrex makes meshlets in its task and mesh
 * shaders and splits them again in the renderer; this is the same contract as
 * a post-pass. */
mtx_status mtx_build_meshlets(mtx_context_t ctx, const mtx_extraction_output *ext, uint32_t maxVertices,
                              uint32_t maxPrimitives, mtx_meshlet_output *out);
mtx_status mtx_meshlet_output_free(mtx_context_t ctx, mtx_meshlet_output *out);

/* ------------------------------------------------------------ export */

/* readDataChunkFromBuffer / readCounterFromBuffer
 * (src/extractionTestUtils.cpp:203-235): copies bytes from offset of a
 * device buffer into host memory, after the work queued on the context's
 * stream. */
mtx_status mtx_read_buffer(mtx_context_t ctx, const mtx_buffer *src, uint64_t offset, void *host, uint64_t bytes);

/* Weld check of a mesh written by mtx_write_obj. */
typedef struct mtx_obj_stats {
    uint32_t vertexCount;
    uint32_t triangleCount;
    uint32_t uniqueVertexCount;       /* distinct position (and normal) bit patterns */
    uint32_t degenerateTriangleCount; /* triangles with two corners at the same vertex or position */
} mtx_obj_stats;

/* writeGPUExtractionToOBJ (src/extractionTestUtils.cpp:203-369) for host
 * copies of the mesh: "v" lines, "vn" lines for the 32-byte VertexData
 * layout (vertexStride 8 floats; 3 = xyz only), and 1-based "f" lines
 * ("f a//a b//b c//c" with normals).  Coordinates are written with 9
 * significant digits, so that they read back to the same float bits
 * (meshtrex writes 6).  Like meshtrex it reports the distinct vertices and
 * the degenerate triangles but writes the mesh as given; PMB writes every
 * vertex once, so the vertex count and the distinct count agree. */
mtx_status mtx_write_obj(const char *path, const float *vertices, uint32_t vertexCount, uint32_t vertexStride,
                         const uint32_t *indices, uint32_t indexCount, mtx_obj_stats *stats);

/* ------------------------------------------------------------ adjoint */

typedef enum mtx_adjoint_mode {
    MTX_ADJOINT_ATOMIC = 0,       /* dL/dfield by FP32 atomics: summation order varies between runs */
    MTX_ADJOINT_DETERMINISTIC = 1 /* per-block partial sums reduced in a fixed order: bitwise reproducible */
} mtx_adjoint_mode;

/* Adjoint of the extraction with the topology held fixed (meshtrex has no
 * backward pass).  Every vertex lies on a cut edge (a, b) at
 * p = a + t * axis with t = (iso - f(a)) / (f(b) - f(a)), which is recomputed
 * from the volume, not stored.  Given dL/dvertex it writes the dense
 * dL/dfield (every voxel; zero away from the surface) and dL/diso:
 *   dL/df(a) += g * (iso - f(b)) / (f(b) - f(a))^2
 *   dL/df(b) += g * (f(a) - iso) / (f(b) - f(a))^2
 *   dL/diso  += g / (f(b) - f(a))
 * with g the gradient of the vertex coordinate along the edge (vertices
 * whose |f(b) - f(a)| <= 1e-5 sit at t = 0.5 and have no gradient).
 * filt and meshlets come from the forward extraction of the same volume and
 * push constants (the count must have been read back); dl_dvertex holds
 * vertexStride floats per vertex with the position gradient first, in the
 * forward's frame.  The output buffers are device memory, overwritten.  A
 * block whose topology no longer matches its meshlet descriptor makes the
 * call fail with MTX_ERR_INTERNAL at mtx_synchronize. */
mtx_status mtx_extract_backward(mtx_context_t ctx, const mtx_volume *vol, const mtx_push_constants *pc,
                                const mtx_filtering_output *filt, const mtx_meshlet_descriptor *meshlets,
                                uint32_t vertexCount, const float *dl_dvertex, uint32_t vertexStride,
                                uint32_t frame, float *dl_dfield, float *dl_diso, uint32_t mode);

/* ------------------------------------------------------------ batches */

/* Many extractions in one go: any number of device-resident volumes (mixed
 * dtypes and sizes), each extracted at one or more isovalues.  A run is two
 * launches -- the leaf min/max of every volume, then one persistent kernel
 * that filters, compacts, counts, scans and emits every job -- and is
 * recorded once into a CUDA graph when useGraph is set.  meshtrex has no
 * batched path; each job's output equals what the plain sequence
 * (mtx_compute_min_max_mip, mtx_filter_active_blocks,
 * mtx_extract_meshlet_descriptors) gives for that volume, block edge and
 * isovalue, with the vertex and meshlet offsets counted from the job's own
 * first vertex and index. */
typedef struct mtx_batch *mtx_batch_t;

typedef struct mtx_batch_job {
    uint32_t volume; /* index into mtx_batch_desc::volumes */
    float isovalue;
} mtx_batch_job;

typedef struct mtx_batch_desc {
    uint32_t volumeCount;
    uint32_t jobCount;
    const mtx_volume *volumes;   /* device-resident; they must outlive the batch */
    const uint32_t *blockEdges;  /* per volume, 2..16 */
    const mtx_batch_job *jobs;
    /* Pooled capacities over all jobs (0 = a default: every block of every
     * job; 4 * B^2 vertices and 8 * B^2 triangles per active block, B the
     * largest block edge).  A run that needs more reports MTX_ERR_CAPACITY
     * with the sizes it needed in mtx_batch_totals. */
    uint64_t maxActiveBlocks;
    uint64_t vertexCapacity;
    uint64_t triangleCapacity;
    uint32_t vertexFormat; /* mtx_vertex_format */
    uint32_t frame;        /* mtx_frame */
    uint32_t normals;      /* MTX_VERTEX_DATA only */
    uint32_t useGraph;     /* 1 = record the run into a CUDA graph at the first mtx_batch_run */
    uint32_t blockWarps;   /* warps of each CTA of the persistent kernel that take blocks, 1..8 (0 = as many
                              as the shared memory holds, at most 8); fewer gives more CTAs an SM */
} mtx_batch_desc;

/* One job's slice of the pooled outputs. */
typedef struct mtx_batch_job_result {
    uint32_t meshletOffset; /* first meshlet descriptor of the job (= its first active block) */
    uint32_t meshletCount;  /* active blocks */
    uint32_t vertexCount;
    uint32_t indexCount;
    uint64_t vertexOffset;  /* first vertex of the job in the pooled vertex buffer */
    uint64_t indexOffset;   /* first index of the job in the pooled index buffer */
} mtx_batch_job_result;

/* Totals of a run.  On MTX_ERR_CAPACITY they are the sizes the run needed. */
typedef struct mtx_batch_totals {
    int32_t status; /* mtx_status of the run */
    uint32_t activeBlocks;
    uint64_t vertexCount;
    uint64_t triangleCount;
} mtx_batch_totals;

typedef struct mtx_batch_outputs {
    mtx_buffer vertexBuffer;            /* pooled vertices of every job */
    mtx_buffer indexBuffer;             /* uint32; each job's indices count from its own first vertex */
    mtx_buffer meshletDescriptorBuffer; /* pooled; offsets count from the job's first vertex and index */
    mtx_buffer jobResultBuffer;         /* mtx_batch_job_result[jobCount] */
    uint32_t vertexStride;              /* 12 or 32 bytes */
    uint32_t _pad;
} mtx_batch_outputs;

/* Allocates everything a run needs (no allocation happens in mtx_batch_run). */
mtx_status mtx_batch_create(mtx_context_t ctx, const mtx_batch_desc *desc, mtx_batch_t *out);
/* Enqueues one run on the context's stream; does not wait. */
mtx_status mtx_batch_run(mtx_batch_t b);
mtx_status mtx_batch_get_outputs(mtx_batch_t b, mtx_batch_outputs *out);
/* Waits for the last run, then copies the per-job results (results may be
 * NULL; else jobCount entries) and the totals (may be NULL). */
mtx_status mtx_batch_read_results(mtx_batch_t b, mtx_batch_job_result *results, mtx_batch_totals *totals);
mtx_status mtx_batch_destroy(mtx_batch_t b);

/* ------------------------------------------------------------ profiler */

/* GPUProfiler (src/gpuProfiler.h:11-160): CUDA events around the stage
 * names MinMax_Leaf_Pass, MinMax_Octree_Reduction, Active_Block_Filtering
 * and Mesh_Extraction. */
mtx_status mtx_profiler_create(mtx_context_t ctx, mtx_profiler_t *out);
mtx_status mtx_profiler_destroy(mtx_profiler_t prof);
mtx_status mtx_profiler_begin_frame(mtx_profiler_t prof);
/* Waits for the frame's events and accumulates per-region times. */
mtx_status mtx_profiler_end_frame(mtx_profiler_t prof);
uint32_t mtx_profiler_region_count(mtx_profiler_t prof);
/* name (<= 63 chars + NUL) and the last frame's and running-average time in ms. */
mtx_status mtx_profiler_region(mtx_profiler_t prof, uint32_t i, char name[64], double *last_ms,
                               double *avg_ms, uint32_t *frames);
/* Launch-shape knobs of the kernels (0 = built-in default), the search space
 * of mtx_autotune; meshtrex's only counterparts are its compile-time
 * workgroup sizes and specialization constants (extractionPipeline.cpp:238-256). */
typedef struct mtx_tuning {
    uint32_t minmaxZChunk;  /* block slabs per warp in the min/max pass */
    uint32_t minmaxSlices;  /* 0 (default): a TMA ring of z slices for 2- and 4-byte voxels (else 2);
                               1, 2 or 4: the load-based pass with that many z slices in flight */
    uint32_t extractWarps;  /* warps per CTA of the extraction passes: 1, 2, 4 (default) or 8 */
    uint32_t staging;       /* mtx_staging used when the extract options say AUTO */
    uint32_t extractCtasPerSm; /* at most this many CTAs an SM in the count and emit passes (0 = as many as
                                  fit): leaves room on each SM for another stream's min/max pass */
} mtx_tuning;
mtx_status mtx_context_set_tuning(mtx_context_t ctx, const mtx_tuning *t);
mtx_status mtx_context_get_tuning(mtx_context_t ctx, mtx_tuning *t);

/* Result of mtx_autotune: pass blockEdge to mtx_push_constants_init and tuning
 * to mtx_context_set_tuning.  The block edge changes the meshlet layout and
 * the output order (one meshlet per block), not the surface. */
typedef struct mtx_autotune_result {
    uint32_t blockEdge;  /* 4, 8 or 16 */
    mtx_tuning tuning;
    double ms;           /* device time of one plain extraction with these choices */
    uint32_t fromCache;  /* 1 if no candidate was timed */
    uint32_t candidates; /* candidates timed */
} mtx_autotune_result;

#define MTX_AUTOTUNE_IGNORE_CACHE 1u /* time the candidates even if a cached choice exists */
#define MTX_AUTOTUNE_QUICK 2u        /* one repetition per candidate instead of the best of three */

/* Picks the block edge (4, 8, 16), the warps per CTA of the extraction passes
 * (2, 4, 8), the staging (TMA or plain loads) and the min/max pass (TMA ring or 1, 2, 4 slices of loads)
 * for one volume by timing the whole plain extraction of each candidate at
 * `isovalue` on the device.  The score is the sum of the stage times that CUDA
 * events record.  The choice is cached per (dims, dtype, device name) in the
 * process and, when cache_path is not NULL, appended to that text file,
 * which later calls and processes read first.  The context's tuning is left
 * as it was.  No meshtrex counterpart: meshtrex fixes these at compile time
 * (extractionPipeline.cpp:238-256, pmb.task.glsl:19,27). */
mtx_status mtx_autotune(mtx_context_t ctx, const mtx_volume *vol, float isovalue, const char *cache_path,
                        uint32_t flags, mtx_autotune_result *out);

/* Result of mtx_autotune_batch (the per-volume block edges go to the
 * caller's array). */
typedef struct mtx_batch_autotune_result {
    uint32_t blockWarps; /* for mtx_batch_desc::blockWarps (0 = as many as fit) */
    uint32_t fromCache;  /* 1 if no candidate was timed */
    uint32_t candidates; /* candidates timed */
    uint32_t _pad;
    double ms;           /* device time of one batched run with these choices */
} mtx_batch_autotune_result;

/* Picks, for a batch, the block edge of every volume (4, 8 or 16, written to
 * blockEdges[volumeCount]) and the batched kernel's block warps by timing the
 * batched run itself on the device: one edge for all volumes at two warp
 * counts, then each dtype's volumes moved to the other edges.  desc's own
 * blockEdges, capacities, blockWarps and useGraph are ignored.  The choice
 * is cached per (the batch's (dims, dtype) list, device name) in the process
 * and, when cache_path is not NULL, appended to that text file, which later
 * calls and processes read first.  flags as mtx_autotune.  No meshtrex
 * counterpart. */
mtx_status mtx_autotune_batch(mtx_context_t ctx, const mtx_batch_desc *desc, const char *cache_path,
                              uint32_t flags, uint32_t *blockEdges, mtx_batch_autotune_result *out);

/* Records the stage times of every later call on this context that is not
 * given its own profiler, the asynchronous whole-path call included (NULL
 * turns it off); the GPUProfiler* argument of meshtrex's managers made
 * context-wide (src/minMaxManager.h:21). */
mtx_status mtx_context_set_profiler(mtx_context_t ctx, mtx_profiler_t prof);
/* ProfilingManager::exportCSV (src/profilingManager.h:141-171). */
mtx_status mtx_profiler_export_csv(mtx_profiler_t prof, const char *path);

#ifdef __cplusplus
}
#endif
#endif /* MESHTREX_MTX_H */
