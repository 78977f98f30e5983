// Host-side internals shared by the translation units of libmeshtrex_b200.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "meshtrex/mtx.h"
#include "mtx_device.cuh"

namespace mtx {

// Per-pipeline control words in device memory.
struct Ctrl {
    DevStatus status;        // first error recorded by any kernel
    uint32_t filter_ticket;  // tile tickets of the compaction scan
    uint32_t count_ticket;   // block tickets of the count scan
    uint32_t active_count;   // compaction result
    uint32_t pad0;
    uint32_t totals[4];      // vertexCount, indexCount, meshletCount, activeBlockCount
    uint32_t batch_ticket[4];
    uint32_t pyr_done;       // octree tiles finished (the last one builds the top levels)
    uint32_t pad1[3];
};

// A grow-only device allocation owned by the context.
struct Scratch {
    void *ptr = nullptr;
    size_t size = 0;
};

struct TensorMapFn;

}  // namespace mtx

struct mtx_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sm_count = 0;
    int max_smem_optin = 0;
    std::string last_error;
    uint32_t fail_alloc_in = 0;  // fault injection: fail the k-th allocation
    uint32_t wait_polls = 0;     // failure injection: look-back polls before giving up (0: kSpinLimit)
    uint32_t withhold = 0;       // failure injection: bit 0 / 1 skip the first compaction / count-scan tile
    mtx::Ctrl *ctrl = nullptr;   // device
    uint32_t *pinned = nullptr;  // pinned host words for count readbacks
    mtx::Scratch filter_status, count_status, faces, state, leaf, ids, rank, desc, misc;
    mtx::Scratch xface;  // leaf pass: the first column of every x-strip but the first, per block row and slab
    mtx::Scratch adj_partial, adj_iso;  // adjoint: per-block partial tiles and isovalue sums
    mtx_profiler *prof = nullptr;  // records stage times of calls given no profiler
    mtx_tuning tuning = {0, 0, 0, 0, 0};
    cudaStream_t copy_stream = nullptr;  // host-to-device slabs of mtx_upload_compute_min_max_mip (made on first use)
    // mtx_context_set_extract_stream: count/scan/emit of the async call on a second stream
    bool has_xstream = false;
    cudaStream_t xstream = nullptr;
    cudaEvent_t ev_filtered = nullptr;   // filter done on `stream` (the extraction may start)
    cudaEvent_t ev_extracted = nullptr;  // extraction done on `xstream` (the scratch is free again)
    bool extract_pending = false;        // ev_extracted recorded and not yet joined into `stream`
};

namespace mtx {

// ------------------------------------------------------------ helpers
// Makes `dev` current for the scope of a call and restores the caller's device.
struct DeviceGuard {
    int prev = -1;
    bool changed = false;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) changed = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        if (changed) cudaSetDevice(prev);
    }
};

mtx_status fail(mtx_context *c, mtx_status s, const std::string &msg);
mtx_status cuda_fail(mtx_context *c, cudaError_t e, const char *what);
#define MTX_CUDA(c, call)                                  \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
    } while (0)

mtx_status dev_alloc(mtx_context *c, void **p, size_t bytes);
void dev_free(mtx_context *c, void *p);  // ordered on c's stream (c may be null: a device-wide wait)
mtx_status scratch_reserve(mtx_context *c, Scratch &s, size_t bytes);
// Makes the context's stream wait for an extraction still running on its
// extraction stream (mtx_context_set_extract_stream); every entry point that
// queues work on the context or touches its scratch calls it first.
mtx_status join_extract(mtx_context *c);

inline uint32_t dtype_size(uint32_t dt) { return dt == MTX_DTYPE_U8 ? 1u : dt == MTX_DTYPE_U16 ? 2u : 4u; }
inline uint64_t nvox(const uint32_t d[3]) { return (uint64_t)d[0] * d[1] * d[2]; }
inline uint32_t ceil_div(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// The kernels' view of a volume, block edge and isovalue.
struct Problem;
Problem make_problem(const mtx_volume *v, uint32_t B, float iso);
// Profiler regions around the launches of a call (no-ops for a null profiler).
void prof_begin(mtx_profiler *p, const char *name, cudaStream_t s);
void prof_end(mtx_profiler *p, cudaStream_t s);

// Validate a volume + push constants pair (cubic block edge in [2, 16]).
mtx_status check_volume(mtx_context *c, const mtx_volume *v);
mtx_status check_pc(mtx_context *c, const mtx_volume *v, const mtx_push_constants *pc);

// Mip level layout of a block grid: 1 + floor(log2(max extent)) levels, ceil extents.
int mip_levels(const uint32_t grid[3]);
void mip_layout(const uint32_t grid[3], int levels, uint32_t ext[][3], uint64_t *offset, uint64_t *total);

// ------------------------------------------------------------ launches
// Geometry of one extraction problem as the kernels see it.
struct Problem {
    const void *vol;
    uint32_t X, Y, Z;
    uint32_t dtype;
    uint32_t B;            // cubic block edge
    uint32_t GX, GY, GZ;   // block grid
    uint64_t nblocks;
    float iso;
};

// Stage 1: leaf min/max (B+1 halo) into leaf[nblocks] (uint2 {min,max}).
// Given l1 and its extents, the TMA pass may also write octree level 1 there;
// *l1_done says whether it did.
mtx_status launch_minmax_leaf(mtx_context *c, const Problem &p, uint2 *leaf, cudaStream_t s,
                              uint32_t zchunk_override = 0, uint2 *l1 = nullptr, const uint32_t *l1ext = nullptr,
                              bool *l1_done = nullptr);
// Octree levels start+1.. from level start (already in all_levels at offset[start]).
mtx_status launch_pyramid(mtx_context *c, uint2 *all_levels, int levels, const uint32_t ext[][3],
                          const uint64_t *offset, cudaStream_t s, int start = 0);

// Stage 2: ordered compaction of active blocks.
//   ids[rank] = block id, rank_map[id] = rank (0xffffffff if inactive),
//   *count = number of active blocks.  count_status: optional per-rank words
//   to zero (pass null).
mtx_status launch_filter(mtx_context *c, const Problem &p, const uint2 *leaf, uint32_t *ids,
                         uint32_t *rank_map, uint32_t *count, uint64_t *count_status, cudaStream_t s);

// Stage 3: per-active-block counts and face records, the scan that fills the
// meshlet descriptors and totals (launch_count); then vertices and triangles
// (launch_emit).
struct ExtractArgs {
    const uint32_t *ids;
    const uint32_t *rank_map;
    const uint32_t *count;      // device: number of active blocks
    uint32_t host_count;        // > 0 when the host knows it (sizes the grid), else 0
    mtx_meshlet_descriptor *desc;  // per active block {vbase, 3*tbase, nv, nt}
    uint64_t desc_capacity;
    uint32_t *faces;            // 3*B*B words per active block
    uint8_t *state;             // block_state_bytes(B) per active block (count -> emit), B <= 8
    uint64_t block_capacity;    // active blocks that desc/faces/count_status can hold
    uint64_t *count_status;     // unused (the scan keeps its own look-back words)
    uint32_t *totals;           // device uint32[4] {vertexCount, indexCount, meshletCount, activeCount}
    uint8_t *cell_cases;        // optional
    void *vertices;             // vertex buffer written by the emit pass, or null
    uint64_t vertex_capacity;
    uint32_t *indices;
    uint64_t tri_capacity;
    uint32_t vertex_format, frame, normals, staging, threads;
};
mtx_status launch_count(mtx_context *c, const Problem &p, const ExtractArgs &a, cudaStream_t s);
// Bytes of the block state the count pass hands to the emit pass (0: none, B > 8).
uint32_t block_state_bytes(uint32_t B);
// The descriptor scan alone over *count descriptors (capacity bounds them).
mtx_status launch_desc_scan(mtx_context *c, mtx_meshlet_descriptor *desc, const uint32_t *count, uint64_t capacity,
                            uint32_t *totals, cudaStream_t s);
mtx_status launch_emit(mtx_context *c, const Problem &p, const ExtractArgs &a, cudaStream_t s);

// Whether the volume can be staged with TMA (row pitch and base 16-byte aligned).
bool tma_ok(const Problem &p);
// Build the 3D tensor map of the volume with a (bx, B+1, B+1) box.
mtx_status make_volume_tensor_map(mtx_context *c, const Problem &p, uint32_t box_x, CUtensorMap *map);
mtx_status make_volume_tensor_map_box(mtx_context *c, const Problem &p, uint32_t box_x, uint32_t box_y,
                                      uint32_t box_z, CUtensorMap *map);

}  // namespace mtx
