// Stage 2: active-block filtering with ordered stream compaction
// (meshtrex: occupiedBlockPrefixSum.comp.glsl:50-177, dispatched by
// activeBlockFilteringPass.cpp:87-153; CPU rule blockFilteringTestUtils.h:438-478).
//
// meshtrex scans within a workgroup and then takes one atomicAdd per
// workgroup, so the compacted list is ordered only inside a workgroup.  Here
// each CTA takes a tile of consecutive block ids by ticket (4096 a tile, 16
// per thread, so that a 1024^3 volume at block 8 is one wave of CTAs; 1024 in
// the no-allocation entry point, whose scratch is sized for them), counts its
// active blocks (warp scan + CTA scan), and resolves its global offset with a
// single-pass decoupled look-back over the tiles before it: the list comes out
// in ascending block order, which is the order the CPU rule produces.  It
// also writes the rank of every block (0xffffffff for inactive ones), which
// the extraction uses to find a neighbouring block's vertices.
#include <cstddef>
#include <mutex>

#include "mtx_internal.h"

namespace mtx {

constexpr int kFilterThreads = 256;
constexpr int kFilterItems = 16;       // blocks a thread: tiles of 4096
constexpr int kNoallocItems = 4;       // tiles of 1024 in mtx_filter_active_blocks_noalloc
constexpr int kFilterTile = kFilterThreads * kFilterItems;
constexpr int kNoallocTile = kFilterThreads * kNoallocItems;

// tile status word: [31:30] flag (0 empty, 1 aggregate, 2 inclusive, 3 aborted), [29:0] count
constexpr uint32_t kFlagAgg = 1u, kFlagInc = 2u, kFlagAbort = 3u;

template <int ITEMS>
__global__ void __launch_bounds__(kFilterThreads)
    filter_compact_kernel(const uint2 *__restrict__ leaf, uint64_t nblocks, uint32_t ntiles, uint32_t dtype,
                          float iso, uint32_t *__restrict__ ids, uint32_t *__restrict__ rank_map,
                          uint32_t *__restrict__ count_out, uint64_t *__restrict__ count_status,
                          uint32_t *tile_status, uint32_t *ticket, DevStatus *st, uint32_t spin_limit) {
    __shared__ uint32_t s_tile, s_prefix, s_abort;
    __shared__ uint32_t s_tmp[kFilterThreads / 32 + 1];
    if (threadIdx.x == 0) {
        s_tile = atomicAdd(ticket, 1u);
        s_abort = 0;
    }
    __syncthreads();
    const uint32_t t = s_tile;
    if (t >= ntiles) return;

    const uint64_t base = (uint64_t)t * (kFilterThreads * ITEMS) + (uint64_t)threadIdx.x * ITEMS;
    uint32_t f[ITEMS];
    if (base + ITEMS <= nblocks) {
        const uint4 *p = reinterpret_cast<const uint4 *>(leaf + base);
        uint4 v[ITEMS / 2];
#pragma unroll
        for (int i = 0; i < ITEMS / 2; ++i) v[i] = __ldg(p + i);  // all loads before any use
#pragma unroll
        for (int i = 0; i < ITEMS / 2; ++i) {
            f[2 * i] = block_active(dtype, v[i].x, v[i].y, iso);
            f[2 * i + 1] = block_active(dtype, v[i].z, v[i].w, iso);
        }
    } else {
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            f[i] = 0;
            if (base + i < nblocks) {
                uint2 v = leaf[base + i];
                f[i] = block_active(dtype, v.x, v.y, iso);
            }
        }
    }
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) c += f[i];
    uint32_t total;
    const uint32_t excl = cta_exclusive_scan<kFilterThreads>(c, s_tmp, &total);

    if (threadIdx.x < 32) {
        const uint32_t lane = threadIdx.x;
        uint32_t prefix = 0;
        bool abort = false;
        if (t == 0) {
            if (lane == 0) st_volatile(&tile_status[0], (kFlagInc << 30) | total);
        } else {
            if (lane == 0) st_volatile(&tile_status[t], (kFlagAgg << 30) | total);
            int64_t j = (int64_t)t - 1;
            uint32_t spins = 0;
            while (true) {
                const int64_t k = j - (int64_t)lane;
                const uint32_t w = k >= 0 ? ld_volatile(&tile_status[k]) : (kFlagInc << 30);
                const uint32_t flag = w >> 30;
                if (__any_sync(0xffffffffu, flag == kFlagAbort)) { abort = true; break; }
                const uint32_t inc = __ballot_sync(0xffffffffu, flag == kFlagInc);
                const uint32_t emp = __ballot_sync(0xffffffffu, flag == 0u);
                const uint32_t first = inc ? (uint32_t)(__ffs(inc) - 1) : 32u;
                const uint32_t window = first >= 31 ? 0xffffffffu : ((2u << first) - 1u);
                if (emp & window) {
                    if (++spins >= spin_limit) {
                        if (lane == 0) report(st, MTX_ERR_TIMEOUT, kSiteFilterLookback, t, (uint32_t)j);
                        abort = true;
                        break;
                    }
                    backoff(spins);
                    continue;
                }
                uint32_t v = lane <= first ? (w & 0x3fffffffu) : 0u;
#pragma unroll
                for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                prefix += v;
                if (first < 32) break;
                j -= 32;
            }
            if (lane == 0)
                st_volatile(&tile_status[t], abort ? (kFlagAbort << 30) : ((kFlagInc << 30) | (prefix + total)));
        }
        if (lane == 0) {
            s_prefix = prefix;
            s_abort = abort ? 1u : 0u;
        }
    }
    __syncthreads();
    if (s_abort) return;
    uint32_t r = s_prefix + excl;
    // rank of every block of the tile: its rank if active, else kNoRank
    uint32_t rk[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        rk[i] = 0xffffffffu;
        if (f[i] && MTX_BC(r, nblocks, kBcRank)) {
            const uint32_t id = (uint32_t)(base + i);
            ids[r] = id;
            rk[i] = r;
            if (count_status) count_status[r] = 0ull;
            ++r;
        }
    }
    if (base + ITEMS <= nblocks) {
#pragma unroll
        for (int i = 0; i < ITEMS / 4; ++i)
            reinterpret_cast<uint4 *>(rank_map + base)[i] = make_uint4(rk[4 * i], rk[4 * i + 1], rk[4 * i + 2],
                                                                       rk[4 * i + 3]);
    } else {
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (base + i < nblocks) rank_map[base + i] = rk[i];
    }
    if (t == ntiles - 1 && threadIdx.x == 0) *count_out = s_prefix + total;
}

MTX_BC_READER(bc_take_filter)

mtx_status launch_filter(mtx_context *c, const Problem &p, const uint2 *leaf, uint32_t *ids, uint32_t *rank_map,
                         uint32_t *count, uint64_t *count_status, cudaStream_t s) {
    if (p.nblocks >= (1ull << 30)) return fail(c, MTX_ERR_UNSUPPORTED, "more than 2^30 blocks");
    const uint32_t ntiles = (uint32_t)((p.nblocks + kFilterTile - 1) / kFilterTile);
    mtx_status rs = scratch_reserve(c, c->filter_status, sizeof(uint32_t) * (size_t)ntiles);
    if (rs != MTX_OK) return rs;
    MTX_CUDA(c, cudaMemsetAsync(c->filter_status.ptr, 0, sizeof(uint32_t) * (size_t)ntiles, s));
    if (count == &c->ctrl->active_count) {  // ticket, count ticket (reset by the count pass too) and count: one memset
        static_assert(offsetof(Ctrl, active_count) == offsetof(Ctrl, filter_ticket) + 8, "Ctrl layout");
        MTX_CUDA(c, cudaMemsetAsync(&c->ctrl->filter_ticket, 0, 3 * sizeof(uint32_t), s));
    } else {
        MTX_CUDA(c, cudaMemsetAsync(&c->ctrl->filter_ticket, 0, sizeof(uint32_t), s));
        MTX_CUDA(c, cudaMemsetAsync(count, 0, sizeof(uint32_t), s));
    }
    if (c->withhold & 1u) {  // failure injection: tile 0 is never handed out, so its successors wait and give up
        static const uint32_t kOne = 1;
        MTX_CUDA(c, cudaMemcpyAsync(&c->ctrl->filter_ticket, &kOne, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    }
    filter_compact_kernel<kFilterItems><<<ntiles, kFilterThreads, 0, s>>>(
        leaf, p.nblocks, ntiles, p.dtype, p.iso, ids, rank_map, count, count_status,
        (uint32_t *)c->filter_status.ptr, &c->ctrl->filter_ticket, &c->ctrl->status,
        c->wait_polls ? c->wait_polls : kSpinLimit);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "filter launch");
    return MTX_OK;
}

}  // namespace mtx

// ------------------------------------------------- compaction without allocation
// Some callers cannot allocate device memory while they run: an application
// with its own fixed device-memory budget, or code that runs where
// cudaMalloc is not allowed.  For them, mtx_filter_active_blocks_noalloc
// runs the same compaction kernel with its scratch (one look-back word per
// 1024-block tile and a ticket counter) in the statically sized array below
// instead of a context's arena.  The array lives in every GPU that loads the
// library until the process exits; it bounds the problem to
// kNoallocMaxTiles * 1024 blocks.  Calls that overlap on the GPU (two
// streams, two host threads) share the array and race: serialise them.
namespace mtx {
constexpr uint32_t kNoallocMaxTiles = 65536;                // up to 65536 * 1024 = 67,108,864 blocks
constexpr uint32_t kNoallocTicket = kNoallocMaxTiles;       // word index of the tile ticket
constexpr uint32_t kNoallocWords = kNoallocMaxTiles + 64;   // 256 KiB + 256 bytes
}  // namespace mtx

// Words [0, ntiles) hold the look-back status of each tile, then the ticket
// counter.
static __device__ __align__(256) uint32_t g_noalloc_scratch[mtx::kNoallocWords];

namespace {
// Device address of g_noalloc_scratch in the calling thread's current CUDA
// context.  Host code must not use the symbol itself as a pointer: on the
// host it names a stand-in object, not device memory.  The address belongs
// to the context that loaded the module, so it is cached per context id
// (cuCtxGetId, unique for the life of the process): after cudaDeviceReset,
// or under another context on the same device, the next call looks it up
// again instead of using a stale address.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);
struct NoallocSlot {
    unsigned long long ctx_id;
    uint32_t *ptr;
};
constexpr int kNoallocSlots = 64;
NoallocSlot g_noalloc_slots[kNoallocSlots] = {};
int g_noalloc_next = 0;
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
std::mutex g_noalloc_mu;

cudaError_t noalloc_scratch(int device, uint32_t **out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_ctx_get_current || !g_ctx_get_id) {
        void *f0 = nullptr, *f1 = nullptr;
        cudaDriverEntryPointQueryResult q0, q1;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0);
        if (e != cudaSuccess) return e;
        e = cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1);
        if (e != cudaSuccess) return e;
        if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
            return cudaErrorNotSupported;
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f0);
        g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f1);
    }
    CUcontext cu = nullptr;
    if (g_ctx_get_current(&cu) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
    if (!cu) {  // no context yet on this thread: bind the device's primary context, as a launch would
        const cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) return e;
        if (g_ctx_get_current(&cu) != CUDA_SUCCESS || !cu) return cudaErrorDeviceUninitialized;
    }
    unsigned long long id = 0;
    if (g_ctx_get_id(cu, &id) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
    for (const NoallocSlot &s : g_noalloc_slots)
        if (s.ptr && s.ctx_id == id) {
            *out = s.ptr;
            return cudaSuccess;
        }
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_slots[g_noalloc_next] = {id, static_cast<uint32_t *>(p)};
    g_noalloc_next = (g_noalloc_next + 1) % kNoallocSlots;
    *out = static_cast<uint32_t *>(p);
    return cudaSuccess;
}
}  // namespace

extern "C" mtx_status mtx_filter_active_blocks_noalloc(const uint32_t *leaf_minmax, uint64_t total_blocks,
                                                       uint32_t dtype, float isovalue, uint32_t *compacted_ids,
                                                       uint32_t *block_rank, uint32_t *active_count,
                                                       uint32_t *device_status, void *stream) {
    using namespace mtx;
    if (!leaf_minmax || !compacted_ids || !block_rank || !active_count || !device_status ||
        dtype > MTX_DTYPE_F32 || total_blocks == 0)
        return MTX_ERR_INVALID_ARG;
    // the kernel reads the keys and writes the ranks as 16-byte words
    if ((reinterpret_cast<uintptr_t>(leaf_minmax) | reinterpret_cast<uintptr_t>(block_rank)) % 16 != 0 ||
        reinterpret_cast<uintptr_t>(compacted_ids) % 4 != 0 || reinterpret_cast<uintptr_t>(active_count) % 4 != 0 ||
        reinterpret_cast<uintptr_t>(device_status) % 4 != 0)
        return MTX_ERR_INVALID_ARG;
    if (total_blocks > (uint64_t)kNoallocMaxTiles * kNoallocTile) return MTX_ERR_CAPACITY;
    const uint32_t ntiles = (uint32_t)((total_blocks + kNoallocTile - 1) / kNoallocTile);
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return MTX_ERR_NO_DEVICE;
    }
    uint32_t *sc = nullptr;
    if (noalloc_scratch(device, &sc) != cudaSuccess) {
        cudaGetLastError();
        return MTX_ERR_CUDA;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DevStatus *st = reinterpret_cast<DevStatus *>(device_status);
    // the array keeps the previous call's contents: clear what must start at zero
    if (cudaMemsetAsync(sc, 0, sizeof(uint32_t) * (size_t)ntiles, s) != cudaSuccess ||
        cudaMemsetAsync(sc + kNoallocTicket, 0, sizeof(uint32_t), s) != cudaSuccess ||
        cudaMemsetAsync(active_count, 0, sizeof(uint32_t), s) != cudaSuccess ||
        cudaMemsetAsync(device_status, 0, sizeof(DevStatus), s) != cudaSuccess) {
        cudaGetLastError();
        return MTX_ERR_CUDA;
    }
    filter_compact_kernel<kNoallocItems><<<ntiles, kFilterThreads, 0, s>>>(
        reinterpret_cast<const uint2 *>(leaf_minmax), total_blocks, ntiles, dtype, isovalue, compacted_ids, block_rank,
        active_count, nullptr, sc, sc + kNoallocTicket, st, kSpinLimit);
    if (cudaGetLastError() != cudaSuccess) return MTX_ERR_CUDA;
    return MTX_OK;
}
