// C ABI of libmeshtrex_b200: context, memory, the three stage calls, the
// asynchronous whole-path call and the stage profiler.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "mtx_internal.h"

using namespace mtx;

struct mtx_profiler {
    mtx_context *ctx = nullptr;
    struct Region {
        std::string name;
        double last_ms = 0, sum_ms = 0;
        uint32_t frames = 0;
    };
    struct Pending {
        int region;
        cudaEvent_t a, b;
    };
    std::vector<Region> regions;
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    int open_region = -1;
    cudaEvent_t open_a = nullptr;
};

namespace mtx {

// ----------------------------------------------------------------- errors
mtx_status fail(mtx_context *c, mtx_status s, const std::string &msg) {
    if (c) c->last_error = msg;
    return s;
}

mtx_status cuda_fail(mtx_context *c, cudaError_t e, const char *what) {
    cudaGetLastError();  // clear a sticky launch error where possible
    mtx_status s = (e == cudaErrorMemoryAllocation) ? MTX_ERR_OOM : MTX_ERR_CUDA;
    return fail(c, s, std::string(what) + ": " + cudaGetErrorString(e));
}

// ----------------------------------------------------------------- memory
// Freed device buffers are kept for reuse.  The drop-in stages allocate their
// outputs per call, as meshtrex's managers do, and cudaMalloc / cudaFree of
// the same sizes call after call cost host time: milliseconds for a 2 GiB
// volume, many more on a busy host.  Freeing is ordered on the freeing
// context's stream, as cudaFreeAsync is: the free records an event there and
// the buffer goes to a per-device list by exact size; an allocation of that
// size takes it back, and the taking context's stream waits for the event
// (no host wait) if the old work is still running.  So a free never stalls
// the device or the host, and work a caller queued on another stream that
// still reads the buffer must be finished, or ordered before the freeing
// context's stream, before the free call -- the contract of any
// stream-ordered allocator.  At most kCacheBytes and kCacheBuffers are kept
// per device; a failed cudaMalloc hands the device's cached buffers back to
// the driver (after their events) and tries again, and so does the
// destruction of a context (dev_cache_release).
namespace {
constexpr size_t kCacheBytes = 16ull << 30;
constexpr uint32_t kCacheBuffers = 64;
constexpr int kCacheDevices = 128;
struct LiveAlloc {
    int device;
    size_t bytes;
};
struct IdleBuf {
    void *ptr;
    cudaEvent_t freed;  // recorded on the freeing stream; null when the free waited already
};
std::mutex g_alloc_mu;
std::unordered_map<void *, LiveAlloc> g_live;                  // every buffer dev_alloc handed out
std::map<std::pair<int, size_t>, std::vector<IdleBuf>> g_idle;  // (device, bytes) -> freed buffers
size_t g_idle_bytes[kCacheDevices];
uint32_t g_idle_count[kCacheDevices];

bool take_idle(int device, size_t bytes, IdleBuf *out) {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    auto it = g_idle.find({device, bytes});
    if (it == g_idle.end() || it->second.empty()) return false;
    *out = it->second.back();
    it->second.pop_back();
    g_idle_bytes[device] -= bytes;
    --g_idle_count[device];
    return true;
}
}  // namespace

// Hands the freed buffers of `device` back to the driver (that device current).
void dev_cache_release(int device) {
    std::vector<IdleBuf> drop;
    {
        std::lock_guard<std::mutex> lk(g_alloc_mu);
        for (auto it = g_idle.begin(); it != g_idle.end();) {
            if (it->first.first == device) {
                for (const IdleBuf &b : it->second) {
                    drop.push_back(b);
                    g_live.erase(b.ptr);
                }
                it = g_idle.erase(it);
            } else {
                ++it;
            }
        }
        if (device >= 0 && device < kCacheDevices) {
            g_idle_bytes[device] = 0;
            g_idle_count[device] = 0;
        }
    }
    for (const IdleBuf &b : drop) {
        if (b.freed) {
            cudaEventSynchronize(b.freed);
            cudaEventDestroy(b.freed);
        }
        cudaFree(b.ptr);
    }
}

mtx_status dev_alloc(mtx_context *c, void **p, size_t bytes) {
    *p = nullptr;
    if (c->fail_alloc_in) {
        if (--c->fail_alloc_in == 0) return fail(c, MTX_ERR_OOM, "injected allocation failure");
    }
    if (bytes == 0) bytes = 16;
    const bool cached = c->device >= 0 && c->device < kCacheDevices;
    IdleBuf idle{nullptr, nullptr};
    if (cached && take_idle(c->device, bytes, &idle)) {
        if (idle.freed) {
            // the freeing stream's work must be done before this stream uses the buffer
            cudaError_t e = cudaEventQuery(idle.freed);
            if (e == cudaErrorNotReady) e = cudaStreamWaitEvent(c->stream, idle.freed, 0);
            cudaEventDestroy(idle.freed);
            if (e != cudaSuccess) {
                cudaGetLastError();
                cudaEventSynchronize(idle.freed);
            }
        }
        *p = idle.ptr;
        return MTX_OK;
    }
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess && cached) {
        cudaGetLastError();
        dev_cache_release(c->device);
        e = cudaMalloc(p, bytes);
    }
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(c, MTX_ERR_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
    }
    if (cached) {
        std::lock_guard<std::mutex> lk(g_alloc_mu);
        g_live[*p] = LiveAlloc{c->device, bytes};
    }
    return MTX_OK;
}

void dev_free(mtx_context *c, void *p) {
    if (!p) return;
    LiveAlloc a{-1, 0};
    {
        std::lock_guard<std::mutex> lk(g_alloc_mu);
        auto it = g_live.find(p);
        if (it != g_live.end()) a = it->second;
    }
    if (a.device < 0) {
        cudaFree(p);
        return;
    }
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != a.device) cudaSetDevice(a.device);
    // ordered on the freeing context's stream; without one, as cudaFree (the whole device)
    cudaEvent_t ev = nullptr;
    if (c && c->device == a.device) {
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventRecord(ev, c->stream) != cudaSuccess) {
            cudaGetLastError();
            if (ev) cudaEventDestroy(ev);
            ev = nullptr;
            cudaDeviceSynchronize();
        }
    } else {
        cudaDeviceSynchronize();
    }
    bool keep = false;
    {
        std::lock_guard<std::mutex> lk(g_alloc_mu);
        if (g_idle_bytes[a.device] + a.bytes <= kCacheBytes && g_idle_count[a.device] < kCacheBuffers) {
            g_idle[{a.device, a.bytes}].push_back(IdleBuf{p, ev});
            g_idle_bytes[a.device] += a.bytes;
            ++g_idle_count[a.device];
            keep = true;
        } else {
            g_live.erase(p);
        }
    }
    if (!keep) {
        if (ev) {
            cudaEventSynchronize(ev);
            cudaEventDestroy(ev);
        }
        cudaFree(p);
    }
    if (cur >= 0 && cur != a.device) cudaSetDevice(cur);
}

mtx_status scratch_reserve(mtx_context *c, Scratch &s, size_t bytes) {
    if (s.size >= bytes && s.ptr) return MTX_OK;
    // grow; the old block is released in the order of the stream, after any
    // extraction still reading it on the extraction stream
    if (s.ptr) {
        join_extract(c);
        dev_free(c, s.ptr);
        s.ptr = nullptr;
        s.size = 0;
    }
    size_t want = std::max(bytes, (size_t)256);
    mtx_status r = dev_alloc(c, &s.ptr, want);
    if (r != MTX_OK) return r;
    s.size = want;
    return MTX_OK;
}

mtx_status join_extract(mtx_context *c) {
    if (!c || !c->extract_pending) return MTX_OK;
    c->extract_pending = false;
    MTX_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_extracted, 0));
    return MTX_OK;
}

// ----------------------------------------------------------- validation
mtx_status check_volume(mtx_context *c, const mtx_volume *v) {
    if (!v || !v->data.ptr) return fail(c, MTX_ERR_INVALID_ARG, "volume is null");
    if (v->dtype > MTX_DTYPE_F32) return fail(c, MTX_ERR_INVALID_ARG, "unknown dtype");
    if (!v->dims[0] || !v->dims[1] || !v->dims[2]) return fail(c, MTX_ERR_INVALID_ARG, "zero volume extent");
    if (v->data.size && v->data.size < nvox(v->dims) * dtype_size(v->dtype))
        return fail(c, MTX_ERR_INVALID_ARG, "volume buffer smaller than its dims");
    return MTX_OK;
}

mtx_status check_pc(mtx_context *c, const mtx_volume *v, const mtx_push_constants *pc) {
    if (!pc) return fail(c, MTX_ERR_INVALID_ARG, "push constants are null");
    for (int a = 0; a < 3; ++a)
        if (pc->volumeDim[a] != v->dims[a])
            return fail(c, MTX_ERR_INVALID_ARG, "pushConstants.volumeDim differs from the volume");
    const uint32_t B = pc->blockDim[0];
    if (pc->blockDim[1] != B || pc->blockDim[2] != B)
        return fail(c, MTX_ERR_UNSUPPORTED, "only cubic blocks are supported");
    if (B < 2 || B > MTX_MAX_BLOCK_EDGE) return fail(c, MTX_ERR_UNSUPPORTED, "block edge must be in [2, 16]");
    for (int a = 0; a < 3; ++a)
        if (pc->blockGridDim[a] != ceil_div(v->dims[a], B))
            return fail(c, MTX_ERR_INVALID_ARG, "pushConstants.blockGridDim != ceil(volumeDim / blockDim)");
    return MTX_OK;
}

int mip_levels(const uint32_t g[3]) {
    uint32_t m = std::max(g[0], std::max(g[1], g[2]));
    int l = 1;
    while (m > 1) {
        m >>= 1;
        ++l;
    }
    return l;
}

void mip_layout(const uint32_t g[3], int levels, uint32_t ext[][3], uint64_t *offset, uint64_t *total) {
    uint64_t off = 0;
    for (int l = 0; l < levels; ++l) {
        for (int a = 0; a < 3; ++a) ext[l][a] = l == 0 ? g[a] : (ext[l - 1][a] + 1) / 2;
        offset[l] = off;
        off += (uint64_t)ext[l][0] * ext[l][1] * ext[l][2];
    }
    *total = off;
}

// ------------------------------------------------------------ tensor maps
mtx_status make_volume_tensor_map(mtx_context *c, const Problem &p, uint32_t box_x, CUtensorMap *map) {
    return make_volume_tensor_map_box(c, p, box_x, p.B + 1, p.B + 1, map);
}

mtx_status make_volume_tensor_map_box(mtx_context *c, const Problem &p, uint32_t box_x, uint32_t box_y,
                                      uint32_t box_z, CUtensorMap *map) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!encode) return fail(c, MTX_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    const uint32_t esz = dtype_size(p.dtype);
    CUtensorMapDataType dt = p.dtype == MTX_DTYPE_U8    ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                             : p.dtype == MTX_DTYPE_U16 ? CU_TENSOR_MAP_DATA_TYPE_UINT16
                                                        : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    cuuint64_t dims[3] = {p.X, p.Y, p.Z};
    cuuint64_t strides[2] = {(cuuint64_t)p.X * esz, (cuuint64_t)p.X * p.Y * esz};
    cuuint32_t box[3] = {box_x, box_y, box_z};
    cuuint32_t estr[3] = {1, 1, 1};
    if ((uintptr_t)p.vol % 16 || strides[0] % 16 || box_x > 256 || box_y > 256 || box_z > 256 || (box_x * esz) % 16)
        return fail(c, MTX_ERR_INTERNAL, "volume layout does not allow a TMA tile");
    CUresult r = encode(map, dt, 3, const_cast<void *>(p.vol), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(c, MTX_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return MTX_OK;
}

// ----------------------------------------------------------------- profiler
static cudaEvent_t prof_event(mtx_profiler *p) {
    if (!p->pool.empty()) {
        cudaEvent_t e = p->pool.back();
        p->pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void prof_begin(mtx_profiler *p, const char *name, cudaStream_t s) {
    if (!p) return;
    int id = -1;
    for (size_t i = 0; i < p->regions.size(); ++i)
        if (p->regions[i].name == name) id = (int)i;
    if (id < 0) {
        p->regions.push_back({name, 0, 0, 0});
        id = (int)p->regions.size() - 1;
    }
    p->open_region = id;
    p->open_a = prof_event(p);
    cudaEventRecord(p->open_a, s);
}

void prof_end(mtx_profiler *p, cudaStream_t s) {
    if (!p || p->open_region < 0) return;
    cudaEvent_t b = prof_event(p);
    cudaEventRecord(b, s);
    p->pending.push_back({p->open_region, p->open_a, b});
    p->open_region = -1;
    p->open_a = nullptr;
}

Problem make_problem(const mtx_volume *v, uint32_t B, float iso) {
    Problem p;
    p.vol = v->data.ptr;
    p.X = v->dims[0];
    p.Y = v->dims[1];
    p.Z = v->dims[2];
    p.dtype = v->dtype;
    p.B = B;
    p.GX = ceil_div(p.X, B);
    p.GY = ceil_div(p.Y, B);
    p.GZ = ceil_div(p.Z, B);
    p.nblocks = (uint64_t)p.GX * p.GY * p.GZ;
    p.iso = iso;
    return p;
}

#ifdef MTX_BOUNDS_CHECK
DevStatus bc_take_extract();
DevStatus bc_take_filter();
DevStatus bc_take_minmax();
DevStatus bc_take_batched();
DevStatus bc_take_adjoint();
#endif

static mtx_status check_device_status(mtx_context *c) {
#ifdef MTX_BOUNDS_CHECK
    // a bounds-check build: the translation units' check records first
    for (DevStatus b : {bc_take_extract(), bc_take_filter(), bc_take_minmax(), bc_take_batched(), bc_take_adjoint()})
        if (b.code) {
            char buf[160];
            snprintf(buf, sizeof(buf), "bounds check failed at site %u: index %u, bound %u", b.where, b.info0,
                     b.info1);
            return fail(c, MTX_ERR_INTERNAL, buf);
        }
#endif
    DevStatus h;
    MTX_CUDA(c, cudaMemcpy(&h, &c->ctrl->status, sizeof(h), cudaMemcpyDeviceToHost));
    if (h.code == 0) return MTX_OK;
    MTX_CUDA(c, cudaMemset(&c->ctrl->status, 0, sizeof(h)));
    char buf[160];
    snprintf(buf, sizeof(buf), "device error %u at site %u (info %u, %u)", h.code, h.where, h.info0, h.info1);
    return fail(c, (mtx_status)h.code, buf);
}

}  // namespace mtx

// ======================================================================= ABI
extern "C" {

const char *mtx_status_string(mtx_status s) {
    switch (s) {
    case MTX_OK: return "MTX_OK";
    case MTX_ERR_INVALID_ARG: return "MTX_ERR_INVALID_ARG";
    case MTX_ERR_UNSUPPORTED: return "MTX_ERR_UNSUPPORTED";
    case MTX_ERR_OOM: return "MTX_ERR_OOM";
    case MTX_ERR_CAPACITY: return "MTX_ERR_CAPACITY";
    case MTX_ERR_TIMEOUT: return "MTX_ERR_TIMEOUT";
    case MTX_ERR_CUDA: return "MTX_ERR_CUDA";
    case MTX_ERR_NO_DEVICE: return "MTX_ERR_NO_DEVICE";
    case MTX_ERR_INTERNAL: return "MTX_ERR_INTERNAL";
    }
    return "MTX_ERR_UNKNOWN";
}

uint32_t mtx_abi_version(void) { return MTX_ABI_VERSION; }

mtx_status mtx_context_create(int device, void *stream, mtx_context_t *out) {
    if (!out) return MTX_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return MTX_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return MTX_ERR_INVALID_ARG;
    mtx_context *c = new (std::nothrow) mtx_context();
    if (!c) return MTX_ERR_OOM;
    c->device = device;
    c->stream = (cudaStream_t)stream;
    DeviceGuard g(device);
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&c->max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (cudaMalloc(&c->ctrl, sizeof(Ctrl)) != cudaSuccess || cudaMemset(c->ctrl, 0, sizeof(Ctrl)) != cudaSuccess ||
        cudaMallocHost(&c->pinned, 64) != cudaSuccess) {
        cudaGetLastError();
        if (c->ctrl) cudaFree(c->ctrl);
        delete c;
        return MTX_ERR_OOM;
    }
    *out = c;
    return MTX_OK;
}

mtx_status mtx_context_destroy(mtx_context_t c) {
    if (!c) return MTX_ERR_INVALID_ARG;
    DeviceGuard g(c->device);
    join_extract(c);
    cudaStreamSynchronize(c->stream);
    for (Scratch *s : {&c->filter_status, &c->count_status, &c->faces, &c->state, &c->leaf, &c->ids, &c->rank,
                       &c->desc, &c->misc, &c->adj_partial, &c->adj_iso, &c->xface})
        dev_free(c, s->ptr);
    dev_cache_release(c->device);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->ev_filtered) cudaEventDestroy(c->ev_filtered);
    if (c->ev_extracted) cudaEventDestroy(c->ev_extracted);
    cudaFree(c->ctrl);
    cudaFreeHost(c->pinned);
    delete c;
    return MTX_OK;
}

mtx_status mtx_context_set_stream(mtx_context_t c, void *stream) {
    if (!c) return MTX_ERR_INVALID_ARG;
    DeviceGuard g(c->device);
    c->stream = (cudaStream_t)stream;
    return join_extract(c);  // the new stream waits for an extraction still in flight
}

mtx_status mtx_context_set_extract_stream(mtx_context_t c, void *stream) {
    if (!c) return MTX_ERR_INVALID_ARG;
    DeviceGuard g(c->device);
    join_extract(c);
    if (stream && !c->ev_filtered) {
        MTX_CUDA(c, cudaEventCreateWithFlags(&c->ev_filtered, cudaEventDisableTiming));
        MTX_CUDA(c, cudaEventCreateWithFlags(&c->ev_extracted, cudaEventDisableTiming));
    }
    c->xstream = (cudaStream_t)stream;
    c->has_xstream = stream != nullptr;
    return MTX_OK;
}

const char *mtx_context_last_error(mtx_context_t c) { return c ? c->last_error.c_str() : "null context"; }

mtx_status mtx_synchronize(mtx_context_t c) {
    if (!c) return MTX_ERR_INVALID_ARG;
    DeviceGuard g(c->device);
    join_extract(c);
    MTX_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_device_status(c);
}

mtx_status mtx_debug_fail_allocation(mtx_context_t c, uint32_t k) {
    if (!c) return MTX_ERR_INVALID_ARG;
    c->fail_alloc_in = k;
    return MTX_OK;
}

mtx_status mtx_debug_set_waits(mtx_context_t c, uint32_t max_polls, uint32_t withhold) {
    if (!c || withhold > 3u) return MTX_ERR_INVALID_ARG;
    c->wait_polls = max_polls;
    c->withhold = withhold;
    return MTX_OK;
}

// ------------------------------------------------------------------ volume
mtx_status mtx_volume_upload(mtx_context_t c, const void *host, const uint32_t dims[3], uint32_t dtype,
                             mtx_volume *out) {
    if (!c || !host || !dims || !out) return c ? fail(c, MTX_ERR_INVALID_ARG, "null argument") : MTX_ERR_INVALID_ARG;
    if (dtype > MTX_DTYPE_F32 || !dims[0] || !dims[1] || !dims[2]) return fail(c, MTX_ERR_INVALID_ARG, "bad volume");
    DeviceGuard g(c->device);
    join_extract(c);
    const uint64_t bytes = nvox(dims) * dtype_size(dtype);
    void *d = nullptr;
    mtx_status r = dev_alloc(c, &d, bytes);
    if (r != MTX_OK) return r;
    cudaError_t e = cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) {
        dev_free(c, d);
        return cuda_fail(c, e, "volume upload");
    }
    memset(out, 0, sizeof(*out));
    out->data.ptr = d;
    out->data.size = bytes;
    for (int a = 0; a < 3; ++a) out->dims[a] = dims[a];
    out->dtype = dtype;
    out->owned = 1;
    return MTX_OK;
}

mtx_status mtx_volume_wrap(void *device_ptr, const uint32_t dims[3], uint32_t dtype, mtx_volume *out) {
    if (!device_ptr || !dims || !out || dtype > MTX_DTYPE_F32 || !dims[0] || !dims[1] || !dims[2])
        return MTX_ERR_INVALID_ARG;
    memset(out, 0, sizeof(*out));
    out->data.ptr = device_ptr;
    out->data.size = nvox(dims) * dtype_size(dtype);
    for (int a = 0; a < 3; ++a) out->dims[a] = dims[a];
    out->dtype = dtype;
    out->owned = 0;
    return MTX_OK;
}

mtx_status mtx_volume_free(mtx_context_t c, mtx_volume *v) {
    if (!c || !v) return MTX_ERR_INVALID_ARG;
    DeviceGuard g(c->device);
    join_extract(c);
    if (v->owned && v->data.ptr) dev_free(c, v->data.ptr);
    memset(v, 0, sizeof(*v));
    return MTX_OK;
}

mtx_status mtx_push_constants_init(const uint32_t dims[3], uint32_t B, float iso, mtx_push_constants *out) {
    if (!dims || !out || !B) return MTX_ERR_INVALID_ARG;
    memset(out, 0, sizeof(*out));
    for (int a = 0; a < 3; ++a) {
        out->volumeDim[a] = dims[a];
        out->blockDim[a] = B;
        out->blockGridDim[a] = (dims[a] + B - 1) / B;
    }
    out->volumeDim[3] = out->blockDim[3] = out->blockGridDim[3] = 1;
    out->isovalue = iso;
    return MTX_OK;
}

float mtx_key_to_float(uint32_t dtype, uint32_t key) { return key_to_float(dtype, key); }

// ----------------------------------------------------------------- stage 1
mtx_status mtx_compute_min_max_mip(mtx_context_t c, const mtx_volume *vol, const mtx_push_constants *pc,
                                   mtx_profiler_t prof, mtx_minmax_output *out) {
    if (!c || !out) return MTX_ERR_INVALID_ARG;
    if (!prof) prof = c->prof;
    mtx_status r = check_volume(c, vol);
    if (r != MTX_OK) return r;
    if ((r = check_pc(c, vol, pc)) != MTX_OK) return r;
    DeviceGuard g(c->device);
    join_extract(c);
    memset(out, 0, sizeof(*out));
    const Problem p = make_problem(vol, pc->blockDim[0], pc->isovalue);
    const uint32_t grid[3] = {p.GX, p.GY, p.GZ};
    const int L = mip_levels(grid);
    if (L > MTX_MAX_MIP_LEVELS) return fail(c, MTX_ERR_UNSUPPORTED, "too many mip levels");
    uint64_t total = 0;
    mip_layout(grid, L, out->levelExtent, out->levelOffset, &total);
    void *mm = nullptr;
    if ((r = dev_alloc(c, &mm, total * sizeof(uint2))) != MTX_OK) return r;
    bool l1_done = false;
    prof_begin(prof, "MinMax_Leaf_Pass", c->stream);
    r = launch_minmax_leaf(c, p, (uint2 *)mm, c->stream, 0, L > 1 ? (uint2 *)mm + out->levelOffset[1] : nullptr,
                           out->levelExtent[1], &l1_done);
    prof_end(prof, c->stream);
    if (r == MTX_OK && L > 1) {
        prof_begin(prof, "MinMax_Octree_Reduction", c->stream);
        r = launch_pyramid(c, (uint2 *)mm, L, out->levelExtent, out->levelOffset, c->stream, l1_done ? 1 : 0);
        prof_end(prof, c->stream);
    }
    if (r != MTX_OK) {
        dev_free(c, mm);
        memset(out, 0, sizeof(*out));
        return r;
    }
    out->volumeImage = *vol;
    out->volumeImage.owned = 0;
    out->minMaxImage.ptr = mm;
    out->minMaxImage.size = total * sizeof(uint2);
    out->mipLevels = (uint32_t)L;
    for (int a = 0; a < 3; ++a) {
        out->blockDim[a] = pc->blockDim[a];
        out->blockGridDim[a] = grid[a];
    }
    return MTX_OK;
}

// Upload and leaf min/max overlapped (no meshtrex counterpart as one call:
// meshtrex stages the whole volume, then dispatches, minMaxManager.cpp:115-133).
// The volume goes to the device in slabs of S block layers on the context's
// copy stream; the leaf pass of slab k runs on the context's stream once
// slab k + 1 has landed (its first voxel slice is slab k's +z halo), as a
// sub-problem over block layers [k*S, (k+1)*S) of the same grid.  The octree
// follows the last slab.
mtx_status mtx_upload_compute_min_max_mip(mtx_context_t c, const void *host, const uint32_t dims[3], uint32_t dtype,
                                          const mtx_push_constants *pc, mtx_profiler_t prof, mtx_volume *vol_out,
                                          mtx_minmax_output *out) {
    if (!c || !host || !dims || !pc || !vol_out || !out)
        return c ? fail(c, MTX_ERR_INVALID_ARG, "null argument") : MTX_ERR_INVALID_ARG;
    if (dtype > MTX_DTYPE_F32 || !dims[0] || !dims[1] || !dims[2]) return fail(c, MTX_ERR_INVALID_ARG, "bad volume");
    if (!prof) prof = c->prof;
    DeviceGuard g(c->device);
    join_extract(c);
    memset(vol_out, 0, sizeof(*vol_out));
    memset(out, 0, sizeof(*out));
    mtx_volume v{};
    for (int a = 0; a < 3; ++a) v.dims[a] = dims[a];
    v.dtype = dtype;
    v.owned = 1;
    const uint64_t bytes = nvox(dims) * dtype_size(dtype);
    v.data.size = bytes;
    v.data.ptr = reinterpret_cast<void *>(uintptr_t(16));  // placeholder for the checks below
    mtx_status r = check_pc(c, &v, pc);
    if (r != MTX_OK) return r;
    if (!c->copy_stream) MTX_CUDA(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    const Problem p0 = make_problem(&v, pc->blockDim[0], pc->isovalue);
    const uint32_t grid[3] = {p0.GX, p0.GY, p0.GZ};
    const int L = mip_levels(grid);
    if (L > MTX_MAX_MIP_LEVELS) return fail(c, MTX_ERR_UNSUPPORTED, "too many mip levels");
    uint64_t total = 0;
    mip_layout(grid, L, out->levelExtent, out->levelOffset, &total);
    void *dv = nullptr, *mm = nullptr;
    if ((r = dev_alloc(c, &dv, bytes)) != MTX_OK) return r;
    if ((r = dev_alloc(c, &mm, total * sizeof(uint2))) != MTX_OK) {
        dev_free(c, dv);
        return r;
    }
    v.data.ptr = dv;
    // slabs of S block layers: about 16 of them, each copy tens of MB or more
    const uint32_t B = p0.B, S = std::max<uint32_t>(1, ceil_div(p0.GZ, 16));
    const uint32_t nslab = ceil_div(p0.GZ, S);
    const uint64_t slice = (uint64_t)dims[0] * dims[1] * dtype_size(dtype);
    std::vector<cudaEvent_t> landed(nslab, nullptr);
    cudaEvent_t ready = nullptr;
    auto cleanup = [&]() {
        for (cudaEvent_t e : landed)
            if (e) cudaEventDestroy(e);
        if (ready) cudaEventDestroy(ready);
    };
    auto bail = [&](mtx_status st) {
        cleanup();
        dev_free(c, mm);
        dev_free(c, dv);
        memset(out, 0, sizeof(*out));
        return st;
    };
    cudaError_t e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    // the copies may start only after what the context's stream owes the new buffers
    if (e == cudaSuccess) e = cudaEventRecord(ready, c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->copy_stream, ready, 0);
    for (uint32_t k = 0; k < nslab && e == cudaSuccess; ++k) {
        const uint64_t z0 = (uint64_t)k * S * B, z1 = std::min<uint64_t>((uint64_t)(k + 1) * S * B, dims[2]);
        e = cudaEventCreateWithFlags(&landed[k], cudaEventDisableTiming);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(static_cast<char *>(dv) + z0 * slice, static_cast<const char *>(host) + z0 * slice,
                                (z1 - z0) * slice, cudaMemcpyHostToDevice, c->copy_stream);
        if (e == cudaSuccess) e = cudaEventRecord(landed[k], c->copy_stream);
    }
    if (e != cudaSuccess) return bail(cuda_fail(c, e, "volume slab upload"));
    prof_begin(prof, "MinMax_Leaf_Pass", c->stream);
    for (uint32_t k = 0; k < nslab && r == MTX_OK; ++k) {
        e = cudaStreamWaitEvent(c->stream, landed[std::min(k + 1, nslab - 1)], 0);
        if (e != cudaSuccess) {
            r = cuda_fail(c, e, "slab wait");
            break;
        }
        const uint32_t b0 = k * S, b1 = std::min(p0.GZ, b0 + S);
        Problem ps = p0;
        ps.vol = static_cast<const char *>(dv) + (uint64_t)b0 * B * slice;
        ps.Z = (uint32_t)(std::min<uint64_t>((uint64_t)b1 * B + 1, dims[2]) - (uint64_t)b0 * B);
        ps.GZ = b1 - b0;
        ps.nblocks = (uint64_t)p0.GX * p0.GY * ps.GZ;
        r = launch_minmax_leaf(c, ps, (uint2 *)mm + (uint64_t)b0 * p0.GX * p0.GY, c->stream, 0);
    }
    prof_end(prof, c->stream);
    if (r == MTX_OK && L > 1) {
        prof_begin(prof, "MinMax_Octree_Reduction", c->stream);
        r = launch_pyramid(c, (uint2 *)mm, L, out->levelExtent, out->levelOffset, c->stream, 0);
        prof_end(prof, c->stream);
    }
    if (r != MTX_OK) return bail(r);
    cleanup();  // events are released once their work completes
    *vol_out = v;
    out->volumeImage = v;
    out->volumeImage.owned = 0;
    out->minMaxImage.ptr = mm;
    out->minMaxImage.size = total * sizeof(uint2);
    out->mipLevels = (uint32_t)L;
    for (int a = 0; a < 3; ++a) {
        out->blockDim[a] = pc->blockDim[a];
        out->blockGridDim[a] = grid[a];
    }
    return MTX_OK;
}

mtx_status mtx_minmax_free(mtx_context_t c, mtx_minmax_output *mm) {
    if (!c || !mm) return MTX_ERR_INVALID_ARG;
    DeviceGuard g(c->device);
    join_extract(c);
    dev_free(c, mm->minMaxImage.ptr);
    memset(mm, 0, sizeof(*mm));
    return MTX_OK;
}

// ----------------------------------------------------------------- stage 2
mtx_status mtx_filter_active_blocks(mtx_context_t c, const mtx_minmax_output *mm, const mtx_push_constants *pc,
                                    mtx_profiler_t prof, mtx_filtering_output *out) {
    if (!c || !mm || !out || !mm->minMaxImage.ptr) return c ? fail(c, MTX_ERR_INVALID_ARG, "null argument") : MTX_ERR_INVALID_ARG;
    if (!prof) prof = c->prof;
    mtx_status r = check_pc(c, &mm->volumeImage, pc);
    if (r != MTX_OK) return r;
    DeviceGuard g(c->device);
    join_extract(c);
    memset(out, 0, sizeof(*out));
    const Problem p = make_problem(&mm->volumeImage, pc->blockDim[0], pc->isovalue);
    void *ids = nullptr, *cnt = nullptr, *rank = nullptr;
    if ((r = dev_alloc(c, &ids, p.nblocks * 4)) != MTX_OK) return r;
    if ((r = dev_alloc(c, &cnt, 4)) != MTX_OK || (r = dev_alloc(c, &rank, p.nblocks * 4)) != MTX_OK) {
        dev_free(c, ids);
        dev_free(c, cnt);
        return r;
    }
    prof_begin(prof, "Active_Block_Filtering", c->stream);
    r = launch_filter(c, p, (const uint2 *)mm->minMaxImage.ptr, (uint32_t *)ids, (uint32_t *)rank, (uint32_t *)cnt,
                      nullptr, c->stream);
    prof_end(prof, c->stream);
    if (r != MTX_OK) {
        dev_free(c, ids);
        dev_free(c, cnt);
        dev_free(c, rank);
        return r;
    }
    out->compactedBlockIdBuffer = {ids, p.nblocks * 4};
    out->activeBlockCountBuffer = {cnt, 4};
    out->blockRankBuffer = {rank, p.nblocks * 4};
    out->activeBlockCount = 0;  // stays on the GPU until read (filteringManager.cpp:123-125)
    out->totalBlocks = (uint32_t)p.nblocks;
    out->isovalue = pc->isovalue;
    return MTX_OK;
}

mtx_status mtx_read_active_block_count(mtx_context_t c, mtx_filtering_output *f) {
    if (!c || !f || !f->activeBlockCountBuffer.ptr) return MTX_ERR_INVALID_ARG;
    DeviceGuard g(c->device);
    join_extract(c);
    MTX_CUDA(c, cudaMemcpyAsync(c->pinned, f->activeBlockCountBuffer.ptr, 4, cudaMemcpyDeviceToHost, c->stream));
    MTX_CUDA(c, cudaStreamSynchronize(c->stream));
    mtx_status r = check_device_status(c);
    if (r != MTX_OK) return r;
    f->activeBlockCount = c->pinned[0];
    return MTX_OK;
}

mtx_status mtx_read_buffer(mtx_context_t c, const mtx_buffer *src, uint64_t offset, void *host, uint64_t bytes) {
    if (!c || !src || (bytes && (!src->ptr || !host))) return c ? fail(c, MTX_ERR_INVALID_ARG, "null argument") : MTX_ERR_INVALID_ARG;
    if (offset > src->size || bytes > src->size - offset) return fail(c, MTX_ERR_INVALID_ARG, "read past the buffer");
    if (!bytes) return MTX_OK;
    DeviceGuard g(c->device);
    join_extract(c);
    MTX_CUDA(c, cudaMemcpyAsync(host, (const char *)src->ptr + offset, bytes, cudaMemcpyDeviceToHost, c->stream));
    MTX_CUDA(c, cudaStreamSynchronize(c->stream));
    return MTX_OK;
}

mtx_status mtx_filtering_free(mtx_context_t c, mtx_filtering_output *f) {
    if (!c || !f) return MTX_ERR_INVALID_ARG;
    DeviceGuard g(c->device);
    join_extract(c);
    dev_free(c, f->compactedBlockIdBuffer.ptr);
    dev_free(c, f->activeBlockCountBuffer.ptr);
    dev_free(c, f->blockRankBuffer.ptr);
    memset(f, 0, sizeof(*f));
    return MTX_OK;
}

// ----------------------------------------------------------------- stage 3
static mtx_extract_options default_opts(const mtx_extract_options *o) {
    mtx_extract_options d;
    memset(&d, 0, sizeof(d));
    if (o) d = *o;
    return d;
}

mtx_status mtx_extract_meshlet_descriptors(mtx_context_t c, const mtx_minmax_output *mm,
                                           const mtx_filtering_output *f, const mtx_push_constants *pc,
                                           const mtx_extract_options *opts_in, mtx_profiler_t prof,
                                           mtx_extraction_output *out) {
    if (!c || !mm || !f || !out) return c ? fail(c, MTX_ERR_INVALID_ARG, "null argument") : MTX_ERR_INVALID_ARG;
    if (!prof) prof = c->prof;
    mtx_status r = check_pc(c, &mm->volumeImage, pc);
    if (r != MTX_OK) return r;
    DeviceGuard g(c->device);
    join_extract(c);
    memset(out, 0, sizeof(*out));
    const mtx_extract_options o = default_opts(opts_in);
    if (o.vertexFormat > MTX_VERTEX_DATA || o.frame > MTX_FRAME_NDC || o.staging > MTX_STAGING_LDG)
        return fail(c, MTX_ERR_INVALID_ARG, "bad extract options");
    out->vertexStride = o.vertexFormat == MTX_VERTEX_XYZ ? 12 : 32;
    const uint32_t n = f->activeBlockCount;
    if (n == 0) return MTX_OK;  // extractionManager.cpp:253-256
    if (!f->compactedBlockIdBuffer.ptr || !f->blockRankBuffer.ptr || n > f->totalBlocks)
        return fail(c, MTX_ERR_INVALID_ARG, "filtering output is incomplete");
    const Problem p = make_problem(&mm->volumeImage, pc->blockDim[0], pc->isovalue);
    const uint32_t B = p.B;

    void *desc = nullptr, *counters = nullptr;
    if ((r = dev_alloc(c, &desc, (size_t)n * sizeof(mtx_meshlet_descriptor))) != MTX_OK) return r;
    if ((r = dev_alloc(c, &counters, 16)) != MTX_OK) {
        dev_free(c, desc);
        return r;
    }
    auto bail = [&](mtx_status s) {
        dev_free(c, desc);
        dev_free(c, counters);
        dev_free(c, out->vertexBuffer.ptr);
        dev_free(c, out->indexBuffer.ptr);
        memset(out, 0, sizeof(*out));
        return s;
    };
    if ((r = scratch_reserve(c, c->faces, (size_t)n * 3 * B * B * 4)) != MTX_OK) return bail(r);
    const uint32_t sb = block_state_bytes(B);
    if (sb && (r = scratch_reserve(c, c->state, (size_t)n * sb)) != MTX_OK) return bail(r);

    ExtractArgs a;
    memset(&a, 0, sizeof(a));
    a.ids = (const uint32_t *)f->compactedBlockIdBuffer.ptr;
    a.rank_map = (const uint32_t *)f->blockRankBuffer.ptr;
    a.count = (const uint32_t *)f->activeBlockCountBuffer.ptr;
    a.host_count = n;
    a.desc = (mtx_meshlet_descriptor *)desc;
    a.desc_capacity = n;
    a.block_capacity = n;
    a.faces = (uint32_t *)c->faces.ptr;
    a.state = sb ? (uint8_t *)c->state.ptr : nullptr;
    a.count_status = (uint64_t *)c->count_status.ptr;
    a.totals = (uint32_t *)counters;
    a.cell_cases = o.cellCases;
    a.vertex_format = o.vertexFormat;
    a.frame = o.frame;
    a.normals = o.normals;
    a.staging = o.staging;
    a.threads = o.threads;

    prof_begin(prof, "Mesh_Extraction", c->stream);
    r = launch_count(c, p, a, c->stream);
    prof_end(prof, c->stream);
    if (r != MTX_OK) return bail(r);
    // exact output sizes: one 8-byte readback instead of worst-case buffers
    cudaError_t e = cudaMemcpyAsync(c->pinned, counters, 8, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return bail(cuda_fail(c, e, "count readback"));
    if ((r = check_device_status(c)) != MTX_OK) return bail(r);
    const uint32_t V = c->pinned[0], I = c->pinned[1];
    void *vb = nullptr, *ib = nullptr;
    if ((r = dev_alloc(c, &vb, (size_t)V * out->vertexStride)) != MTX_OK) return bail(r);
    out->vertexBuffer = {vb, (uint64_t)V * out->vertexStride};
    if ((r = dev_alloc(c, &ib, (size_t)I * 4)) != MTX_OK) return bail(r);
    out->indexBuffer = {ib, (uint64_t)I * 4};
    a.vertices = vb;  // sizes are known only now
    a.vertex_capacity = V;
    a.indices = (uint32_t *)ib;
    a.tri_capacity = I / 3;
    prof_begin(prof, "Mesh_Extraction", c->stream);
    r = launch_emit(c, p, a, c->stream);
    prof_end(prof, c->stream);
    if (r != MTX_OK) return bail(r);

    out->vertexCountBuffer = {counters, 4};
    out->indexCountBuffer = {(char *)counters + 4, 4};
    out->meshletDescriptorCountBuffer = {(char *)counters + 8, 4};
    out->meshletDescriptorBuffer = {desc, (uint64_t)n * sizeof(mtx_meshlet_descriptor)};
    out->meshletCount = n;
    out->vertexCount = V;
    out->indexCount = I;
    return MTX_OK;
}

mtx_status mtx_extraction_free(mtx_context_t c, mtx_extraction_output *x) {
    if (!c || !x) return MTX_ERR_INVALID_ARG;
    DeviceGuard g(c->device);
    join_extract(c);
    dev_free(c, x->vertexBuffer.ptr);
    dev_free(c, x->indexBuffer.ptr);
    dev_free(c, x->meshletDescriptorBuffer.ptr);
    dev_free(c, x->vertexCountBuffer.ptr);  // the three counters share one allocation
    const uint32_t stride = x->vertexStride;
    memset(x, 0, sizeof(*x));
    x->vertexStride = stride;
    return MTX_OK;
}

// ---------------------------------------------------------- whole path
mtx_status mtx_extract_plain_async(mtx_context_t c, const mtx_volume *vol, const mtx_push_constants *pc,
                                   const mtx_extract_options *opts_in, const mtx_mesh_buffers *out) {
    if (!c || !out || !out->counters) return c ? fail(c, MTX_ERR_INVALID_ARG, "null argument") : MTX_ERR_INVALID_ARG;
    mtx_status r = check_volume(c, vol);
    if (r != MTX_OK) return r;
    if ((r = check_pc(c, vol, pc)) != MTX_OK) return r;
    const mtx_extract_options o = default_opts(opts_in);
    if (o.vertexFormat > MTX_VERTEX_DATA || o.frame > MTX_FRAME_NDC || o.staging > MTX_STAGING_LDG)
        return fail(c, MTX_ERR_INVALID_ARG, "bad extract options");
    if ((out->vertexCapacity && !out->vertices) || (out->triangleCapacity && !out->indices))
        return fail(c, MTX_ERR_INVALID_ARG, "capacity without a buffer");
    DeviceGuard g(c->device);
    const Problem p = make_problem(vol, pc->blockDim[0], pc->isovalue);
    const uint64_t maxa = out->maxActiveBlocks ? std::min<uint64_t>(out->maxActiveBlocks, p.nblocks) : p.nblocks;
    const uint32_t B = p.B;
    const uint32_t grid[3] = {p.GX, p.GY, p.GZ};
    const int L = mip_levels(grid);
    if (L > MTX_MAX_MIP_LEVELS) return fail(c, MTX_ERR_UNSUPPORTED, "too many mip levels");
    uint32_t ext[MTX_MAX_MIP_LEVELS][3];
    uint64_t off[MTX_MAX_MIP_LEVELS], texels = 0;
    mip_layout(grid, L, ext, off, &texels);
    if ((r = scratch_reserve(c, c->leaf, texels * 8)) != MTX_OK) return r;
    if ((r = scratch_reserve(c, c->ids, p.nblocks * 4)) != MTX_OK) return r;
    if ((r = scratch_reserve(c, c->rank, p.nblocks * 4)) != MTX_OK) return r;
    if ((r = scratch_reserve(c, c->faces, maxa * 3 * B * B * 4)) != MTX_OK) return r;
    const uint32_t sb = block_state_bytes(B);
    if (sb && (r = scratch_reserve(c, c->state, maxa * sb)) != MTX_OK) return r;
    mtx_meshlet_descriptor *desc = out->meshlets;
    uint64_t dcap = out->meshletCapacity;
    if (!desc || dcap < maxa) {
        if ((r = scratch_reserve(c, c->desc, maxa * sizeof(mtx_meshlet_descriptor))) != MTX_OK) return r;
        desc = (mtx_meshlet_descriptor *)c->desc.ptr;
        dcap = maxa;
    }
    cudaStream_t s = c->stream;
    mtx_profiler *P = c->prof;
    bool l1_done = false;
    prof_begin(P, "MinMax_Leaf_Pass", s);
    r = launch_minmax_leaf(c, p, (uint2 *)c->leaf.ptr, s, 0, L > 1 ? (uint2 *)c->leaf.ptr + off[1] : nullptr, ext[1],
                           &l1_done);
    prof_end(P, s);
    if (r != MTX_OK) return r;
    if (L > 1) {
        prof_begin(P, "MinMax_Octree_Reduction", s);
        r = launch_pyramid(c, (uint2 *)c->leaf.ptr, L, ext, off, s, l1_done ? 1 : 0);
        prof_end(P, s);
        if (r != MTX_OK) return r;
    }
    // the filter overwrites the ids, ranks and count a previous call's extraction may still read
    if ((r = join_extract(c)) != MTX_OK) return r;
    prof_begin(P, "Active_Block_Filtering", s);
    r = launch_filter(c, p, (const uint2 *)c->leaf.ptr, (uint32_t *)c->ids.ptr, (uint32_t *)c->rank.ptr,
                      &c->ctrl->active_count, nullptr, s);
    prof_end(P, s);
    if (r != MTX_OK) return r;
    cudaStream_t es = s;  // the extraction passes' stream
    if (c->has_xstream) {
        es = c->xstream;
        MTX_CUDA(c, cudaEventRecord(c->ev_filtered, s));
        MTX_CUDA(c, cudaStreamWaitEvent(es, c->ev_filtered, 0));
    }
    ExtractArgs a;
    memset(&a, 0, sizeof(a));
    a.ids = (const uint32_t *)c->ids.ptr;
    a.rank_map = (const uint32_t *)c->rank.ptr;
    a.count = &c->ctrl->active_count;
    a.host_count = 0;
    a.desc = desc;
    a.desc_capacity = dcap;
    a.block_capacity = maxa;
    a.faces = (uint32_t *)c->faces.ptr;
    a.state = sb ? (uint8_t *)c->state.ptr : nullptr;
    a.count_status = (uint64_t *)c->count_status.ptr;
    a.totals = out->counters;
    a.cell_cases = o.cellCases;
    a.vertices = out->vertices;
    a.vertex_capacity = out->vertexCapacity;
    a.indices = out->indices;
    a.tri_capacity = out->triangleCapacity;
    a.vertex_format = o.vertexFormat;
    a.frame = o.frame;
    a.normals = o.normals;
    a.staging = o.staging;
    a.threads = o.threads;
    prof_begin(P, "Mesh_Extraction_Count", es);
    r = launch_count(c, p, a, es);
    prof_end(P, es);
    if (r != MTX_OK) return r;
    prof_begin(P, "Mesh_Extraction_Emit", es);
    r = launch_emit(c, p, a, es);
    prof_end(P, es);
    if (r != MTX_OK) return r;
    if (desc != out->meshlets && out->meshlets && out->meshletCapacity) {
        // the caller's descriptor buffer was too small for the bound: copy what fits
        MTX_CUDA(c, cudaMemcpyAsync(out->meshlets, desc, out->meshletCapacity * sizeof(mtx_meshlet_descriptor),
                                    cudaMemcpyDeviceToDevice, es));
    }
    MTX_CUDA(c, cudaMemcpyAsync(out->counters + 4, &c->ctrl->status.code, 4, cudaMemcpyDeviceToDevice, es));
    if (c->has_xstream) {
        MTX_CUDA(c, cudaEventRecord(c->ev_extracted, es));
        c->extract_pending = true;
    }
    return MTX_OK;
}

// ----------------------------------------------------------------- profiler
mtx_status mtx_profiler_create(mtx_context_t c, mtx_profiler_t *out) {
    if (!c || !out) return MTX_ERR_INVALID_ARG;
    mtx_profiler *p = new (std::nothrow) mtx_profiler();
    if (!p) return MTX_ERR_OOM;
    p->ctx = c;
    *out = p;
    return MTX_OK;
}

mtx_status mtx_context_set_tuning(mtx_context_t c, const mtx_tuning *t) {
    if (!c || !t) return MTX_ERR_INVALID_ARG;
    if (t->minmaxSlices > 4 || t->minmaxSlices == 3 || t->staging > MTX_STAGING_LDG ||
        (t->extractWarps && t->extractWarps != 1 && t->extractWarps != 2 && t->extractWarps != 4 &&
         t->extractWarps != 8))
        return fail(c, MTX_ERR_INVALID_ARG, "bad tuning values");
    c->tuning = *t;
    return MTX_OK;
}

mtx_status mtx_context_get_tuning(mtx_context_t c, mtx_tuning *t) {
    if (!c || !t) return MTX_ERR_INVALID_ARG;
    *t = c->tuning;
    return MTX_OK;
}

mtx_status mtx_context_set_profiler(mtx_context_t c, mtx_profiler_t p) {
    if (!c) return MTX_ERR_INVALID_ARG;
    c->prof = p;
    return MTX_OK;
}

mtx_status mtx_profiler_destroy(mtx_profiler_t p) {
    if (!p) return MTX_ERR_INVALID_ARG;
    if (p->ctx && p->ctx->prof == p) p->ctx->prof = nullptr;
    DeviceGuard g(p->ctx->device);
    for (auto &q : p->pending) {
        cudaEventDestroy(q.a);
        cudaEventDestroy(q.b);
    }
    for (auto e : p->pool) cudaEventDestroy(e);
    delete p;
    return MTX_OK;
}

mtx_status mtx_profiler_begin_frame(mtx_profiler_t p) {
    if (!p) return MTX_ERR_INVALID_ARG;
    return MTX_OK;
}

mtx_status mtx_profiler_end_frame(mtx_profiler_t p) {
    if (!p) return MTX_ERR_INVALID_ARG;
    DeviceGuard g(p->ctx->device);
    std::vector<double> frame(p->regions.size(), 0.0);
    std::vector<bool> seen(p->regions.size(), false);
    for (auto &q : p->pending) {
        float ms = 0;
        if (cudaEventSynchronize(q.b) != cudaSuccess || cudaEventElapsedTime(&ms, q.a, q.b) != cudaSuccess) {
            cudaGetLastError();
            ms = 0;
        }
        frame[q.region] += ms;
        seen[q.region] = true;
        p->pool.push_back(q.a);
        p->pool.push_back(q.b);
    }
    p->pending.clear();
    for (size_t i = 0; i < p->regions.size(); ++i)
        if (seen[i]) {
            p->regions[i].last_ms = frame[i];
            p->regions[i].sum_ms += frame[i];
            p->regions[i].frames += 1;
        }
    return MTX_OK;
}

uint32_t mtx_profiler_region_count(mtx_profiler_t p) { return p ? (uint32_t)p->regions.size() : 0u; }

mtx_status mtx_profiler_region(mtx_profiler_t p, uint32_t i, char name[64], double *last_ms, double *avg_ms,
                               uint32_t *frames) {
    if (!p || i >= p->regions.size()) return MTX_ERR_INVALID_ARG;
    const auto &r = p->regions[i];
    if (name) {
        strncpy(name, r.name.c_str(), 63);
        name[63] = 0;
    }
    if (last_ms) *last_ms = r.last_ms;
    if (avg_ms) *avg_ms = r.frames ? r.sum_ms / r.frames : 0.0;
    if (frames) *frames = r.frames;
    return MTX_OK;
}

mtx_status mtx_profiler_export_csv(mtx_profiler_t p, const char *path) {
    if (!p || !path) return MTX_ERR_INVALID_ARG;
    FILE *f = fopen(path, "w");
    if (!f) return fail(p->ctx, MTX_ERR_INVALID_ARG, std::string("cannot write ") + path);
    fprintf(f, "Stage,Last (ms),Average (ms),Frames\n");
    for (const auto &r : p->regions)
        fprintf(f, "%s,%.6f,%.6f,%u\n", r.name.c_str(), r.last_ms, r.frames ? r.sum_ms / r.frames : 0.0, r.frames);
    fclose(f);
    return MTX_OK;
}

}  // extern "C"
