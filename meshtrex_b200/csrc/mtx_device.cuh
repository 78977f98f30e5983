// Device-side building blocks shared by the kernels: voxel keys, the device
// error word, bounded waits, TMA/mbarrier wrappers and CTA scans.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "mc_case_table.h"

namespace mtx {

// ------------------------------------------------------------ error word
// One per context, in device memory.  The first error a kernel records wins;
// the host reads and clears it in mtx_synchronize.
struct DevStatus {
    uint32_t code;   // mtx_status
    uint32_t where;  // kernel-specific site id
    uint32_t info0;
    uint32_t info1;
};

enum : uint32_t {
    kSiteFilterLookback = 1,
    kSiteCountLookback = 2,
    kSiteTmaWait = 3,
    kSiteEmitCapacity = 4,
    kSiteEmitNeighbour = 5,
    kSiteCountOverflow = 6,
    kSiteBatched = 7,
    kSiteAdjoint = 8,
    kSiteMinMaxTma = 9,
};

__device__ __forceinline__ void report(DevStatus *st, uint32_t code, uint32_t where, uint32_t i0 = 0,
                                       uint32_t i1 = 0) {
    if (st && atomicCAS(&st->code, 0u, code) == 0u) {
        st->where = where;
        st->info0 = i0;
        st->info1 = i1;
    }
}

// ----------------------------------------------------------- bounds checks
// A debug build of the library (-DMTX_BOUNDS_CHECK, `make check`) checks the
// shared- and global-memory indices of the extraction kernels: an index
// outside its range is recorded in the translation unit's check record
// (site, index, bound), the access is skipped, and mtx_synchronize reports
// the record as MTX_ERR_INTERNAL.  There is no trap.  In the normal build
// MTX_BC is the constant true and the checks compile away.
enum : uint32_t {
    kBcTile = 101,      // voxel tile in shared memory
    kBcRows = 102,      // inside masks, crossing rows, prefixes, case bytes, mixed masks
    kBcJobs = 103,      // job window
    kBcVertex = 104,    // vertex buffer
    kBcIndex = 105,     // index buffer
    kBcFaces = 106,     // face records (read and write)
    kBcContext = 107,   // context layer (neighbour ids and masks)
    kBcVoxTab = 108,    // voxel table
    kBcState = 109,     // block state
    kBcRank = 110,      // rank map and compacted ids
    kBcLeaf = 111,      // min/max leaf level
    kBcDesc = 112,      // meshlet descriptors
};
#ifdef MTX_BOUNDS_CHECK
static __device__ DevStatus g_bc_record;
__device__ __forceinline__ bool bc_ok(uint64_t i, uint64_t n, uint32_t site) {
    if (i < n) return true;
    if (atomicCAS(&g_bc_record.code, 0u, (uint32_t)MTX_ERR_INTERNAL) == 0u) {
        g_bc_record.where = site;
        g_bc_record.info0 = (uint32_t)i;
        g_bc_record.info1 = (uint32_t)n;
    }
    return false;
}
#define MTX_BC(i, n, site) ::mtx::bc_ok((uint64_t)(i), (uint64_t)(n), (site))
// Defines the host reader of this translation unit's check record: it copies
// the record out, clears it and returns it.
#define MTX_BC_READER(name)                                                        \
    ::mtx::DevStatus name() {                                                      \
        ::mtx::DevStatus h{}, z{};                                                 \
        if (cudaMemcpyFromSymbol(&h, ::mtx::g_bc_record, sizeof(h)) != cudaSuccess) \
            cudaGetLastError();                                                    \
        else if (h.code)                                                           \
            cudaMemcpyToSymbol(::mtx::g_bc_record, &z, sizeof(z));                 \
        return h;                                                                  \
    }
#else
#define MTX_BC(i, n, site) true
#define MTX_BC_READER(name)
#endif

__device__ __forceinline__ bool failed(const DevStatus *st) {
    return st && *(volatile const uint32_t *)&st->code != 0u;
}

// Bounded waits: about 2^22 polls with a growing back-off, well over a second
// on B200, after which the waiter records MTX_ERR_TIMEOUT and gives up.
constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ void backoff(uint32_t it) {
    if (it > 64) __nanosleep(it < 4096 ? 32 : 256);
}

// ------------------------------------------------------------------ keys
template <typename T> struct Vox;

template <> struct Vox<uint8_t> {
    static constexpr uint32_t code = 0;
    __device__ __forceinline__ static uint32_t key(uint8_t v) { return v; }
    __device__ __forceinline__ static float val(uint8_t v) { return (float)v; }
};
template <> struct Vox<uint16_t> {
    static constexpr uint32_t code = 1;
    __device__ __forceinline__ static uint32_t key(uint16_t v) { return v; }
    __device__ __forceinline__ static float val(uint16_t v) { return (float)v; }
};
template <> struct Vox<float> {
    static constexpr uint32_t code = 2;
    // order-preserving: negative floats flip all bits, positive set the sign bit
    __device__ __forceinline__ static uint32_t key(float v) {
        uint32_t b = __float_as_uint(v);
        return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    }
    __device__ __forceinline__ static float val(float v) { return v; }
};

__host__ __device__ __forceinline__ float key_to_float(uint32_t dtype, uint32_t k) {
    if (dtype != 2) return (float)k;
    uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float f;
    memcpy(&f, &b, 4);
    return f;
#endif
}

// Block activity (blockFilteringTestUtils.h:456-469): min != max and the
// isovalue in [min, max]; integer volumes compare round(iso) (half away from
// zero, as std::round), float volumes compare in float.
__device__ __forceinline__ bool block_active(uint32_t dtype, uint32_t kmin, uint32_t kmax, float iso) {
    if (dtype == 2) {
        float a = key_to_float(2, kmin), b = key_to_float(2, kmax);
        return (a != b) && iso >= a && iso <= b;
    }
    float r = roundf(iso);
    return (kmin != kmax) && r >= (float)kmin && r <= (float)kmax;
}

// ---------------------------------------------------------- relaxed words
__device__ __forceinline__ uint32_t ld_volatile(const uint32_t *p) { return *(volatile const uint32_t *)p; }
__device__ __forceinline__ uint64_t ld_volatile(const uint64_t *p) {
    return *(volatile const unsigned long long *)p;
}
__device__ __forceinline__ void st_volatile(uint32_t *p, uint32_t v) { *(volatile uint32_t *)p = v; }
__device__ __forceinline__ void st_volatile(uint64_t *p, uint64_t v) {
    *(volatile unsigned long long *)p = v;
}

// ------------------------------------------------------------- mbarrier/TMA
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// try_wait with a suspend-time hint: a thread whose phase is not complete is
// suspended (issues nothing) until the phase completes or `ns` nanoseconds pass.
__device__ __forceinline__ bool mbar_try_wait_for(uint64_t *bar, uint32_t parity, uint32_t ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr uint32_t kMbarSuspendNs = 1u << 20;          // about 1 ms per try
constexpr uint64_t kMbarWaitLimitNs = 2000000000ull;  // 2 s in all

// Waits for the phase with the given parity; false after about 2 s (by the
// global timer, or kSpinLimit tries should the timer not advance).  Waiting
// warps sleep in try_wait instead of polling, so that the warps with work
// get the issue slots.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 0; it < kSpinLimit; ++it) {
        if (mbar_try_wait_for(bar, parity, kMbarSuspendNs)) return true;
        if (globaltimer_ns() - t0 > kMbarWaitLimitNs) return false;
    }
    return false;
}

// 3D tiled TMA load (no multicast) of the box at element coordinates
// (x, y, z) into shared memory, completing on the mbarrier.
__device__ __forceinline__ void tma_load_3d(void *smem_dst, const CUtensorMap *map, uint64_t *bar, int x,
                                            int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(smem_dst)),
        "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// Untiled bulk copy (no multicast) of `bytes` from global to shared memory,
// completing on the mbarrier; both addresses 16-byte aligned, bytes a
// multiple of 16.
__device__ __forceinline__ void bulk_load(void *smem_dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(smem_dst)),
        "l"((uint64_t)src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap *map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)map) : "memory");
}

// ------------------------------------------------------------ CTA scans
// Exclusive scan of one value per thread across a CTA of NT threads;
// returns the exclusive prefix and writes the total to *total.  `tmp` needs
// NT/32 + 1 words of shared memory.  Contains __syncthreads (three).
template <int NT>
__device__ __forceinline__ uint32_t cta_exclusive_scan(uint32_t v, uint32_t *tmp, uint32_t *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) tmp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < NT / 32 ? tmp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < NT / 32) tmp[lane] = w; // inclusive per warp
        if (lane == NT / 32 - 1) tmp[NT / 32] = w;
    }
    __syncthreads();
    uint32_t base = warp ? tmp[warp - 1] : 0u;
    *total = tmp[NT / 32];
    __syncthreads(); // tmp may be reused right after
    return base + x - v;
}

// Same for 64-bit values.
template <int NT>
__device__ __forceinline__ uint64_t cta_exclusive_scan64(uint64_t v, uint64_t *tmp, uint64_t *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) tmp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = lane < NT / 32 ? tmp[lane] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < NT / 32) tmp[lane] = w;
        if (lane == NT / 32 - 1) tmp[NT / 32] = w;
    }
    __syncthreads();
    uint64_t base = warp ? tmp[warp - 1] : 0ull;
    *total = tmp[NT / 32];
    __syncthreads();
    return base + x - v;
}

}  // namespace mtx
