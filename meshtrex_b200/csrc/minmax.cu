// Stage 1 kernels: per-block min/max over (B+1)^3 voxels and the min/max
// octree (meshtrex: minMaxLeaf.comp.glsl:31-128 and
// minMaxOctreeReduce.comp.glsl:23-59, dispatched by minMaxPass.cpp:147-253).
//
// The leaf pass streams the volume once from HBM.  A warp owns a 32 x 16-byte
// strip of voxel rows for one block row (by) and a run of block slabs (bz):
// per z slice it loads the B+1 rows of its strip with 16-byte vector loads,
// folds them with packed SIMD min/max, reduces each block's B+1 columns
// (the +1 halo column comes from the next lane by shuffle), and folds the
// slice into the running block of its z run.  The slice at z = (bz+1)*B is
// the halo of block bz and the first slice of bz+1, so it is loaded once.
// Only the halo row of the y direction is read twice, by two warps that run
// side by side, so DRAM sees each voxel once and L2 serves the repeat.
#include "mtx_internal.h"

namespace mtx {

// ---------------------------------------------------- packed 16-byte lanes
template <typename T> struct Lane16;

template <> struct Lane16<uint8_t> {
    static constexpr int V = 16;
    __device__ __forceinline__ static uint4 lo_id() { return make_uint4(~0u, ~0u, ~0u, ~0u); }
    __device__ __forceinline__ static uint4 hi_id() { return make_uint4(0, 0, 0, 0); }
    __device__ __forceinline__ static void fold(uint4 &mn, uint4 &mx, uint4 v) {
        mn.x = __vminu4(mn.x, v.x); mn.y = __vminu4(mn.y, v.y); mn.z = __vminu4(mn.z, v.z); mn.w = __vminu4(mn.w, v.w);
        mx.x = __vmaxu4(mx.x, v.x); mx.y = __vmaxu4(mx.y, v.y); mx.z = __vmaxu4(mx.z, v.z); mx.w = __vmaxu4(mx.w, v.w);
    }
    __device__ __forceinline__ static uint32_t elem(const uint4 &w, int i, bool is_max) {
        uint32_t word = (i >> 2) == 0 ? w.x : (i >> 2) == 1 ? w.y : (i >> 2) == 2 ? w.z : w.w;
        return (word >> (8 * (i & 3))) & 0xFFu;
    }
};

template <> struct Lane16<uint16_t> {
    static constexpr int V = 8;
    __device__ __forceinline__ static uint4 lo_id() { return make_uint4(~0u, ~0u, ~0u, ~0u); }
    __device__ __forceinline__ static uint4 hi_id() { return make_uint4(0, 0, 0, 0); }
    __device__ __forceinline__ static void fold(uint4 &mn, uint4 &mx, uint4 v) {
        mn.x = __vminu2(mn.x, v.x); mn.y = __vminu2(mn.y, v.y); mn.z = __vminu2(mn.z, v.z); mn.w = __vminu2(mn.w, v.w);
        mx.x = __vmaxu2(mx.x, v.x); mx.y = __vmaxu2(mx.y, v.y); mx.z = __vmaxu2(mx.z, v.z); mx.w = __vmaxu2(mx.w, v.w);
    }
    __device__ __forceinline__ static uint32_t elem(const uint4 &w, int i, bool is_max) {
        uint32_t word = (i >> 1) == 0 ? w.x : (i >> 1) == 1 ? w.y : (i >> 1) == 2 ? w.z : w.w;
        return (word >> (16 * (i & 1))) & 0xFFFFu;
    }
};

template <> struct Lane16<float> {
    static constexpr int V = 4;
    // lanes hold order-preserving keys, one per float
    __device__ __forceinline__ static uint4 lo_id() { return make_uint4(~0u, ~0u, ~0u, ~0u); }
    __device__ __forceinline__ static uint4 hi_id() { return make_uint4(0, 0, 0, 0); }
    __device__ __forceinline__ static void fold(uint4 &mn, uint4 &mx, uint4 v) {
        uint32_t k0 = Vox<float>::key(__uint_as_float(v.x)), k1 = Vox<float>::key(__uint_as_float(v.y));
        uint32_t k2 = Vox<float>::key(__uint_as_float(v.z)), k3 = Vox<float>::key(__uint_as_float(v.w));
        mn.x = min(mn.x, k0); mn.y = min(mn.y, k1); mn.z = min(mn.z, k2); mn.w = min(mn.w, k3);
        mx.x = max(mx.x, k0); mx.y = max(mx.y, k1); mx.z = max(mx.z, k2); mx.w = max(mx.w, k3);
    }
    __device__ __forceinline__ static uint32_t elem(const uint4 &w, int i, bool is_max) {
        return i == 0 ? w.x : i == 1 ? w.y : i == 2 ? w.z : w.w;
    }
};

template <typename T, int B>
__global__ void __launch_bounds__(128) minmax_leaf_vec_kernel(const T *__restrict__ vol, uint32_t X,
                                                              uint32_t Y, uint32_t Z, uint32_t GX,
                                                              uint32_t GY, uint32_t GZ, uint32_t nXS,
                                                              uint32_t zchunk, uint64_t nwarps,
                                                              uint2 *__restrict__ leaf) {
    using L16 = Lane16<T>;
    constexpr int V = L16::V;
    constexpr int SEG = 32 * V;
    constexpr int NB = V >= B ? V / B : 1;      // blocks per lane
    constexpr int LPB = V >= B ? 1 : B / V;     // lanes per block
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t w = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w >= nwarps) return;  // uniform per warp
    const uint32_t xs = (uint32_t)(w % nXS);
    const uint64_t rest = w / nXS;
    const uint32_t by = (uint32_t)(rest % GY);
    const uint32_t zc = (uint32_t)(rest / GY);
    const uint32_t bz0 = zc * zchunk;
    const uint32_t bz1 = min(GZ, bz0 + zchunk);
    if (bz0 >= GZ) return;

    const uint32_t x0 = xs * SEG + lane * V;
    const bool on = x0 < X;                       // X is a multiple of V
    const uint32_t xh = xs * SEG + SEG;           // halo column of the strip
    const bool halo_on = lane == 31 && xh < X;
    const uint32_t y0 = by * B;
    const uint32_t ny = min((uint32_t)B + 1u, Y - y0);
    const uint64_t plane = (uint64_t)X * Y;

    uint32_t amn[NB], amx[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) { amn[j] = ~0u; amx[j] = 0u; }

    const uint32_t zend = min(bz1 * B, Z - 1);
    uint32_t bz = bz0;
    for (uint32_t z = bz0 * B; z <= zend; ++z) {
        const T *row = vol + (uint64_t)z * plane + (uint64_t)y0 * X;
        uint4 mn = L16::lo_id(), mx = L16::hi_id();
        uint32_t hmn = ~0u, hmx = 0u;
        if (on) {
#pragma unroll
            for (int r = 0; r <= B; ++r) {
                if ((uint32_t)r < ny) {
                    uint4 v = __ldg(reinterpret_cast<const uint4 *>(row + (uint64_t)r * X + x0));
                    L16::fold(mn, mx, v);
                }
            }
        }
        if (halo_on) {
#pragma unroll
            for (int r = 0; r <= B; ++r) {
                if ((uint32_t)r < ny) {
                    uint32_t k = Vox<T>::key(__ldg(row + (uint64_t)r * X + xh));
                    hmn = min(hmn, k);
                    hmx = max(hmx, k);
                }
            }
        }
        // first column of the next lane is this lane's halo column
        uint32_t nmn = __shfl_down_sync(0xffffffffu, L16::elem(mn, 0, false), 1);
        uint32_t nmx = __shfl_down_sync(0xffffffffu, L16::elem(mx, 0, true), 1);
        if (lane == 31) { nmn = hmn; nmx = hmx; }

        uint32_t smn[NB], smx[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            uint32_t a = ~0u, b = 0u;
            constexpr int CNT = V >= B ? B : V;
#pragma unroll
            for (int i = 0; i < CNT; ++i) {
                a = min(a, L16::elem(mn, j * CNT + i, false));
                b = max(b, L16::elem(mx, j * CNT + i, true));
            }
            const bool take_halo = V >= B ? true : ((lane % LPB) == LPB - 1);
            if (take_halo) {
                if (V >= B && j + 1 < NB) {
                    a = min(a, L16::elem(mn, (j + 1) * B, false));
                    b = max(b, L16::elem(mx, (j + 1) * B, true));
                } else {
                    a = min(a, nmn);
                    b = max(b, nmx);
                }
            }
            smn[j] = a;
            smx[j] = b;
        }

        const bool boundary = z == bz * B + B;  // halo slice of bz, first slice of bz + 1
#pragma unroll
        for (int j = 0; j < NB; ++j) { amn[j] = min(amn[j], smn[j]); amx[j] = max(amx[j], smx[j]); }
        if (boundary) {
            // write block bz
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                uint32_t a = amn[j], b = amx[j];
#pragma unroll
                for (int o = 1; o < LPB; o <<= 1) {
                    a = min(a, __shfl_xor_sync(0xffffffffu, a, o));
                    b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
                }
                if (on && (lane % LPB) == 0) {
                    uint32_t bx = x0 / B + j;
                    leaf[((uint64_t)bz * GY + by) * GX + bx] = make_uint2(a, b);
                }
                amn[j] = smn[j];
                amx[j] = smx[j];
            }
            ++bz;
        }
    }
    if (bz < bz1) {
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            uint32_t a = amn[j], b = amx[j];
#pragma unroll
            for (int o = 1; o < LPB; o <<= 1) {
                a = min(a, __shfl_xor_sync(0xffffffffu, a, o));
                b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
            }
            if (on && (lane % LPB) == 0) {
                uint32_t bx = x0 / B + j;
                leaf[((uint64_t)bz * GY + by) * GX + bx] = make_uint2(a, b);
            }
        }
    }
}

// Fallback for any block edge and any row alignment: one thread per block.
template <typename T>
__global__ void __launch_bounds__(128) minmax_leaf_generic_kernel(const T *__restrict__ vol, uint32_t X,
                                                                  uint32_t Y, uint32_t Z, uint32_t B,
                                                                  uint32_t GX, uint32_t GY,
                                                                  uint64_t nblocks, uint2 *__restrict__ leaf) {
    uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    uint32_t bx = (uint32_t)(b % GX), by = (uint32_t)((b / GX) % GY), bz = (uint32_t)(b / ((uint64_t)GX * GY));
    uint32_t x0 = bx * B, y0 = by * B, z0 = bz * B;
    uint32_t x1 = min(x0 + B, X - 1), y1 = min(y0 + B, Y - 1), z1 = min(z0 + B, Z - 1);
    uint32_t mn = ~0u, mx = 0u;
    for (uint32_t z = z0; z <= z1; ++z)
        for (uint32_t y = y0; y <= y1; ++y) {
            const T *row = vol + ((uint64_t)z * Y + y) * X;
            for (uint32_t x = x0; x <= x1; ++x) {
                uint32_t k = Vox<T>::key(__ldg(row + x));
                mn = min(mn, k);
                mx = max(mx, k);
            }
        }
    leaf[b] = make_uint2(mn, mx);
}

// One octree level: each texel reduces its up-to-8 children; children past
// the source extent are skipped (minMaxOctreeReduce.comp.glsl:37-47).
__global__ void __launch_bounds__(256) pyramid_level_kernel(const uint2 *__restrict__ src, uint32_t sx,
                                                            uint32_t sy, uint32_t sz, uint2 *__restrict__ dst,
                                                            uint32_t dx, uint32_t dy, uint32_t dz) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t n = (uint64_t)dx * dy * dz;
    if (i >= n) return;
    uint32_t x = (uint32_t)(i % dx), y = (uint32_t)((i / dx) % dy), z = (uint32_t)(i / ((uint64_t)dx * dy));
    uint32_t mn = ~0u, mx = 0u;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        uint32_t cx = 2 * x + (c & 1), cy = 2 * y + ((c >> 1) & 1), cz = 2 * z + (c >> 2);
        if (cx < sx && cy < sy && cz < sz) {
            uint2 v = src[((uint64_t)cz * sy + cy) * sx + cx];
            mn = min(mn, v.x);
            mx = max(mx, v.y);
        }
    }
    dst[i] = make_uint2(mn, mx);
}

// ------------------------------------------------------------------ host
template <typename T, int B>
static cudaError_t launch_vec(const Problem &p, uint2 *leaf, cudaStream_t s, int sm_count, uint32_t zover) {
    constexpr uint32_t SEG = 32 * (16 / sizeof(T));
    uint32_t nXS = ceil_div(p.X, SEG);
    uint64_t cols = (uint64_t)nXS * p.GY;
    // enough warps to keep ~64 KiB of loads in flight per SM
    uint64_t want = (uint64_t)sm_count * 48;
    uint32_t nzc = (uint32_t)std::min<uint64_t>(p.GZ, std::max<uint64_t>(1, (want + cols - 1) / cols));
    uint32_t zchunk = zover ? zover : ceil_div(p.GZ, nzc);
    nzc = ceil_div(p.GZ, zchunk);
    uint64_t nwarps = cols * nzc;
    uint64_t blocks = (nwarps + 3) / 4;
    minmax_leaf_vec_kernel<T, B><<<(unsigned)blocks, 128, 0, s>>>((const T *)p.vol, p.X, p.Y, p.Z, p.GX, p.GY,
                                                                 p.GZ, nXS, zchunk, nwarps, leaf);
    return cudaGetLastError();
}

template <typename T>
static cudaError_t launch_generic(const Problem &p, uint2 *leaf, cudaStream_t s) {
    uint64_t blocks = (p.nblocks + 127) / 128;
    minmax_leaf_generic_kernel<T><<<(unsigned)blocks, 128, 0, s>>>((const T *)p.vol, p.X, p.Y, p.Z, p.B, p.GX,
                                                                   p.GY, p.nblocks, leaf);
    return cudaGetLastError();
}

template <typename T>
static cudaError_t dispatch_leaf(const Problem &p, uint2 *leaf, cudaStream_t s, int sm, uint32_t zover) {
    const bool vec_ok = ((uintptr_t)p.vol % 16 == 0) && (((uint64_t)p.X * sizeof(T)) % 16 == 0);
    if (vec_ok) {
        switch (p.B) {
        case 4: return launch_vec<T, 4>(p, leaf, s, sm, zover);
        case 8: return launch_vec<T, 8>(p, leaf, s, sm, zover);
        case 16: return launch_vec<T, 16>(p, leaf, s, sm, zover);
        default: break;
        }
    }
    return launch_generic<T>(p, leaf, s);
}

mtx_status launch_minmax_leaf(mtx_context *c, const Problem &p, uint2 *leaf, cudaStream_t s, uint32_t zover) {
    cudaError_t e;
    switch (p.dtype) {
    case MTX_DTYPE_U8: e = dispatch_leaf<uint8_t>(p, leaf, s, c->sm_count, zover); break;
    case MTX_DTYPE_U16: e = dispatch_leaf<uint16_t>(p, leaf, s, c->sm_count, zover); break;
    default: e = dispatch_leaf<float>(p, leaf, s, c->sm_count, zover); break;
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "minmax leaf launch");
    return MTX_OK;
}

mtx_status launch_pyramid(mtx_context *c, uint2 *all, int levels, const uint32_t ext[][3],
                          const uint64_t *offset, cudaStream_t s) {
    for (int l = 1; l < levels; ++l) {
        uint64_t n = (uint64_t)ext[l][0] * ext[l][1] * ext[l][2];
        unsigned blocks = (unsigned)((n + 255) / 256);
        pyramid_level_kernel<<<blocks, 256, 0, s>>>(all + offset[l - 1], ext[l - 1][0], ext[l - 1][1],
                                                     ext[l - 1][2], all + offset[l], ext[l][0], ext[l][1],
                                                     ext[l][2]);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(c, e, "pyramid launch");
    }
    return MTX_OK;
}

}  // namespace mtx
