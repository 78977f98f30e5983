// Device bodies of the leaf min/max pass (meshtrex: minMaxLeaf.comp.glsl:31-128),
// shared by the single-volume kernels (minmax.cu) and the batched kernel
// (batched.cu).
//
// A warp owns a 32 x 16-byte strip of voxel rows for one block row (by) and a
// run of block slabs (bz): per z slice it loads the B+1 rows of its strip with
// 16-byte vector loads, folds them with packed SIMD min/max, reduces each
// block's B+1 columns (the +1 halo column comes from the next lane by
// shuffle), and folds the slice into the running block of its z run.  The
// slice at z = (bz+1)*B is the halo of block bz and the first slice of bz+1,
// so it is loaded once.
#pragma once

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
    __device__ __forceinline__ static void merge(uint4 &mn, uint4 &mx, const uint4 &mn2, const uint4 &mx2) {
        mn.x = __vminu4(mn.x, mn2.x); mn.y = __vminu4(mn.y, mn2.y); mn.z = __vminu4(mn.z, mn2.z); mn.w = __vminu4(mn.w, mn2.w);
        mx.x = __vmaxu4(mx.x, mx2.x); mx.y = __vmaxu4(mx.y, mx2.y); mx.z = __vmaxu4(mx.z, mx2.z); mx.w = __vmaxu4(mx.w, mx2.w);
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
    __device__ __forceinline__ static void merge(uint4 &mn, uint4 &mx, const uint4 &mn2, const uint4 &mx2) {
        mn.x = __vminu2(mn.x, mn2.x); mn.y = __vminu2(mn.y, mn2.y); mn.z = __vminu2(mn.z, mn2.z); mn.w = __vminu2(mn.w, mn2.w);
        mx.x = __vmaxu2(mx.x, mx2.x); mx.y = __vmaxu2(mx.y, mx2.y); mx.z = __vmaxu2(mx.z, mx2.z); mx.w = __vmaxu2(mx.w, mx2.w);
    }
    __device__ __forceinline__ static uint32_t elem(const uint4 &w, int i, bool is_max) {
        uint32_t word = (i >> 1) == 0 ? w.x : (i >> 1) == 1 ? w.y : (i >> 1) == 2 ? w.z : w.w;
        return (word >> (16 * (i & 1))) & 0xFFFFu;
    }
    __device__ __forceinline__ static void init(uint4 &mn, uint4 &mx, uint4 v) { mn = v; mx = v; }
    // two rows per instruction: three-input packed min/max
    __device__ __forceinline__ static void fold2(uint4 &mn, uint4 &mx, uint4 a, uint4 b) {
        mn.x = __vimin3_u16x2(mn.x, a.x, b.x); mn.y = __vimin3_u16x2(mn.y, a.y, b.y);
        mn.z = __vimin3_u16x2(mn.z, a.z, b.z); mn.w = __vimin3_u16x2(mn.w, a.w, b.w);
        mx.x = __vimax3_u16x2(mx.x, a.x, b.x); mx.y = __vimax3_u16x2(mx.y, a.y, b.y);
        mx.z = __vimax3_u16x2(mx.z, a.z, b.z); mx.w = __vimax3_u16x2(mx.w, a.w, b.w);
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
    __device__ __forceinline__ static void merge(uint4 &mn, uint4 &mx, const uint4 &mn2, const uint4 &mx2) {
        mn.x = min(mn.x, mn2.x); mn.y = min(mn.y, mn2.y); mn.z = min(mn.z, mn2.z); mn.w = min(mn.w, mn2.w);
        mx.x = max(mx.x, mx2.x); mx.y = max(mx.y, mx2.y); mx.z = max(mx.z, mx2.z); mx.w = max(mx.w, mx2.w);
    }
    __device__ __forceinline__ static uint32_t elem(const uint4 &w, int i, bool is_max) {
        return i == 0 ? w.x : i == 1 ? w.y : i == 2 ? w.z : w.w;
    }
    __device__ __forceinline__ static uint4 keys(uint4 v) {
        return make_uint4(Vox<float>::key(__uint_as_float(v.x)), Vox<float>::key(__uint_as_float(v.y)),
                          Vox<float>::key(__uint_as_float(v.z)), Vox<float>::key(__uint_as_float(v.w)));
    }
    __device__ __forceinline__ static void init(uint4 &mn, uint4 &mx, uint4 v) { mn = mx = keys(v); }
    __device__ __forceinline__ static void fold2(uint4 &mn, uint4 &mx, uint4 a, uint4 b) {
        const uint4 ka = keys(a), kb = keys(b);
        mn.x = __vimin3_u32(mn.x, ka.x, kb.x); mn.y = __vimin3_u32(mn.y, ka.y, kb.y);
        mn.z = __vimin3_u32(mn.z, ka.z, kb.z); mn.w = __vimin3_u32(mn.w, ka.w, kb.w);
        mx.x = __vimax3_u32(mx.x, ka.x, kb.x); mx.y = __vimax3_u32(mx.y, ka.y, kb.y);
        mx.z = __vimax3_u32(mx.z, ka.z, kb.z); mx.w = __vimax3_u32(mx.w, ka.w, kb.w);
    }
};

// One warp's share of the leaf pass: warp w of the volume's
// nXS * GY * ceil(GZ / zchunk) warps.
template <typename T, int B, int ZU>
__device__ __forceinline__ void minmax_leaf_vec_warp(const T *__restrict__ vol, uint32_t X, uint32_t Y, uint32_t Z,
                                                     uint32_t GX, uint32_t GY, uint32_t GZ, uint32_t nXS,
                                                     uint32_t zchunk, uint64_t w, uint2 *__restrict__ leaf) {
    using L16 = Lane16<T>;
    constexpr int V = L16::V;
    constexpr int SEG = 32 * V;
    constexpr int NB = V >= B ? V / B : 1;      // blocks per lane
    constexpr int LPB = V >= B ? 1 : B / V;     // lanes per block
    constexpr int CNT = V >= B ? B : V;         // elements of one block in one lane
    const uint32_t lane = threadIdx.x & 31;
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
    for (uint32_t z0 = bz0 * B; z0 <= zend; z0 += ZU) {
        // issue every load of the ZU slices before any of them is folded
        uint4 v[ZU][B + 1];
        uint32_t hv[ZU][B + 1];
#pragma unroll
        for (int u = 0; u < ZU; ++u) {
            const T *row = vol + (uint64_t)(z0 + u) * plane + (uint64_t)y0 * X;
            const bool zon = z0 + u <= zend;
#pragma unroll
            for (int r = 0; r <= B; ++r) {
                v[u][r] = L16::lo_id();
                if (on && zon && (uint32_t)r < ny)
                    v[u][r] = __ldg(reinterpret_cast<const uint4 *>(row + (uint64_t)r * X + x0));
                hv[u][r] = 0;
                if (halo_on && zon && (uint32_t)r < ny) hv[u][r] = Vox<T>::key(__ldg(row + (uint64_t)r * X + xh));
            }
        }
#pragma unroll
        for (int u = 0; u < ZU; ++u) {
            const uint32_t z = z0 + u;
            if (z > zend) break;
            uint4 mn = L16::lo_id(), mx = L16::hi_id();
            uint32_t hmn = ~0u, hmx = 0u;
#pragma unroll
            for (int r = 0; r <= B; ++r) {
                if ((uint32_t)r < ny) {
                    if (on) L16::fold(mn, mx, v[u][r]);
                    if (halo_on) {
                        hmn = min(hmn, hv[u][r]);
                        hmx = max(hmx, hv[u][r]);
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
#pragma unroll
            for (int j = 0; j < NB; ++j) { amn[j] = min(amn[j], smn[j]); amx[j] = max(amx[j], smx[j]); }
            if (z == bz * B + B) {
                // halo slice of bz, first slice of bz + 1: write block bz
#pragma unroll
                for (int j = 0; j < NB; ++j) {
                    uint32_t a = amn[j], b = amx[j];
#pragma unroll
                    for (int o = 1; o < LPB; o <<= 1) {
                        a = min(a, __shfl_xor_sync(0xffffffffu, a, o));
                        b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
                    }
                    if (on && (lane % LPB) == 0) {
                        const uint32_t bx = x0 / B + j;
                        if (MTX_BC(((uint64_t)bz * GY + by) * GX + bx, (uint64_t)GX * GY * GZ, kBcLeaf))
                            leaf[((uint64_t)bz * GY + by) * GX + bx] = make_uint2(a, b);
                    }
                    amn[j] = smn[j];
                    amx[j] = smx[j];
                }
                ++bz;
            }
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
                const uint32_t bx = x0 / B + j;
                if (MTX_BC(((uint64_t)bz * GY + by) * GX + bx, (uint64_t)GX * GY * GZ, kBcLeaf))
                    leaf[((uint64_t)bz * GY + by) * GX + bx] = make_uint2(a, b);
            }
        }
    }
}

// Fallback for any block edge and any row alignment: one thread per block.
template <typename T>
__device__ __forceinline__ void minmax_leaf_one(const T *__restrict__ vol, uint32_t X, uint32_t Y, uint32_t Z,
                                                uint32_t B, uint32_t GX, uint32_t GY, uint64_t b,
                                                uint2 *__restrict__ leaf) {
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

}  // namespace mtx
