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
#include <algorithm>

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

template <typename T, int B, int ZU>
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
    constexpr int CNT = V >= B ? B : V;         // elements of one block in one lane
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

// Three octree levels per launch: a CTA of 512 threads loads an 8x8x8 tile
// of level l and writes the 4^3, 2^3 and 1 texels it covers in levels l+1..l+3
// (each texel the min/max of its up-to-8 children; children past the level's
// extent are skipped, minMaxOctreeReduce.comp.glsl:37-47).
struct PyrLevels {
    uint2 *base[4];      // level l .. l+3
    uint32_t ext[4][3];  // their extents
    int nout;            // levels written (1..3)
};

__global__ void __launch_bounds__(512) pyramid3_kernel(PyrLevels L, uint32_t tiles_x, uint32_t tiles_y) {
    __shared__ uint2 s[512];
    const uint32_t tx = blockIdx.x % tiles_x, ty = (blockIdx.x / tiles_x) % tiles_y, tz = blockIdx.x / (tiles_x * tiles_y);
    const uint32_t lx = threadIdx.x & 7, ly = (threadIdx.x >> 3) & 7, lz = threadIdx.x >> 6;
    const uint32_t x = tx * 8 + lx, y = ty * 8 + ly, z = tz * 8 + lz;
    uint2 v = make_uint2(~0u, 0u);
    if (x < L.ext[0][0] && y < L.ext[0][1] && z < L.ext[0][2])
        v = L.base[0][((uint64_t)z * L.ext[0][1] + y) * L.ext[0][0] + x];
    s[threadIdx.x] = v;
    __syncthreads();
    uint32_t n = 8;  // current tile edge in shared memory
    for (int k = 1; k <= L.nout; ++k) {
        const uint32_t m = n >> 1;
        uint2 r = make_uint2(~0u, 0u);
        const bool act = threadIdx.x < m * m * m;
        const uint32_t cx = threadIdx.x % m, cy = (threadIdx.x / m) % m, cz = threadIdx.x / (m * m);
        if (act) {
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const uint2 w = s[((2 * cz + (c >> 2)) * n + 2 * cy + ((c >> 1) & 1)) * n + 2 * cx + (c & 1)];
                r.x = min(r.x, w.x);
                r.y = max(r.y, w.y);
            }
        }
        __syncthreads();
        if (act) {
            s[threadIdx.x] = r;  // compact m^3 layout for the next level
            const uint32_t ox = tx * m + cx, oy = ty * m + cy, oz = tz * m + cz;
            if (ox < L.ext[k][0] && oy < L.ext[k][1] && oz < L.ext[k][2])
                L.base[k][((uint64_t)oz * L.ext[k][1] + oy) * L.ext[k][0] + ox] = r;
        }
        __syncthreads();
        n = m;
    }
}

// ------------------------------------------------------------------ host
template <typename T, int B, int ZU>
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
    minmax_leaf_vec_kernel<T, B, ZU><<<(unsigned)blocks, 128, 0, s>>>((const T *)p.vol, p.X, p.Y, p.Z, p.GX, p.GY,
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

template <typename T, int ZU>
static cudaError_t dispatch_b(const Problem &p, uint2 *leaf, cudaStream_t s, int sm, uint32_t zover) {
    switch (p.B) {
    case 4: return launch_vec<T, 4, ZU>(p, leaf, s, sm, zover);
    case 8: return launch_vec<T, 8, ZU>(p, leaf, s, sm, zover);
    default: return launch_vec<T, 16, ZU>(p, leaf, s, sm, zover);
    }
}

template <typename T>
static cudaError_t dispatch_leaf(const Problem &p, uint2 *leaf, cudaStream_t s, int sm, uint32_t zover,
                                 uint32_t slices) {
    const bool vec_ok = ((uintptr_t)p.vol % 16 == 0) && (((uint64_t)p.X * sizeof(T)) % 16 == 0) &&
                        (p.B == 4 || p.B == 8 || p.B == 16);
    if (!vec_ok) return launch_generic<T>(p, leaf, s);
    switch (slices) {
    case 1: return dispatch_b<T, 1>(p, leaf, s, sm, zover);
    case 4: return dispatch_b<T, 4>(p, leaf, s, sm, zover);
    default: return dispatch_b<T, 2>(p, leaf, s, sm, zover);
    }
}

mtx_status launch_minmax_leaf(mtx_context *c, const Problem &p, uint2 *leaf, cudaStream_t s, uint32_t zover) {
    cudaError_t e;
    if (!zover) zover = c->tuning.minmaxZChunk;
    const uint32_t sl = c->tuning.minmaxSlices;
    switch (p.dtype) {
    case MTX_DTYPE_U8: e = dispatch_leaf<uint8_t>(p, leaf, s, c->sm_count, zover, sl); break;
    case MTX_DTYPE_U16: e = dispatch_leaf<uint16_t>(p, leaf, s, c->sm_count, zover, sl); break;
    default: e = dispatch_leaf<float>(p, leaf, s, c->sm_count, zover, sl); break;
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "minmax leaf launch");
    return MTX_OK;
}

mtx_status launch_pyramid(mtx_context *c, uint2 *all, int levels, const uint32_t ext[][3],
                          const uint64_t *offset, cudaStream_t s) {
    for (int l = 0; l + 1 < levels; l += 3) {
        PyrLevels P;
        P.nout = std::min(3, levels - 1 - l);
        for (int k = 0; k <= 3; ++k) {
            const int lv = std::min(l + k, levels - 1);
            P.base[k] = all + offset[lv];
            for (int a = 0; a < 3; ++a) P.ext[k][a] = ext[lv][a];
        }
        const uint32_t tx = ceil_div(ext[l][0], 8), ty = ceil_div(ext[l][1], 8), tz = ceil_div(ext[l][2], 8);
        pyramid3_kernel<<<tx * ty * tz, 512, 0, s>>>(P, tx, ty);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(c, e, "pyramid launch");
    }
    return MTX_OK;
}

}  // namespace mtx
