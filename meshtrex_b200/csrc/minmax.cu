// Stage 1 kernels: per-block min/max over (B+1)^3 voxels and the min/max
// octree (meshtrex: minMaxLeaf.comp.glsl:31-128 and
// minMaxOctreeReduce.comp.glsl:23-59, dispatched by minMaxPass.cpp:147-253).
//
// The leaf pass streams the volume once from HBM (the warp layout is described
// in minmax_device.cuh).  Only the halo row of the y direction is read twice,
// by two warps that run side by side, so DRAM sees each voxel once and L2
// serves the repeat.
#include <algorithm>

#include "minmax_device.cuh"

namespace mtx {

template <typename T, int B, int ZU>
__global__ void __launch_bounds__(128) minmax_leaf_vec_kernel(const T *__restrict__ vol, uint32_t X,
                                                              uint32_t Y, uint32_t Z, uint32_t GX,
                                                              uint32_t GY, uint32_t GZ, uint32_t nXS,
                                                              uint32_t zchunk, uint64_t nwarps,
                                                              uint2 *__restrict__ leaf) {
    const uint64_t w = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w >= nwarps) return;  // uniform per warp
    minmax_leaf_vec_warp<T, B, ZU>(vol, X, Y, Z, GX, GY, GZ, nXS, zchunk, w, leaf);
}

// Fallback for any block edge and any row alignment: one thread per block.
template <typename T>
__global__ void __launch_bounds__(128) minmax_leaf_generic_kernel(const T *__restrict__ vol, uint32_t X,
                                                                  uint32_t Y, uint32_t Z, uint32_t B,
                                                                  uint32_t GX, uint32_t GY,
                                                                  uint64_t nblocks, uint2 *__restrict__ leaf) {
    const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nblocks) minmax_leaf_one<T>(vol, X, Y, Z, B, GX, GY, b, leaf);
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
