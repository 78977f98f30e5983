// Stage 1 kernels: per-block min/max over (B+1)^3 voxels and the min/max
// octree (meshtrex: minMaxLeaf.comp.glsl:31-128 and
// minMaxOctreeReduce.comp.glsl:23-59, dispatched by minMaxPass.cpp:147-253).
//
// The leaf pass streams the volume once from HBM (the warp layout is described
// in minmax_device.cuh).  The halo rows and slices it reads twice are read by
// items that run side by side, so L2 serves the repeat; the TMA pass reads no
// halo column at all (minmax_xface_patch_kernel).
#include <algorithm>
#include <cstring>

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

// TMA-fed leaf pass for 2- and 4-byte voxels: persistent CTAs of four warps,
// four per SM.  A work item is (x-strip of 512 bytes, run of ZC block slabs,
// group of four block rows), taken in that order so that the strips of one row
// and the items sharing a halo slice or row run side by side (L2 serves the
// repeats, DRAM sees whole rows).  Per z slice thread 0 issues one TMA box of
// the strip's 4B+1 rows into a ring of S stages (out-of-volume parts read as
// zero and are masked).  Warp w folds block row w of the group with the
// per-lane arithmetic of the load-based body: lane l owns 16 bytes of every
// row, the +1 column of a block comes from the next lane by shuffle, and a
// slice at z = (bz+1)*B closes block bz and opens bz+1; rows fold two at a
// time with three-input packed min/max.
// The +1 column of a strip's last block is the next strip's first column.
// Loaded beside the strip, that 16-byte column cost a 32-byte DRAM sector
// per row (98 MB, 4.6% of a 1024^3 uint16 volume, 0.016 ms of 0.353): instead
// lane 0 of every strip but the first folds its own first column over each
// block's (B+1)^2 rows and slices into xface, and minmax_xface_patch_kernel
// merges it into the previous strip's last block (and its level-1 texel).
// Loads in flight live in shared memory (about 34 KB per CTA), not in
// registers, so an SM keeps room for the extraction kernels of other streams.
constexpr int kTmaRows(int B) { return 4 * B + 1; }
constexpr uint32_t kTmaMain(int B) { return (uint32_t)kTmaRows(B) * 512u; }
constexpr uint32_t kTmaStage(int B) { return (kTmaMain(B) + 127u) / 128u * 128u; }
constexpr int kTmaStages(int B) { return B == 4 ? 4 : 2; }  // about 34 KB per CTA at B = 4 and 8
constexpr int kTmaCtasPerSm = 4;  // 16 warps: enough to hide the fold's latencies, smem left for other kernels

struct TmaLeafArgs {
    uint32_t X, Y, Z, GX, GY, GZ;
    uint32_t nXS, nYG, nZC, zchunk;
    uint32_t nitems;
    uint32_t E1[3];  // extents of octree level 1 (written when the kernel's l1 is set)
};

// Octree level 1 in the same pass (l1 set; one block per lane, even z runs):
// a texel is the min/max of 2 x 2 x 2 blocks -- two consecutive blocks of a
// warp's z run, the x pair by shuffle, the y pair (warps w and w + 1) through
// shared memory after the slice's barrier.  Blocks outside the grid count as
// the identity {~0, 0}.
// xface: (nXS - 1) x GY x GZ strip-start columns (minmax_xface_patch_kernel).
template <typename T, int B>
__global__ void __launch_bounds__(128) minmax_leaf_tma_kernel(const __grid_constant__ CUtensorMap map_main,
                                                                 const TmaLeafArgs a, uint2 *__restrict__ leaf,
                                                                 uint2 *__restrict__ l1, uint2 *__restrict__ xface,
                                                                 DevStatus *st) {
    using L16 = Lane16<T>;
    constexpr int V = L16::V;
    constexpr int SEG = 32 * V;
    constexpr int NB = V >= B ? V / B : 1;   // blocks per lane
    constexpr int LPB = V >= B ? 1 : B / V;  // lanes per block
    constexpr int CNT = V >= B ? B : V;      // elements of one block in one lane
    constexpr int S = kTmaStages(B);
    constexpr uint32_t MAIN = kTmaMain(B), STAGE = kTmaStage(B);
    constexpr uint32_t TX = MAIN;  // bytes per stage
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[S];
    __shared__ uint32_t s_fail;
    __shared__ uint2 s_l1[4][32];  // level-1 y pairs: the z- and x-combined value of each warp's lanes
    const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;

    if (tid == 0) {
        for (int i = 0; i < S; ++i) mbar_init(&bars[i], 1);
        fence_mbar_init();
        s_fail = 0;
        prefetch_tensormap(&map_main);
    }
    __syncthreads();

    // the CTA's slices in order: items blockIdx.x, blockIdx.x + gridDim.x, ...
    // each from z = bz0*B to min(bz1*B, Z-1)
    auto item_of = [&](uint32_t k, uint32_t &xs, uint32_t &g, uint32_t &zs, uint32_t &ze, uint32_t &bz0,
                       uint32_t &bz1) {
        xs = k % a.nXS;
        const uint32_t rest = k / a.nXS, zc = rest % a.nZC;
        g = rest / a.nZC;
        bz0 = zc * a.zchunk;
        bz1 = min(a.GZ, bz0 + a.zchunk);
        zs = bz0 * B;
        ze = min(bz1 * B, a.Z - 1);
    };
    // producer cursor (thread 0 only): next slice to load
    uint32_t pk = blockIdx.x, pz = 0, pze = 0, pxs = 0, pg = 0;
    uint32_t issued = 0;  // slices issued so far
    if (tid == 0 && pk < a.nitems) {
        uint32_t b0, b1;
        item_of(pk, pxs, pg, pz, pze, b0, b1);
    }
    auto issue_next = [&]() {  // thread 0: one slice into stage issued % S
        if (pk >= a.nitems) return;
        uint64_t *bar = &bars[issued % S];
        unsigned char *dst = smem + (issued % S) * STAGE;
        fence_proxy_async();
        mbar_arrive_expect_tx(bar, TX);
        const int x0 = (int)(pxs * SEG), y0 = (int)(pg * 4 * B);
        tma_load_3d(dst, &map_main, bar, x0, y0, (int)pz);
        ++issued;
        if (++pz > pze) {
            pk += gridDim.x;
            if (pk < a.nitems) {
                uint32_t b0, b1;
                item_of(pk, pxs, pg, pz, pze, b0, b1);
            }
        }
    };
    if (tid == 0)
        for (int i = 0; i < S; ++i) issue_next();

    uint32_t seq = 0;  // slices consumed
    bool ok = true;
    for (uint32_t k = blockIdx.x; k < a.nitems && ok; k += gridDim.x) {
        uint32_t xs, g, zs, ze, bz0, bz1;
        item_of(k, xs, g, zs, ze, bz0, bz1);
        const uint32_t x0 = xs * SEG + lane * V;
        const bool on = x0 < a.X;  // X is a multiple of V
        const uint32_t by = g * 4 + w;
        const bool row_on = by < a.GY;
        // lane 0 of a strip that has one to its left: the first column, per block
        const bool f_on = lane == 0 && xs > 0 && row_on && on;
        uint32_t fmn = ~0u, fmx = 0u;
        auto f_write = [&](uint32_t cbz) {
            if (f_on && MTX_BC(((uint64_t)cbz * a.GY + by) * (a.nXS - 1) + xs - 1,
                               (uint64_t)(a.nXS - 1) * a.GY * a.GZ, kBcLeaf))
                xface[((uint64_t)cbz * a.GY + by) * (a.nXS - 1) + xs - 1] = make_uint2(fmn, fmx);
        };
        const uint32_t ny = row_on ? min((uint32_t)B + 1u, a.Y - by * B) : 0u;
        uint32_t amn[NB], amx[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j) { amn[j] = ~0u; amx[j] = 0u; }
        uint32_t bz = bz0;
        // level 1: the held even block of a z pair, and a texel waiting for its y pair
        uint32_t zlo = ~0u, zhi = 0u, pz = 0;
        bool pend = false;
        const bool bx_in = row_on && x0 / B < a.GX;
        auto l1_close = [&](uint32_t lo, uint32_t hi, uint32_t cbz) {
            if constexpr (NB == 1) {
                uint32_t vlo = bx_in ? lo : ~0u, vhi = bx_in ? hi : 0u;
                if ((cbz & 1u) == 0) {
                    zlo = vlo;
                    zhi = vhi;
                    if (cbz + 1 < a.GZ) return;  // the odd partner closes next
                } else {
                    vlo = min(vlo, zlo);
                    vhi = max(vhi, zhi);
                }
                vlo = min(vlo, __shfl_xor_sync(0xffffffffu, vlo, LPB));
                vhi = max(vhi, __shfl_xor_sync(0xffffffffu, vhi, LPB));
                s_l1[w][lane] = make_uint2(vlo, vhi);
                pz = cbz >> 1;
                pend = true;
            }
        };
        auto l1_finish = [&]() {  // after a barrier that follows l1_close
            if constexpr (NB == 1) {
                pend = false;
                if ((w & 1u) == 0 && lane % (2 * LPB) == 0) {
                    const uint2 m = s_l1[w][lane], o = s_l1[w + 1][lane];
                    const uint32_t X1 = (x0 / B) >> 1, Y1 = by >> 1;
                    if (X1 < a.E1[0] && Y1 < a.E1[1] && pz < a.E1[2])
                        l1[((uint64_t)pz * a.E1[1] + Y1) * a.E1[0] + X1] = make_uint2(min(m.x, o.x), max(m.y, o.y));
                }
            }
        };
        for (uint32_t z = zs; z <= ze; ++z, ++seq) {
            if (!mbar_wait_bounded(&bars[seq % S], (seq / S) & 1u)) {
                if (lane == 0) {
                    report(st, MTX_ERR_TIMEOUT, kSiteMinMaxTma, blockIdx.x, seq);
                    atomicExch(&s_fail, 1u);
                }
            }
            const unsigned char *stg = smem + (seq % S) * STAGE;
            // row 0, then two rows per three-input min/max; rows past the volume
            // read row 0 again, which leaves min and max unchanged
            uint4 mn = L16::lo_id(), mx = L16::hi_id();
            if (on) {
                const unsigned char *src = stg + w * B * 512u + lane * 16u;
                auto row = [&](int r) {
                    return *reinterpret_cast<const uint4 *>(src + ((uint32_t)r < ny ? (uint32_t)r : 0u) * 512u);
                };
                L16::init(mn, mx, row(0));
#pragma unroll
                for (int r = 1; r + 1 <= B; r += 2) L16::fold2(mn, mx, row(r), row(r + 1));
                if constexpr (B % 2 == 1) L16::fold2(mn, mx, row(B), row(B));
            }
            // first column of the next lane is this lane's halo column; lane 31's
            // is the next strip's first column, merged in by the patch kernel
            const uint32_t c0mn = L16::elem(mn, 0, false), c0mx = L16::elem(mx, 0, true);
            uint32_t nmn = __shfl_down_sync(0xffffffffu, c0mn, 1);
            uint32_t nmx = __shfl_down_sync(0xffffffffu, c0mx, 1);
            if (lane == 31) { nmn = ~0u; nmx = 0u; }
            fmn = min(fmn, c0mn);
            fmx = max(fmx, c0mx);
            uint32_t smn[NB], smx[NB];
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                uint32_t lo = ~0u, hi = 0u;
                if constexpr (sizeof(T) == 2 && CNT == 8) {  // all 8 lanes of the word: a SIMD tree
                    const uint32_t a2 = __vminu2(__vminu2(mn.x, mn.y), __vminu2(mn.z, mn.w));
                    const uint32_t b2 = __vmaxu2(__vmaxu2(mx.x, mx.y), __vmaxu2(mx.z, mx.w));
                    lo = min(a2 & 0xFFFFu, a2 >> 16);
                    hi = max(b2 & 0xFFFFu, b2 >> 16);
                } else {
#pragma unroll
                    for (int i = 0; i < CNT; ++i) {
                        lo = min(lo, L16::elem(mn, j * CNT + i, false));
                        hi = max(hi, L16::elem(mx, j * CNT + i, true));
                    }
                }
                const bool take_halo = V >= B ? true : ((lane % LPB) == LPB - 1);
                if (take_halo) {
                    if (V >= B && j + 1 < NB) {
                        lo = min(lo, L16::elem(mn, (j + 1) * B, false));
                        hi = max(hi, L16::elem(mx, (j + 1) * B, true));
                    } else {
                        lo = min(lo, nmn);
                        hi = max(hi, nmx);
                    }
                }
                smn[j] = lo;
                smx[j] = hi;
            }
#pragma unroll
            for (int j = 0; j < NB; ++j) { amn[j] = min(amn[j], smn[j]); amx[j] = max(amx[j], smx[j]); }
            if (z == bz * B + B) {
                // halo slice of bz, first slice of bz + 1: write block bz
                uint32_t clo = ~0u, chi = 0u;
#pragma unroll
                for (int j = 0; j < NB; ++j) {
                    uint32_t lo = amn[j], hi = amx[j];
#pragma unroll
                    for (int o = 1; o < LPB; o <<= 1) {
                        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
                    }
                    if (row_on && on && (lane % LPB) == 0 &&
                        MTX_BC(((uint64_t)bz * a.GY + by) * a.GX + x0 / B + j, (uint64_t)a.GX * a.GY * a.GZ, kBcLeaf))
                        leaf[((uint64_t)bz * a.GY + by) * a.GX + x0 / B + j] = make_uint2(lo, hi);
                    amn[j] = smn[j];
                    amx[j] = smx[j];
                    clo = lo;
                    chi = hi;
                }
                if (l1) l1_close(clo, chi, bz);
                f_write(bz);
                fmn = c0mn;  // the closing slice opens the next block
                fmx = c0mx;
                ++bz;
            }
            __syncthreads();  // every warp is done with this stage
            if (s_fail) {
                ok = false;
                ++seq;
                break;
            }
            if (tid == 0) issue_next();
            if (pend) l1_finish();
        }
        if (ok && bz < bz1) {
            uint32_t clo = ~0u, chi = 0u;
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                uint32_t lo = amn[j], hi = amx[j];
#pragma unroll
                for (int o = 1; o < LPB; o <<= 1) {
                    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
                }
                if (row_on && on && (lane % LPB) == 0 &&
                    MTX_BC(((uint64_t)bz * a.GY + by) * a.GX + x0 / B + j, (uint64_t)a.GX * a.GY * a.GZ, kBcLeaf))
                    leaf[((uint64_t)bz * a.GY + by) * a.GX + x0 / B + j] = make_uint2(lo, hi);
                clo = lo;
                chi = hi;
            }
            f_write(bz);
            if (l1) {
                l1_close(clo, chi, bz);
                __syncthreads();
                if (pend) l1_finish();
            }
        }
    }
    // no copy may still be in flight into this CTA's shared memory when it exits
    if (tid == 0)
        for (; seq < issued; ++seq) mbar_wait_bounded(&bars[seq % S], (seq / S) & 1u);
}

// Merges each strip-start column record (the x halo the TMA leaf pass leaves
// out) into the last block of the strip before it: the leaf entry, and, when
// the leaf pass wrote octree level 1, the texel that holds that block.  One
// record per leaf entry; four records share a texel, hence the atomics there.
__global__ void __launch_bounds__(256) minmax_xface_patch_kernel(uint2 *__restrict__ leaf, uint2 *__restrict__ l1,
                                                                 const uint2 *__restrict__ xface, uint32_t GX,
                                                                 uint32_t GY, uint32_t GZ, uint32_t nS, uint32_t SB,
                                                                 uint32_t E1x, uint32_t E1y, uint32_t E1z) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)nS * GY * GZ) return;
    const uint32_t s = (uint32_t)(e % nS);
    const uint64_t rest = e / nS;
    const uint32_t by = (uint32_t)(rest % GY), bz = (uint32_t)(rest / GY);
    const uint32_t bx = (s + 1) * SB - 1;
    const uint2 f = xface[e];
    const uint64_t li = ((uint64_t)bz * GY + by) * GX + bx;
    if (bx < GX && MTX_BC(li, (uint64_t)GX * GY * GZ, kBcLeaf)) {
        const uint2 v = leaf[li];
        leaf[li] = make_uint2(min(v.x, f.x), max(v.y, f.y));
    }
    if (l1) {
        const uint32_t X1 = bx >> 1, Y1 = by >> 1, Z1 = bz >> 1;
        if (X1 < E1x && Y1 < E1y && Z1 < E1z) {
            uint2 *t = l1 + ((uint64_t)Z1 * E1y + Y1) * E1x + X1;
            atomicMin(&t->x, f.x);
            atomicMax(&t->y, f.y);
        }
    }
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

// Every octree level in one launch (minMaxOctreeReduce.comp.glsl:23-59 runs
// one dispatch per level): a CTA of 512 threads loads an 8^3 tile of the
// launch's first level (the leaf level, or level 1 when the leaf pass wrote
// it) and writes the 4^3, 2^3 and 1 texels it covers in the next three
// levels; the CTA that finishes last builds the rest from the third and
// zeroes the counter (zero since the context's creation) for the next
// launch.  Each texel is the min/max of its up-to-8 children; children past
// their level's extent are skipped (minMaxOctreeReduce.comp.glsl:37-47),
// which the identity {~0, 0} of the texels outside the first level's extent
// gives for free.  The tile stays at 8^3 (4 KB of shared memory) so that the
// CTAs fit beside the extraction kernels of other streams.
constexpr int kPyrMaxLevels = 32;
struct PyrAll {
    uint2 *base[kPyrMaxLevels];
    uint32_t ext[kPyrMaxLevels][3];
    int levels;
};

__global__ void __launch_bounds__(512) pyramid_all_kernel(const __grid_constant__ PyrAll L, uint32_t tiles_x,
                                                          uint32_t tiles_y, uint32_t ntiles, uint32_t *done) {
    __shared__ uint2 s[512];
    __shared__ uint32_t s_last;
    const uint32_t t = threadIdx.x;
    const uint32_t tx = blockIdx.x % tiles_x, ty = (blockIdx.x / tiles_x) % tiles_y, tz = blockIdx.x / (tiles_x * tiles_y);
    {
        const uint32_t x = tx * 8 + (t & 7), y = ty * 8 + ((t >> 3) & 7), z = tz * 8 + (t >> 6);
        uint2 v = make_uint2(~0u, 0u);
        if (x < L.ext[0][0] && y < L.ext[0][1] && z < L.ext[0][2])
            v = L.base[0][((uint64_t)z * L.ext[0][1] + y) * L.ext[0][0] + x];
        s[t] = v;
    }
    __syncthreads();
    const int top = min(3, L.levels - 1);
    uint32_t n = 8;  // current tile edge in shared memory
    for (int k = 1; k <= top; ++k) {
        const uint32_t m = n >> 1;
        uint2 r = make_uint2(~0u, 0u);
        const bool act = t < m * m * m;
        const uint32_t cx = t % m, cy = (t / m) % m, cz = t / (m * m);
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
            s[t] = r;  // compact m^3 layout for the next level
            const uint32_t ox = tx * m + cx, oy = ty * m + cy, oz = tz * m + cz;
            if (ox < L.ext[k][0] && oy < L.ext[k][1] && oz < L.ext[k][2])
                L.base[k][((uint64_t)oz * L.ext[k][1] + oy) * L.ext[k][0] + ox] = r;
        }
        __syncthreads();
        n = m;
    }
    if (L.levels <= 4) return;
    // level 3 of every tile is written: the last CTA to get here builds the rest
    __threadfence();
    __syncthreads();
    if (t == 0) s_last = atomicAdd(done, 1u) == ntiles - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int k = 4; k < L.levels; ++k) {
        const uint32_t ex = L.ext[k][0], ey = L.ext[k][1], ez = L.ext[k][2];
        const uint32_t px = L.ext[k - 1][0], py = L.ext[k - 1][1], pz = L.ext[k - 1][2];
        const uint64_t cnt = (uint64_t)ex * ey * ez;
        for (uint64_t i = t; i < cnt; i += 512) {
            const uint32_t x = (uint32_t)(i % ex), y = (uint32_t)((i / ex) % ey), z = (uint32_t)(i / ((uint64_t)ex * ey));
            uint2 r = make_uint2(~0u, 0u);
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const uint32_t ux = 2 * x + (c & 1), uy = 2 * y + ((c >> 1) & 1), uz = 2 * z + (c >> 2);
                if (ux < px && uy < py && uz < pz) {
                    const uint2 w = __ldcg(&L.base[k - 1][((uint64_t)uz * py + uy) * px + ux]);
                    r.x = min(r.x, w.x);
                    r.y = max(r.y, w.y);
                }
            }
            L.base[k][i] = r;
        }
        __threadfence();
        __syncthreads();
    }
    if (t == 0) *done = 0;
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

template <typename T, int B>
static mtx_status launch_tma(mtx_context *c, const Problem &p, uint2 *leaf, cudaStream_t s, uint32_t zover,
                             uint2 *l1, const uint32_t *l1ext, bool *l1_done) {
    constexpr uint32_t SEG = 32 * (16 / sizeof(T));
    CUtensorMap mmain;
    mtx_status r = make_volume_tensor_map_box(c, p, SEG, kTmaRows(B), 1, &mmain);
    if (r != MTX_OK) return r;
    TmaLeafArgs a;
    a.X = p.X; a.Y = p.Y; a.Z = p.Z;
    a.GX = p.GX; a.GY = p.GY; a.GZ = p.GZ;
    a.nXS = ceil_div(p.X, SEG);
    a.nYG = ceil_div(p.GY, 4);
    // slab runs of 128 voxel slices (a 1/129 halo repeat, and few item starts,
    // each of which refills the TMA ring), shorter when the volume is too small
    // to give every resident CTA an item.  On the 1024^3 uint16 volume at B = 8
    // (1024 items) three concurrent extractions take 1.465-1.482 ms against
    // 1.544-1.587 ms with runs of 32 slices.
    uint32_t zc = zover ? zover : std::max<uint32_t>(1, 128 / B);
    if (!zover)
        while (zc > 1 && (uint64_t)a.nXS * a.nYG * ceil_div(p.GZ, zc) < (uint64_t)kTmaCtasPerSm * c->sm_count)
        zc = (zc + 1) / 2;
    a.zchunk = zc;
    a.nZC = ceil_div(p.GZ, zc);
    a.nitems = a.nXS * a.nYG * a.nZC;
    // level 1 in the same pass: one block per lane (16 / sizeof(T) <= B) and z runs of whole pairs
    constexpr bool kOneBlockPerLane = 16 / sizeof(T) <= B;
    const bool with_l1 = kOneBlockPerLane && l1 && l1ext && zc % 2 == 0;
    for (int i = 0; i < 3; ++i) a.E1[i] = with_l1 ? l1ext[i] : 0u;
    if (l1_done) *l1_done = with_l1;
    const uint32_t smem = kTmaStages(B) * kTmaStage(B);
    auto k = minmax_leaf_tma_kernel<T, B>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(c, e, "minmax tma attribute");
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 128, smem);
    if (e != cudaSuccess) return cuda_fail(c, e, "minmax tma occupancy");
    occ = std::max(1, std::min(occ, kTmaCtasPerSm));
    const uint64_t nface = (uint64_t)(a.nXS - 1) * a.GY * a.GZ;  // strip-start column records
    if (nface && (r = scratch_reserve(c, c->xface, nface * sizeof(uint2))) != MTX_OK) return r;
    uint2 *xface = nface ? (uint2 *)c->xface.ptr : nullptr;
    const uint32_t grid = std::min<uint32_t>(a.nitems, (uint32_t)c->sm_count * (uint32_t)occ);
    k<<<grid, 128, smem, s>>>(mmain, a, leaf, with_l1 ? l1 : nullptr, xface, &c->ctrl->status);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "minmax tma launch");
    if (nface) {
        minmax_xface_patch_kernel<<<(unsigned)((nface + 255) / 256), 256, 0, s>>>(
            leaf, with_l1 ? l1 : nullptr, xface, a.GX, a.GY, a.GZ, a.nXS - 1, SEG / B, a.E1[0], a.E1[1], a.E1[2]);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(c, e, "minmax halo patch launch");
    }
    return MTX_OK;
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

mtx_status launch_minmax_leaf(mtx_context *c, const Problem &p, uint2 *leaf, cudaStream_t s, uint32_t zover,
                              uint2 *l1, const uint32_t *l1ext, bool *l1_done) {
    cudaError_t e;
    if (l1_done) *l1_done = false;
    if (!zover) zover = c->tuning.minmaxZChunk;
    const uint32_t sl = c->tuning.minmaxSlices;
    // TMA ring (the default for 2- and 4-byte voxels whose rows are 16-byte
    // aligned); the load-based body when tuning asks for 1, 2 or 4 slices
    const uint32_t esz = dtype_size(p.dtype);
    const bool tma = sl == 0 && esz >= 2 && (uintptr_t)p.vol % 16 == 0 && ((uint64_t)p.X * esz) % 16 == 0 &&
                     (p.B == 4 || p.B == 8 || p.B == 16);
    if (tma) {
        if (p.dtype == MTX_DTYPE_U16) {
            switch (p.B) {
            case 4: return launch_tma<uint16_t, 4>(c, p, leaf, s, zover, l1, l1ext, l1_done);
            case 8: return launch_tma<uint16_t, 8>(c, p, leaf, s, zover, l1, l1ext, l1_done);
            default: return launch_tma<uint16_t, 16>(c, p, leaf, s, zover, l1, l1ext, l1_done);
            }
        }
        switch (p.B) {
        case 4: return launch_tma<float, 4>(c, p, leaf, s, zover, l1, l1ext, l1_done);
        case 8: return launch_tma<float, 8>(c, p, leaf, s, zover, l1, l1ext, l1_done);
        default: return launch_tma<float, 16>(c, p, leaf, s, zover, l1, l1ext, l1_done);
        }
    }
    switch (p.dtype) {
    case MTX_DTYPE_U8: e = dispatch_leaf<uint8_t>(p, leaf, s, c->sm_count, zover, sl); break;
    case MTX_DTYPE_U16: e = dispatch_leaf<uint16_t>(p, leaf, s, c->sm_count, zover, sl); break;
    default: e = dispatch_leaf<float>(p, leaf, s, c->sm_count, zover, sl); break;
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "minmax leaf launch");
    return MTX_OK;
}

mtx_status launch_pyramid(mtx_context *c, uint2 *all, int levels, const uint32_t ext[][3],
                          const uint64_t *offset, cudaStream_t s, int start) {
    if (levels - start < 2) return MTX_OK;
    if (levels > kPyrMaxLevels) return fail(c, MTX_ERR_UNSUPPORTED, "too many mip levels");
    PyrAll P;
    memset(&P, 0, sizeof(P));
    P.levels = levels - start;
    for (int k = 0; k < P.levels; ++k) {
        P.base[k] = all + offset[start + k];
        for (int a = 0; a < 3; ++a) P.ext[k][a] = ext[start + k][a];
    }
    const uint32_t tx = ceil_div(P.ext[0][0], 8), ty = ceil_div(P.ext[0][1], 8), tz = ceil_div(P.ext[0][2], 8);
    pyramid_all_kernel<<<tx * ty * tz, 512, 0, s>>>(P, tx, ty, tx * ty * tz, &c->ctrl->pyr_done);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "pyramid launch");
    return MTX_OK;
}

MTX_BC_READER(bc_take_minmax)

}  // namespace mtx
