// Device building blocks of the PMB marching-cubes passes, shared by the
// single-volume kernels (extract.cu) and the batched kernel (batched.cu):
// per-warp shared-memory plans, tile staging, inside bitmasks, PMB edge
// ownership by bit operations, the per-block count and emit bodies, and the
// decoupled look-back used by the scans.
//
// Output order is canonical and equals the CPU oracle's: vertices by (block
// rank, owner voxel x-fastest in the block, axis x<y<z); triangles by (block
// rank, cell x-fastest in the block, triangle number in the case).
#pragma once

#include <algorithm>
#include <cstring>

#include "mtx_internal.h"

namespace mtx {

// Each translation unit has its own copy (no relocatable device code); load
// them with load_case_tables() before the first launch from that unit.
static __constant__ uint64_t c_mc_cases[256];
static __constant__ uint8_t c_mc_owner[12];

static mtx_status load_case_tables(mtx_context *c) {
    static bool loaded[128] = {false};
    if (c->device >= 0 && c->device < 128 && loaded[c->device]) return MTX_OK;
    MTX_CUDA(c, cudaMemcpyToSymbol(c_mc_cases, MTX_MC_CASES, sizeof(MTX_MC_CASES)));
    MTX_CUDA(c, cudaMemcpyToSymbol(c_mc_owner, MTX_MC_EDGE_OWNER, sizeof(MTX_MC_EDGE_OWNER)));
    if (c->device >= 0 && c->device < 128) loaded[c->device] = true;
    return MTX_OK;
}

constexpr uint32_t kNoVertex = 0xffffffffu;
// packed cases (2048 B), triangle counts (256 B), owners (16 B), the emit
// pass's edge offsets (24 B, edge_offsets), rounded up so that every warp's
// region -- and the TMA tile at its start -- is 128-byte aligned
constexpr uint32_t kTableBytes = 2432;
static_assert(kTableBytes % 128 == 0 && kTableBytes >= 2048 + 256 + 16 + 24, "table region must keep warp regions aligned");
constexpr uint32_t kJobWin = 256;                   // jobs (vertices or triangles) resolved per window
constexpr int kMaxWarps = 8;                        // warps per CTA of the extraction kernels

__host__ __device__ inline uint32_t align_up(uint32_t v, uint32_t a) { return (v + a - 1) / a * a; }

// Bytes of a CTA's shared memory before its warps' regions: the case tables,
// and for the emit pass the context-layer map (ctx_map_entry, one word per
// voxel of the (B+1)^3 context outside the block).
__host__ __device__ inline uint32_t cta_fixed_bytes(uint32_t B, bool emit) {
    return kTableBytes + (emit ? align_up(4 * (3 * B * B + 3 * B + 1), 128) : 0u);
}

// ------------------------------------------------------- per-warp smem plan
struct WPlan {
    uint32_t B, B1, BB, PX, nbuf, nb3;
    uint32_t rB, rB1, rBB;  // ceil(2^32 / d) reciprocals: n / d == __umulhi(n, r) for the sizes used here
    uint32_t R;             // block rows walked per round of 32 lanes (32 / B)
    uint32_t off_tile[2], off_bar, off_rows, off_cross, off_vp, off_tp, off_nvid, off_nm, off_jobs;
    uint32_t off_case, off_mm;  // case byte of each mixed cell, mixed-cell mask of each cell row (kept)
    uint32_t state_bytes;       // block state handed from count to emit (B <= 8): [off_cross, off_mm + 2BB)
    uint32_t off_vtab, off_vmsk, off_list;  // balanced bodies only (pmb_balanced.cuh)
    uint32_t bytes;       // per warp
    uint32_t tile_bytes;  // one tile (the TMA transaction size)
};

__host__ __device__ inline uint32_t tile_pitch(uint32_t B, uint32_t esz, bool tma) {
    if (!tma) return B + 1;
    const uint32_t A = 16 / esz;  // elements per 16 bytes
    uint32_t g = 1;
    for (uint32_t d = 1; d <= A; ++d)
        if (B % d == 0 && A % d == 0) g = d;
    const uint32_t xoff_max = (B % A == 0) ? 0 : A - g;
    return align_up(xoff_max + B + 1, A);
}

// tri_pass: the emit pass's plan.  keep: room for the case bytes and mixed
// masks (always in the emit pass); for B <= 8 the count pass keeps them too
// and hands the block state -- crossing rows, row prefixes, case bytes and
// mixed masks, one contiguous range -- to the emit pass through global memory.
__host__ __device__ inline WPlan make_wplan(uint32_t B, uint32_t esz, bool tma, bool tri_pass,
                                            bool single_buffer = false, bool keep = false) {
    WPlan p{};
    p.B = B;
    p.B1 = B + 1;
    p.BB = B * B;
    p.nb3 = 3 * B * B + 3 * B + 1;  // voxels of the (B+1)^3 context outside the block
    p.rB = (uint32_t)((0x100000000ull + B - 1) / B);
    p.rB1 = (uint32_t)((0x100000000ull + B) / (B + 1));
    p.rBB = (uint32_t)((0x100000000ull + B * B - 1) / (B * B));
    p.R = 32 / B;
    p.PX = tile_pitch(B, esz, tma);
    p.tile_bytes = p.PX * p.B1 * p.B1 * esz;
    p.nbuf = (p.tile_bytes <= 4096 && !single_buffer) ? 2 : 1;
    // the emit pass puts its vertex table (build_utab, B <= 8) in the tile's slot
    const uint32_t slot = (tri_pass && B <= 8) ? std::max(p.tile_bytes, 3 * p.B1 * p.B1 * p.B1) : p.tile_bytes;
    uint32_t o = 0;
    for (uint32_t b = 0; b < 2; ++b) {  // a TMA destination is 128-byte aligned; what follows the last, 16
        p.off_tile[b] = o;
        if (b < p.nbuf) o = align_up(o + slot, b + 1 < p.nbuf ? 128 : 16);
    }
    if (p.nbuf == 1) p.off_tile[1] = p.off_tile[0];
    p.off_bar = o;
    o += 16;
    if (tri_pass && B <= 8) o += 32;  // first vertex of the block and of its seven +x/+y/+z neighbours (emit)
    p.off_rows = o;
    // the emit pass with TMA and B <= 8 takes the count pass's block state and builds no rows
    if (!(tri_pass && tma && B <= 8)) o = align_up(o + 4 * p.B1 * p.B1, 16);
    p.off_cross = o;
    o = align_up(o + 12 * p.BB, 16);
    p.off_vp = o;
    o = align_up(o + 4 * p.BB, 16);
    p.off_tp = o;
    o = align_up(o + 4 * p.BB, 16);
    if (tri_pass || keep) {
        p.off_case = o;
        o = align_up(o + B * B * B, 16);
        p.off_mm = o;
        o = align_up(o + 2 * B * B, 16);
        p.state_bytes = B <= 8 ? o - p.off_cross : 0u;
    }
    if (tri_pass) {  // context first vertices: 16-bit packed entries for B <= 8 (gather_finish<CPL, true>)
        p.off_nvid = o;
        o = align_up(o + (B <= 8 ? 2 : 4) * p.nb3, 16);
        p.off_nm = o;  // owned-edge masks (B > 8; packed into the entries for B <= 8)
        if (B > 8) o = align_up(o + p.nb3, 16);
    }
    p.off_jobs = o;  // a window of packed jobs (triangles or vertices) in output order: the emit pass only
    if (tri_pass) o = align_up(o + 4 * kJobWin, 16);
    p.bytes = align_up(o, 128);
    return p;
}

// n / d and n % d for the block-local sizes (n < 70000, 2 <= d < 300), exact.
__device__ __forceinline__ uint32_t fdiv(uint32_t n, uint32_t r) { return __umulhi(n, r); }
__device__ __forceinline__ uint32_t fmod(uint32_t n, uint32_t r, uint32_t d) { return n - __umulhi(n, r) * d; }

struct Geo {
    uint32_t ox, oy, oz;  // block origin (voxels)
    uint32_t bx, by, bz;
    uint32_t nx;          // voxels of the block inside the volume along x (<= B)
    uint32_t xoff;        // tile column of the block's first voxel
};

// Exact division of a block id by the grid's row and slice sizes through a
// 64-bit reciprocal and one high multiply (Lemire's method: m = floor((2^64 - 1)
// / d) + 1 gives floor(a / d) = high 64 bits of m * a for every 32-bit a; d = 1
// is taken apart), computed once per thread instead of two integer divisions
// per block.
struct GridDiv {
    uint64_t mx, mxy;
    uint32_t dx, dxy;
};
__host__ __device__ inline GridDiv grid_div(const Problem &p) {
    GridDiv d;
    d.dx = p.GX;
    d.dxy = p.GX * p.GY;
    d.mx = d.dx > 1 ? ~0ull / d.dx + 1 : 0;
    d.mxy = d.dxy > 1 ? ~0ull / d.dxy + 1 : 0;
    return d;
}
__device__ __forceinline__ uint32_t div_by(uint32_t a, uint64_t m, uint32_t d) {
    return d > 1 ? (uint32_t)__umul64hi(m, a) : a;
}

__device__ __forceinline__ Geo block_geo(uint32_t id, const Problem &p, bool tma, uint32_t esz, const GridDiv &dv) {
    Geo g;
    g.bz = div_by(id, dv.mxy, dv.dxy);
    const uint32_t rest = id - g.bz * dv.dxy;
    g.by = div_by(rest, dv.mx, dv.dx);
    g.bx = rest - g.by * dv.dx;
    g.ox = g.bx * p.B;
    g.oy = g.by * p.B;
    g.oz = g.bz * p.B;
    g.nx = min(p.B, p.X - g.ox);
    g.xoff = tma ? (g.ox % (16 / esz)) : 0u;
    return g;
}

__device__ __forceinline__ Geo block_geo(uint32_t id, const Problem &p, bool tma, uint32_t esz) {
    Geo g;
    g.bx = id % p.GX;
    g.by = (id / p.GX) % p.GY;
    g.bz = id / (p.GX * p.GY);
    g.ox = g.bx * p.B;
    g.oy = g.by * p.B;
    g.oz = g.bz * p.B;
    g.nx = min(p.B, p.X - g.ox);
    g.xoff = tma ? (g.ox % (16 / esz)) : 0u;
    return g;
}

// ----------------------------------------------------------- warp tiles
// Starts the load of a block's (B+1)^3 tile into buffer `buf`.  TMA: lane 0
// issues one cp.async.bulk.tensor (zero fill outside the volume).  Plain
// loads are done in tile_wait instead.
// state: also bring the block's state (pl.state_bytes from global memory)
// into [off_cross, ...) on the same barrier (TMA only).
template <typename T, bool TMA>
__device__ __forceinline__ void tile_issue(const WPlan &pl, unsigned char *ws, uint32_t buf, const Geo &g,
                                           const CUtensorMap *map, const unsigned char *state = nullptr) {
    if (!TMA) return;
    __syncwarp();
    if ((threadIdx.x & 31) == 0) {
        uint64_t *bar = reinterpret_cast<uint64_t *>(ws + pl.off_bar) + buf;
        fence_proxy_async();  // earlier generic reads of this buffer come first
        mbar_arrive_expect_tx(bar, pl.tile_bytes + (state ? pl.state_bytes : 0u));
        tma_load_3d(ws + pl.off_tile[buf], map, bar, (int)(g.ox - g.xoff), (int)g.oy, (int)g.oz);
        if (state) bulk_load(ws + pl.off_cross, state, pl.state_bytes, bar);
    }
}

template <typename T, bool TMA>
__device__ __forceinline__ bool tile_wait(const Problem &p, const WPlan &pl, unsigned char *ws, uint32_t buf,
                                          const Geo &g, uint32_t &parity, DevStatus *st) {
    if (TMA) {
        uint64_t *bar = reinterpret_cast<uint64_t *>(ws + pl.off_bar) + buf;
        const bool ok = mbar_wait_bounded(bar, (parity >> buf) & 1u);
        if (!__all_sync(0xffffffffu, ok)) {
            if ((threadIdx.x & 31) == 0) report(st, MTX_ERR_TIMEOUT, kSiteTmaWait, g.ox, g.oy);
            // give the copy in flight one more bounded wait before the warp leaves
            mbar_wait_bounded(bar, (parity >> buf) & 1u);
            parity ^= 1u << buf;
            return false;
        }
        parity ^= 1u << buf;
        return true;
    }
    // plain loads, kLdgBatch per lane in flight before any is stored
    constexpr uint32_t kLdgBatch = 8;
    T *tile = reinterpret_cast<T *>(ws + pl.off_tile[buf]);
    const T *vol = reinterpret_cast<const T *>(p.vol);
    const uint32_t n = pl.B1 * pl.B1 * pl.B1;
    for (uint32_t i0 = 0; i0 < n; i0 += 32 * kLdgBatch) {
        T v[kLdgBatch];
        uint32_t dst[kLdgBatch];
#pragma unroll
        for (uint32_t k = 0; k < kLdgBatch; ++k) {
            const uint32_t i = i0 + k * 32 + (threadIdx.x & 31);
            const uint32_t iq = fdiv(i, pl.rB1);
            const uint32_t x = i - iq * pl.B1, z = fdiv(iq, pl.rB1), y = iq - z * pl.B1;
            const uint32_t gx = g.ox + x, gy = g.oy + y, gz = g.oz + z;
            v[k] = T(0);
            dst[k] = i < n ? (z * pl.B1 + y) * pl.PX + x : 0xffffffffu;
            if (i < n && gx < p.X && gy < p.Y && gz < p.Z) v[k] = __ldg(vol + ((uint64_t)gz * p.Y + gy) * p.X + gx);
        }
#pragma unroll
        for (uint32_t k = 0; k < kLdgBatch; ++k)
            if (dst[k] != 0xffffffffu && MTX_BC(dst[k], pl.PX * pl.B1 * pl.B1, kBcTile)) tile[dst[k]] = v[k];
    }
    __syncwarp();
    return true;
}

// Plain loads of a block's (B+1)^3 tile from a volume of run-time dtype
// p.dtype, stored as float (exact for uint8 and uint16), so that one set of
// block bodies serves every dtype.
template <typename S>
__device__ __forceinline__ void tile_load_float_from(const Problem &p, const WPlan &pl, float *tile, const Geo &g) {
    constexpr uint32_t kLdgBatch = 8;
    const S *vol = reinterpret_cast<const S *>(p.vol);
    const uint32_t n = pl.B1 * pl.B1 * pl.B1;
    for (uint32_t i0 = 0; i0 < n; i0 += 32 * kLdgBatch) {
        float v[kLdgBatch];
        uint32_t dst[kLdgBatch];
#pragma unroll
        for (uint32_t k = 0; k < kLdgBatch; ++k) {
            const uint32_t i = i0 + k * 32 + (threadIdx.x & 31);
            const uint32_t iq = fdiv(i, pl.rB1);
            const uint32_t x = i - iq * pl.B1, z = fdiv(iq, pl.rB1), y = iq - z * pl.B1;
            const uint32_t gx = g.ox + x, gy = g.oy + y, gz = g.oz + z;
            v[k] = 0.0f;
            dst[k] = i < n ? (z * pl.B1 + y) * pl.PX + x : 0xffffffffu;
            if (i < n && gx < p.X && gy < p.Y && gz < p.Z)
                v[k] = Vox<S>::val(__ldg(vol + ((uint64_t)gz * p.Y + gy) * p.X + gx));
        }
#pragma unroll
        for (uint32_t k = 0; k < kLdgBatch; ++k)
            if (dst[k] != 0xffffffffu && MTX_BC(dst[k], pl.PX * pl.B1 * pl.B1, kBcTile)) tile[dst[k]] = v[k];
    }
    __syncwarp();
}

__device__ __forceinline__ void tile_load_float(const Problem &p, const WPlan &pl, float *tile, const Geo &g) {
    if (p.dtype == MTX_DTYPE_U8) tile_load_float_from<uint8_t>(p, pl, tile, g);
    else if (p.dtype == MTX_DTYPE_U16) tile_load_float_from<uint16_t>(p, pl, tile, g);
    else tile_load_float_from<float>(p, pl, tile, g);
}

// Waits (bounded) for a prefetched tile that will not be used, so that no
// copy into this warp's shared memory is in flight when it leaves.
template <bool TMA>
__device__ __forceinline__ void tile_drain(const WPlan &pl, unsigned char *ws, uint32_t buf, uint32_t &parity) {
    if (!TMA) return;
    uint64_t *bar = reinterpret_cast<uint64_t *>(ws + pl.off_bar) + buf;
    mbar_wait_bounded(bar, (parity >> buf) & 1u);
    parity ^= 1u << buf;
}

// Inside bitmask of every tile row: bit x <=> voxel at or below iso and inside
// the volume.  Integer voxels compare against floor(iso); rows that start on a
// 4-byte boundary are tested 2 (uint16) or 4 (uint8) voxels per instruction.
template <typename T>
__device__ __forceinline__ void build_rows(const Problem &p, const WPlan &pl, unsigned char *ws, uint32_t buf,
                                           const Geo &g) {
    const T *tile = reinterpret_cast<const T *>(ws + pl.off_tile[buf]);
    uint32_t *rows = reinterpret_cast<uint32_t *>(ws + pl.off_rows);
    const uint32_t xin = min(pl.B1, p.X - g.ox);
    const uint32_t xmask = (1u << xin) - 1u;  // xin <= 17
    // integer voxels: value <= iso  <=>  value <= floor(iso) (never when iso < 0 or NaN)
    const bool never = !(p.iso >= 0.0f);
    const uint32_t thr = never ? 0u : (uint32_t)fminf(floorf(p.iso), sizeof(T) == 1 ? 255.0f : 65535.0f);
    const bool simd = Vox<T>::code != 2 && ((pl.PX * sizeof(T)) % 4 == 0) && ((g.xoff * sizeof(T)) % 4 == 0);
    for (uint32_t q = threadIdx.x & 31; q < pl.B1 * pl.B1; q += 32) {
        const uint32_t z = fdiv(q, pl.rB1), y = q - z * pl.B1;
        uint32_t m = 0;
        if (g.oy + y < p.Y && g.oz + z < p.Z &&
            MTX_BC((z * pl.B1 + y) * pl.PX + g.xoff + xin, pl.PX * pl.B1 * pl.B1 + 1, kBcTile)) {
            const T *r = tile + (z * pl.B1 + y) * pl.PX + g.xoff;
            if (Vox<T>::code == 2) {
                for (uint32_t x = 0; x < xin; ++x) m |= (Vox<T>::val(r[x]) <= p.iso ? 1u : 0u) << x;
            } else if (never) {
                m = 0;
            } else if (simd && sizeof(T) == 2) {
                const uint32_t *w = reinterpret_cast<const uint32_t *>(r);
                const uint32_t t2 = thr | (thr << 16);
                for (uint32_t i = 0; 2 * i < xin; ++i) {
                    const uint32_t c = __vcmpleu2(w[i], t2) & 0x00010001u;
                    m |= ((c | (c >> 15)) & 3u) << (2 * i);
                }
                m &= xmask;
            } else if (simd && sizeof(T) == 1) {
                const uint32_t *w = reinterpret_cast<const uint32_t *>(r);
                const uint32_t t4 = thr * 0x01010101u;
                for (uint32_t i = 0; 4 * i < xin; ++i) {
                    const uint32_t c = __vcmpleu4(w[i], t4) & 0x01010101u;
                    m |= ((c * 0x01020408u) >> 24) << (4 * i);
                }
                m &= xmask;
            } else {
                for (uint32_t x = 0; x < xin; ++x) m |= ((uint32_t)r[x] <= thr ? 1u : 0u) << x;
            }
        }
        if (MTX_BC(q, pl.B1 * pl.B1, kBcRows)) rows[q] = m;
    }
    __syncwarp();
}

// Crossing masks of owned voxel row (y, z) (bit x of xc/yc/zc: the +x/+y/+z
// edge owned by voxel (x, y, z) is cut) from the inside bitmasks.
__device__ __forceinline__ void row_cross(const Problem &p, const WPlan &pl, const Geo &g, const uint32_t *rows,
                                          uint32_t y, uint32_t z, uint32_t &xc, uint32_t &yc, uint32_t &zc) {
    xc = yc = zc = 0;
    if (g.oy + y >= p.Y || g.oz + z >= p.Z) return;
    const uint32_t own = (1u << g.nx) - 1u;
    const uint32_t r0 = rows[z * pl.B1 + y];
    const uint32_t xe = p.X - g.ox - 1;  // +x edges exist for x < X - ox - 1
    const uint32_t xmask = xe >= 32 ? 0xffffffffu : ((1u << xe) - 1u);
    xc = (r0 ^ (r0 >> 1)) & own & xmask;
    if (g.oy + y + 1 < p.Y) yc = (r0 ^ rows[z * pl.B1 + y + 1]) & own;
    if (g.oz + z + 1 < p.Z) zc = (r0 ^ rows[(z + 1) * pl.B1 + y]) & own;
}

// Case index of the cell at (x, y, z) from the inside bitmasks (corner order
// of marching_cubes_pmb.mesh.glsl:84-93: r00 = row (y,z), r01 = (y+1,z),
// r10 = (y,z+1), r11 = (y+1,z+1)).
__device__ __forceinline__ uint32_t cell_case(const uint32_t *rows, uint32_t B1, uint32_t x, uint32_t y, uint32_t z) {
    const uint32_t r00 = rows[z * B1 + y] >> x, r01 = rows[z * B1 + y + 1] >> x;
    const uint32_t r10 = rows[(z + 1) * B1 + y] >> x, r11 = rows[(z + 1) * B1 + y + 1] >> x;
    return (r00 & 1u) | (r00 & 2u) | ((r01 & 2u) << 1) | ((r01 & 1u) << 3) | ((r10 & 1u) << 4) |
           ((r10 & 2u) << 4) | ((r11 & 2u) << 5) | ((r11 & 1u) << 7);
}

// Whether the cell at (x, y, z) of the block lies inside the volume.
__device__ __forceinline__ bool cell_valid(const Problem &p, const Geo &g, uint32_t x, uint32_t y, uint32_t z) {
    return g.ox + x + 1 < p.X && g.oy + y + 1 < p.Y && g.oz + z + 1 < p.Z;
}

__device__ __forceinline__ uint32_t warp_excl_scan(uint32_t v, uint32_t &total) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}

// Cells x of cell row (y, z) whose case is neither 0 nor 255 (bit x set), and
// those that are entirely inside (all 8 corners at or below iso).
__device__ __forceinline__ uint32_t mixed_cells(const Problem &p, const WPlan &pl, const Geo &g, const uint32_t *rows,
                                                uint32_t y, uint32_t z, uint32_t &all_inside) {
    all_inside = 0;
    if (g.oy + y + 1 >= p.Y || g.oz + z + 1 >= p.Z || g.ox + 1 >= p.X) return 0;
    const uint32_t ncell = min(pl.B, p.X - 1 - g.ox), B1 = pl.B1;
    const uint32_t cells = (1u << ncell) - 1u;
    const uint32_t r00 = rows[z * B1 + y], r01 = rows[z * B1 + y + 1];
    const uint32_t r10 = rows[(z + 1) * B1 + y], r11 = rows[(z + 1) * B1 + y + 1];
    const uint32_t all = r00 & r01 & r10 & r11, any = r00 | r01 | r10 | r11;
    all_inside = all & (all >> 1) & cells;
    return (any | (any >> 1)) & ~(all & (all >> 1)) & cells;
}

// Per-row crossing masks, vertex prefixes and (want_tris) triangle prefixes,
// and the block's vertex/triangle counts.  Lane l owns rows [l*R, l*R + R) so
// that the row prefixes follow from one warp scan.  Optionally writes the
// per-cell case bytes (cases_out: every cell, 0 / 255 for cells that are not
// mixed) and keeps, in the warp's shared memory, the mixed-cell mask of each
// cell row and the case byte of each mixed cell (keep: the emit pass).
__device__ __forceinline__ void block_counts(const Problem &p, const WPlan &pl, unsigned char *ws, const Geo &g,
                                             const uint8_t *ntab, bool want_tris, uint8_t *cases_out,
                                             uint32_t &nv, uint32_t &nt, bool keep = false) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t *rows = reinterpret_cast<const uint32_t *>(ws + pl.off_rows);
    uint32_t *cross = reinterpret_cast<uint32_t *>(ws + pl.off_cross);
    uint32_t *vp = reinterpret_cast<uint32_t *>(ws + pl.off_vp);
    uint32_t *tp = reinterpret_cast<uint32_t *>(ws + pl.off_tp);
    const uint32_t B = pl.B, BB = pl.BB;
    const uint32_t R = (BB + 31) / 32;
    uint32_t sv = 0, stri = 0;
    for (uint32_t k = 0; k < R; ++k) {
        const uint32_t q = lane * R + k;
        if (q >= BB) break;
        const uint32_t z = fdiv(q, pl.rB), y = q - z * B;
        uint32_t xc, yc, zc;
        row_cross(p, pl, g, rows, y, z, xc, yc, zc);
        cross[q] = xc;
        cross[BB + q] = yc;
        cross[2 * BB + q] = zc;
        vp[q] = sv;  // lane-local prefixes, rebased below
        sv += __popc(xc) + __popc(yc) + __popc(zc);
        if (want_tris) {
            tp[q] = stri;
            uint32_t inside;
            uint32_t mm = mixed_cells(p, pl, g, rows, y, z, inside);
            if (cases_out)
                for (uint32_t x = 0; x < B; ++x) cases_out[q * B + x] = ((inside >> x) & 1u) ? 255 : 0;
            if (keep) reinterpret_cast<uint16_t *>(ws + pl.off_mm)[q] = (uint16_t)mm;
            // the four rows of the cell row, read once for all its mixed cells
            const uint32_t r00 = mm ? rows[z * pl.B1 + y] : 0u, r01 = mm ? rows[z * pl.B1 + y + 1] : 0u;
            const uint32_t r10 = mm ? rows[(z + 1) * pl.B1 + y] : 0u, r11 = mm ? rows[(z + 1) * pl.B1 + y + 1] : 0u;
            while (mm) {
                const uint32_t x = __ffs(mm) - 1;
                mm &= mm - 1u;
                const uint32_t a = r00 >> x, b = r01 >> x, c = r10 >> x, e = r11 >> x;
                const uint32_t cfg = (a & 3u) | ((b & 2u) << 1) | ((b & 1u) << 3) | ((c & 3u) << 4) | ((e & 2u) << 5) |
                                     ((e & 1u) << 7);
                stri += ntab[cfg];
                if (!MTX_BC(q * B + x, B * BB, kBcRows)) continue;
                if (cases_out) cases_out[q * B + x] = (uint8_t)cfg;
                if (keep) ws[pl.off_case + q * B + x] = (uint8_t)cfg;
            }
        }
    }
    uint32_t tv, tt;
    const uint32_t pv = warp_excl_scan(sv, tv);
    const uint32_t pt = warp_excl_scan(stri, tt);
    for (uint32_t k = 0; k < R; ++k) {
        const uint32_t q = lane * R + k;
        if (q >= BB) break;
        vp[q] += pv;
        if (want_tris) tp[q] += pt;
    }
    __syncwarp();
    nv = tv;
    nt = tt;
}

// Owned-edge mask of voxel (x, y, z) of the block, from the crossing rows.
__device__ __forceinline__ uint32_t voxel_mask(const uint32_t *cross, uint32_t BB, uint32_t q, uint32_t x) {
    return ((cross[q] >> x) & 1u) | (((cross[BB + q] >> x) & 1u) << 1) | (((cross[2 * BB + q] >> x) & 1u) << 2);
}

// Block-relative index of the first vertex owned by voxel (x, y, z).
__device__ __forceinline__ uint32_t voxel_prefix(const uint32_t *cross, const uint32_t *vp, uint32_t BB, uint32_t q,
                                                 uint32_t x) {
    const uint32_t below = (1u << x) - 1u;
    return vp[q] + __popc(cross[q] & below) + __popc(cross[BB + q] & below) + __popc(cross[2 * BB + q] & below);
}

// ------------------------------------------------------------- numerics
// Edge parameter (marching_cubes_pmb.mesh.glsl:129-134): t = (iso - a)/(b - a)
// when |b - a| > 1e-5 else 0.5, clamped to [0, 1]; every operation rounds once.
__device__ __forceinline__ float edge_t(float fa, float fb, float iso) {
    const float den = __fsub_rn(fb, fa);
    float t = 0.5f;
    if (fabsf(den) > 1e-5f) t = __fdiv_rn(__fsub_rn(iso, fa), den);
    t = t < 0.0f ? 0.0f : t;
    t = t > 1.0f ? 1.0f : t;
    return t;
}

template <typename T>
__device__ __forceinline__ float gval(const Problem &p, uint32_t x, uint32_t y, uint32_t z) {
    const T *vol = reinterpret_cast<const T *>(p.vol);
    return Vox<T>::val(__ldg(vol + ((uint64_t)z * p.Y + y) * p.X + x));
}

__device__ __forceinline__ void normalize3(float &a, float &b, float &c) {
    float d = __fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b));
    d = __fadd_rn(d, __fmul_rn(c, c));
    if (d == 0.0f) {
        a = b = c = 0.0f;
        return;
    }
    const float l = __fsqrt_rn(d);
    a = __fdiv_rn(a, l);
    b = __fdiv_rn(b, l);
    c = __fdiv_rn(c, l);
}

// Clamped central difference, normalised (calculate_normal, pmb.mesh.glsl:111-120).
template <typename T>
__device__ __forceinline__ void voxel_normal(const Problem &p, uint32_t x, uint32_t y, uint32_t z, float n[3]) {
    const uint32_t xl = x ? x - 1 : 0, xh = min(x + 1, p.X - 1);
    const uint32_t yl = y ? y - 1 : 0, yh = min(y + 1, p.Y - 1);
    const uint32_t zl = z ? z - 1 : 0, zh = min(z + 1, p.Z - 1);
    n[0] = __fsub_rn(gval<T>(p, xl, y, z), gval<T>(p, xh, y, z));
    n[1] = __fsub_rn(gval<T>(p, x, yl, z), gval<T>(p, x, yh, z));
    n[2] = __fsub_rn(gval<T>(p, x, y, zl), gval<T>(p, x, y, zh));
    normalize3(n[0], n[1], n[2]);
}

// Normal of the vertex at parameter t on the +axis edge of volume voxel
// (gx, gy, gz): normalize(mix(n1, n2, t)) (marching_cubes_pmb.mesh.glsl:126-137).
template <typename T>
__device__ __noinline__ float3 vertex_normal(const Problem &p, uint32_t gx, uint32_t gy, uint32_t gz, uint32_t a,
                                             float t) {
    float n1[3], n2[3];
    voxel_normal<T>(p, gx, gy, gz, n1);
    voxel_normal<T>(p, gx + (a == 0), gy + (a == 1), gz + (a == 2), n2);
    const float omt = __fsub_rn(1.0f, t);
    float3 n;
    n.x = __fadd_rn(__fmul_rn(n1[0], omt), __fmul_rn(n2[0], t));
    n.y = __fadd_rn(__fmul_rn(n1[1], omt), __fmul_rn(n2[1], t));
    n.z = __fadd_rn(__fmul_rn(n1[2], omt), __fmul_rn(n2[2], t));
    normalize3(n.x, n.y, n.z);
    return n;
}

// vertex_normal for a volume whose dtype is known only at run time (p.dtype).
static __device__ __noinline__ float3 vertex_normal_any(const Problem &p, uint32_t gx, uint32_t gy, uint32_t gz,
                                                        uint32_t a, float t) {
    if (p.dtype == MTX_DTYPE_U8) return vertex_normal<uint8_t>(p, gx, gy, gz, a, t);
    if (p.dtype == MTX_DTYPE_U16) return vertex_normal<uint16_t>(p, gx, gy, gz, a, t);
    return vertex_normal<float>(p, gx, gy, gz, a, t);
}

// Position of the vertex on the +axis edge of block voxel (x,y,z); its edge
// parameter goes to *tout.
template <typename T>
__device__ __forceinline__ float3 vertex_pos(const Problem &p, const WPlan &pl, const T *tile, const Geo &g, uint32_t x,
                                             uint32_t y, uint32_t z, uint32_t a, bool ndc, float *tout) {
    uint32_t i0 = (z * pl.B1 + y) * pl.PX + g.xoff + x;
    uint32_t i1 = i0 + (a == 0 ? 1u : a == 1 ? pl.PX : pl.PX * pl.B1);
    if (!MTX_BC(i1, pl.PX * pl.B1 * pl.B1, kBcTile)) i1 = i0 = 0;
    const float t = edge_t(Vox<T>::val(tile[i0]), Vox<T>::val(tile[i1]), p.iso);
    *tout = t;
    float3 pos = make_float3((float)(g.ox + x), (float)(g.oy + y), (float)(g.oz + z));
    if (a == 0) pos.x = __fadd_rn(pos.x, t);
    else if (a == 1) pos.y = __fadd_rn(pos.y, t);
    else pos.z = __fadd_rn(pos.z, t);
    if (ndc) {
        pos.x = __fsub_rn(__fmul_rn(__fdiv_rn(pos.x, (float)p.X), 2.0f), 1.0f);
        pos.y = __fsub_rn(__fmul_rn(__fdiv_rn(pos.y, (float)p.Y), 2.0f), 1.0f);
        pos.z = __fsub_rn(__fmul_rn(__fdiv_rn(pos.z, (float)p.Z), 2.0f), 1.0f);
    }
    return pos;
}


// Writes the block's own vertices (vbase .. vbase + nv) in canonical order.
// Each lane walks the cut edges of its rows and writes one job per vertex
// (voxel index | axis << 12) at the vertex's own position in a window of
// kJobWin jobs; the warp then resolves the window 32 vertices at a time, one
// per lane, each lane storing its own vertex record.
// GENERIC selects the VertexData / NDC / normals options; the plain form
// writes xyz in the voxel frame.  ANY: the tile holds the voxels converted to
// T = float and the volume's own dtype is p.dtype (used for the normals).
template <typename T, bool GENERIC, bool ANY = false>
__device__ __forceinline__ void emit_vertices(const Problem &p, const WPlan &pl, unsigned char *ws, uint32_t buf,
                                              const Geo &g, uint32_t vbase, uint32_t nv, void *vertices, uint32_t vfmt,
                                              uint32_t frame, uint32_t normals) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t B = pl.B, BB = pl.BB, R = (BB + 31) / 32;
    const uint32_t *cross = reinterpret_cast<const uint32_t *>(ws + pl.off_cross);
    const uint32_t *vp = reinterpret_cast<const uint32_t *>(ws + pl.off_vp);
    const T *tile = reinterpret_cast<const T *>(ws + pl.off_tile[buf]);
    uint32_t *jobs = reinterpret_cast<uint32_t *>(ws + pl.off_jobs);
    const bool xyz = !GENERIC || vfmt == MTX_VERTEX_XYZ;
    for (uint32_t w0 = 0; w0 < nv; w0 += kJobWin) {
        const uint32_t w1 = w0 + kJobWin;
        if (nv <= kJobWin) {  // one window (the common case): no window checks
            for (uint32_t k = 0; k < R; ++k) {
                const uint32_t q = lane * R + k;
                if (q >= BB) break;
                const uint32_t xc = cross[q], yc = cross[BB + q], zc = cross[2 * BB + q];
                uint32_t j = vp[q], any = xc | yc | zc;
                while (any) {
                    const uint32_t x = __ffs(any) - 1;
                    any &= any - 1u;
                    const uint32_t base = (q * B + x);
                    if ((xc >> x) & 1u) jobs[j++] = base;
                    if ((yc >> x) & 1u) jobs[j++] = base | (1u << 12);
                    if ((zc >> x) & 1u) jobs[j++] = base | (2u << 12);
                }
            }
        } else {
            for (uint32_t k = 0; k < R; ++k) {
                const uint32_t q = lane * R + k;
                if (q >= BB) break;
                const uint32_t xc = cross[q], yc = cross[BB + q], zc = cross[2 * BB + q];
                uint32_t j = vp[q];
                if (j >= w1 || j + __popc(xc) + __popc(yc) + __popc(zc) <= w0) continue;
                uint32_t any = xc | yc | zc;
                while (any) {
                    const uint32_t x = __ffs(any) - 1;
                    any &= any - 1u;
                    const uint32_t base = (q * B + x);
                    if ((xc >> x) & 1u) { if (j >= w0 && j < w1) jobs[j - w0] = base; ++j; }
                    if ((yc >> x) & 1u) { if (j >= w0 && j < w1) jobs[j - w0] = base | (1u << 12); ++j; }
                    if ((zc >> x) & 1u) { if (j >= w0 && j < w1) jobs[j - w0] = base | (2u << 12); ++j; }
                }
            }
        }
        __syncwarp();
        const uint32_t cnt = min(kJobWin, nv - w0);
        for (uint32_t b = 0; b < cnt; b += 32) {
            const uint32_t n = min(32u, cnt - b);
            if (lane < n && MTX_BC(w0 + b + lane, nv, kBcVertex)) {
                const uint32_t job = jobs[b + lane];
                const uint32_t i = job & 0xfffu, a = job >> 12;
                const uint32_t q = fdiv(i, pl.rB), x = i - q * B;
                const uint32_t z = fdiv(q, pl.rB), y = q - z * B;
                float t;
                const float3 pos =
                    vertex_pos<T>(p, pl, tile, g, x, y, z, a, GENERIC && frame == MTX_FRAME_NDC, &t);
                if (xyz) {  // each lane its own 12 bytes: L2 merges the warp's 384-byte span
                    float *o = reinterpret_cast<float *>(vertices) + 3ull * (vbase + w0 + b + lane);
                    o[0] = pos.x;
                    o[1] = pos.y;
                    o[2] = pos.z;
                } else {
                    float3 nn = make_float3(0.0f, 0.0f, 0.0f);
                    if (normals) {
                        if constexpr (ANY) nn = vertex_normal_any(p, g.ox + x, g.oy + y, g.oz + z, a, t);
                        else nn = vertex_normal<T>(p, g.ox + x, g.oy + y, g.oz + z, a, t);
                    }
                    float4 *v = reinterpret_cast<float4 *>(vertices) + 2ull * (vbase + w0 + b + lane);
                    v[0] = make_float4(pos.x, pos.y, pos.z, 1.0f);
                    v[1] = make_float4(nn.x, nn.y, nn.z, 0.0f);
                }
            }
            __syncwarp();
        }
    }
}

// -------------------------------------------------------------- emit pass
// Index of a voxel of the (B+1)^3 context outside the block (some coordinate == B).
__device__ __forceinline__ uint32_t ctx_index(uint32_t B, uint32_t x, uint32_t y, uint32_t z) {
    const uint32_t B1 = B + 1;
    if (x == B) return z * B1 + y;
    if (y == B) return B1 * B1 + z * B + x;
    return B1 * B1 + B * B1 + y * B + x;
}

// Context voxel of compact index j (inverse of ctx_index).
__device__ __forceinline__ void ctx_voxel(const WPlan &pl, uint32_t j, uint32_t &x, uint32_t &y, uint32_t &z) {
    const uint32_t B = pl.B, B1 = pl.B1;
    if (j < B1 * B1) {
        x = B;
        z = fdiv(j, pl.rB1);
        y = j - z * B1;
    } else if (j < B1 * B1 + B * B1) {
        const uint32_t i = j - B1 * B1;
        y = B;
        z = fdiv(i, pl.rB);
        x = i - z * B;
    } else {
        const uint32_t i = j - B1 * B1 - B * B1;
        z = B;
        y = fdiv(i, pl.rB);
        x = i - y * B;
    }
}

// Resolves the vertex id of edge e of the cell at block cell (x, y, z).
__device__ __forceinline__ uint32_t edge_vertex(uint32_t x, uint32_t y, uint32_t z, uint32_t e, const uint8_t *owner,
                                                const uint32_t *cross, const uint32_t *vp, const uint32_t *nvid,
                                                const uint8_t *nm, uint32_t B, uint32_t BB, uint32_t vbase,
                                                bool &bad) {
    const uint32_t own = owner[e];
    const uint32_t ux = x + (own & 1u), uy = y + ((own >> 1) & 1u), uz = z + ((own >> 2) & 1u);
    const uint32_t ax = own >> 3;
    uint32_t base, m;
    if (ux < B && uy < B && uz < B) {
        const uint32_t q = uz * B + uy;
        base = vbase + voxel_prefix(cross, vp, BB, q, ux);
        m = voxel_mask(cross, BB, q, ux);
    } else {
        const uint32_t jx = ctx_index(B, ux, uy, uz);
        if (!MTX_BC(jx, 3 * B * B + 3 * B + 1, kBcContext)) {
            bad = true;
            return 0;
        }
        base = nvid[jx];
        m = nm[jx];
    }
    if (base == kNoVertex || !((m >> ax) & 1u)) {
        bad = true;
        return 0;
    }
    return base + __popc(m & ((1u << ax) - 1u));
}

// Unified vertex table over the block's (B+1)^3 voxels for B <= 8, built in
// the tile's slot once the vertices are written: a 16-bit entry per voxel,
// the first vertex of the voxel relative to its block's first vertex (11
// bits) | the block's number c << 11 (0 = this block, 1-7 = the +x/+y/+z
// neighbour dx | dy << 1 | dz << 2), then a mask byte per voxel with its
// owned cut edges.  Own voxels come from the crossing rows; the context layer
// from the packed gather (gather_finish<CPL, true>).  A triangle corner is
// then one entry, one mask and one base word.  Only voxels that own a cut
// edge are written; triangle corners refer to no other.
__device__ __forceinline__ void build_utab(const WPlan &pl, unsigned char *ws, uint16_t *ut, uint8_t *um,
                                           const uint32_t *cmap) {
    const uint32_t lane = threadIdx.x & 31, B = pl.B, B1 = pl.B1, BB = pl.BB, R = (BB + 31) / 32;
    const uint32_t *cross = reinterpret_cast<const uint32_t *>(ws + pl.off_cross);
    const uint32_t *vp = reinterpret_cast<const uint32_t *>(ws + pl.off_vp);
    for (uint32_t k = 0; k < R; ++k) {
        const uint32_t q = lane * R + k;
        if (q >= BB) break;
        const uint32_t xc = cross[q], yc = cross[BB + q], zc = cross[2 * BB + q];
        const uint32_t z = fdiv(q, pl.rB), y = q - z * B, row = (z * B1 + y) * B1;
        uint32_t any = xc | yc | zc, run = vp[q];
        while (any) {
            const uint32_t x = __ffs(any) - 1;
            any &= any - 1u;
            const uint32_t m = ((xc >> x) & 1u) | (((yc >> x) & 1u) << 1) | (((zc >> x) & 1u) << 2);
            if (MTX_BC(row + x, B1 * B1 * B1, kBcVoxTab)) {
                ut[row + x] = (uint16_t)run;
                um[row + x] = (uint8_t)m;
            }
            run += __popc(m);
        }
    }
    const uint16_t *nvid = reinterpret_cast<const uint16_t *>(ws + pl.off_nvid);
    for (uint32_t j = lane; j < pl.nb3; j += 32) {
        const uint32_t e = cmap[j], v = nvid[j];
        const uint32_t ti = (((e >> 23) & 31u) * B1 + ((e >> 18) & 31u)) * B1 + ((e >> 13) & 31u);
        if (MTX_BC(ti, B1 * B1 * B1, kBcVoxTab)) {
            ut[ti] = (uint16_t)((v & 0x7ffu) | ((e & 7u) << 11));
            um[ti] = (uint8_t)(v >> 11);
        }
    }
    __syncwarp();
}

// Edge offsets of the unified table for one CTA (B <= 8): entry e holds the
// table offset of cube edge e's owner voxel from the cell's low corner,
// dx + dy (B+1) + dz (B+1)^2, and its axis << 8 (from the owner table).
__device__ __forceinline__ void edge_offsets(uint16_t *eoff, uint32_t B1) {
    if (threadIdx.x < 12) {
        const uint32_t o = c_mc_owner[threadIdx.x];
        eoff[threadIdx.x] = (uint16_t)((o & 1u) + ((o >> 1) & 1u) * B1 + ((o >> 2) & 1u) * B1 * B1 + ((o >> 3) << 8));
    }
}

// The vertex id of cube edge e of the cell whose low corner is tile voxel ti,
// from the unified table (build_utab); nbase: the eight block first vertices.
__device__ __forceinline__ uint32_t edge_vertex_ut(uint32_t ti, uint32_t e, const uint16_t *eoff, const uint16_t *ut,
                                                   const uint8_t *um, const uint32_t *nbase, uint32_t B1, bool &bad) {
    const uint32_t eo = eoff[e];
    const uint32_t i = ti + (eo & 0xffu), ax = eo >> 8;
    if (!MTX_BC(i, B1 * B1 * B1, kBcVoxTab)) {
        bad = true;
        return 0;
    }
    const uint32_t m = um[i], v = ut[i];
    bad |= !((m >> ax) & 1u);
    return nbase[v >> 11] + (v & 0x7ffu) + __popc(m & ((1u << ax) - 1u));
}

// -------------------------------------------------------------- scan pass
constexpr uint64_t kCnt31 = 0x7fffffffull;

// Warp-cooperative decoupled look-back over per-tile status words
// ([63:62] flag 1 aggregate / 2 inclusive / 3 aborted, [61:31] triangles,
// [30:0] vertices).  Publishes this tile's aggregate, then its inclusive
// prefix; returns the exclusive prefix, false if aborted.  Totals that do
// not fit 31 bits (or 3 x triangles that do not fit 32) abort with
// MTX_ERR_CAPACITY.
// Sums the (vertices, triangles) of the tile words before tile r, back to and
// including the first inclusive one, in windows of 32 read by the warp;
// false if a predecessor aborted or the wait timed out.
__device__ __forceinline__ bool lookback_sum31(const uint64_t *status, uint32_t r, uint64_t &ev, uint64_t &et,
                                               DevStatus *st, uint32_t spin_limit = kSpinLimit) {
    const uint32_t lane = threadIdx.x & 31;
    ev = et = 0;
    int64_t j = (int64_t)r - 1;
    uint32_t spins = 0;
    while (true) {
        const int64_t k = j - (int64_t)lane;
        const uint64_t w = k >= 0 ? ld_volatile(&status[k]) : (2ull << 62);
        const uint32_t flag = (uint32_t)(w >> 62);
        if (__any_sync(0xffffffffu, flag == 3u)) return false;
        const uint32_t inc = __ballot_sync(0xffffffffu, flag == 2u);
        const uint32_t emp = __ballot_sync(0xffffffffu, flag == 0u);
        const uint32_t first = inc ? (uint32_t)(__ffs(inc) - 1) : 32u;
        const uint32_t window = first >= 31 ? 0xffffffffu : ((2u << first) - 1u);
        if (emp & window) {
            if (++spins >= spin_limit) {
                if (lane == 0) report(st, MTX_ERR_TIMEOUT, kSiteCountLookback, r, (uint32_t)j);
                return false;
            }
            backoff(spins);
            continue;
        }
        uint64_t a = lane <= first ? (w & kCnt31) : 0ull;
        uint64_t b = lane <= first ? ((w >> 31) & kCnt31) : 0ull;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        ev += a;
        et += b;
        if (first < 32) return true;
        j -= 32;
    }
}

__device__ __forceinline__ bool lookback_counts(uint64_t *status, uint32_t r, uint32_t bnv, uint32_t bnt,
                                                uint64_t &ev, uint64_t &et, DevStatus *st,
                                                uint32_t spin_limit = kSpinLimit) {
    const uint32_t lane = threadIdx.x & 31;
    ev = et = 0;
    bool abort = false;
    if (r > 0) {
        if (lane == 0) st_volatile(&status[r], (1ull << 62) | ((uint64_t)bnt << 31) | bnv);
        abort = !lookback_sum31(status, r, ev, et, st, spin_limit);
    }
    const uint64_t iv = ev + bnv, it = et + bnt;
    if (!abort && (iv > kCnt31 || it > kCnt31 || 3ull * it > 0xffffffffull)) {
        if (lane == 0) report(st, MTX_ERR_CAPACITY, kSiteCountOverflow, (uint32_t)(iv >> 32), (uint32_t)it);
        abort = true;
    }
    if (lane == 0) st_volatile(&status[r], abort ? (3ull << 62) : ((2ull << 62) | (it << 31) | iv));
    return !abort;
}

// ----------------------------------------------------------- block bodies
// Data written earlier in the same launch must not be read through the
// read-only (non-coherent) cache; NC selects that path for data produced by
// an earlier launch, and L2-only loads are used otherwise.
template <bool NC, typename U>
__device__ __forceinline__ U ld_in(const U *p) {
    if constexpr (NC) return __ldg(p);
    else return __ldcg(p);
}

// Lane c in 1..7 returns the rank of neighbour block c = (dx, dy, dz) bits of
// block `id`, or kNoVertex when it is outside the grid or inactive.
template <bool NC = true>
__device__ __forceinline__ uint32_t neighbour_rank(const Problem &p, const Geo &g, uint32_t id,
                                                   const uint32_t *rank_map) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t rk = kNoVertex;
    if (lane >= 1 && lane < 8) {
        const uint32_t dx = lane & 1u, dy = (lane >> 1) & 1u, dz = lane >> 2;
        if (g.bx + dx < p.GX && g.by + dy < p.GY && g.bz + dz < p.GZ &&
            MTX_BC((uint64_t)id + dx + dy * p.GX + (uint64_t)dz * p.GX * p.GY, p.nblocks, kBcRank))
            rk = ld_in<NC>(rank_map + id + dx + dy * p.GX + dz * p.GX * p.GY);
    }
    return rk;
}

// Issues the loads of the face records of the block's +x/+y/+z context layer
// (all of them before any is used); bit 31 of rec marks a present record and
// bits 27-29 hold the number c of the neighbour it came from (face records
// use bits 0-26).
template <int CPL, bool NC = true>
__device__ __forceinline__ void gather_issue(const Problem &p, const WPlan &pl, const Geo &g, uint32_t nb_rk,
                                             const uint32_t *faces, uint32_t face_stride, uint32_t rec[CPL]) {
    const uint32_t lane = threadIdx.x & 31, B = pl.B, BB = pl.BB, nb3 = pl.nb3;
#pragma unroll
    for (uint32_t k = 0; k < CPL; ++k) {
        rec[k] = 0;
        if (k * 32 >= nb3) continue;  // warp-uniform
        const uint32_t j = k * 32 + lane;
        uint32_t x, y, z;
        ctx_voxel(pl, j < nb3 ? j : 0, x, y, z);
        const uint32_t dx = x == B, dy = y == B, dz = z == B;
        const uint32_t c = j < nb3 ? (dx | (dy << 1) | (dz << 2)) : 1u;
        const uint32_t rk = __shfl_sync(0xffffffffu, nb_rk, c);
        if (j < nb3 && rk != kNoVertex && g.ox + x < p.X && g.oy + y < p.Y && g.oz + z < p.Z) {
            const uint32_t lx = dx ? 0 : x, ly = dy ? 0 : y, lz = dz ? 0 : z;
            const uint32_t e = dx ? lz * B + ly : (dy ? BB + lz * B + lx : 2 * BB + ly * B + lx);
            rec[k] = ld_in<NC>(faces + (uint64_t)rk * face_stride + e) | 0x80000000u | (c << 27);
        }
    }
}

// Map entry of context voxel j: neighbour number c (bits 0-2), the index of its
// face record in that neighbour (bits 3-12), and the voxel's block coordinates
// x, y, z (5 bits each from bit 13).  It depends on B alone, so the emit kernel
// builds the map once per CTA.
__device__ __forceinline__ uint32_t ctx_map_entry(const WPlan &pl, uint32_t j) {
    const uint32_t B = pl.B, BB = pl.BB;
    uint32_t x, y, z;
    ctx_voxel(pl, j, x, y, z);
    const uint32_t dx = x == B, dy = y == B, dz = z == B;
    const uint32_t lx = dx ? 0 : x, ly = dy ? 0 : y, lz = dz ? 0 : z;
    const uint32_t e = dx ? lz * B + ly : (dy ? BB + lz * B + lx : 2 * BB + ly * B + lx);
    return (dx | (dy << 1) | (dz << 2)) | (e << 3) | (x << 13) | (y << 18) | (z << 23);
}

// gather_issue with the context-layer map in shared memory.
template <int CPL>
__device__ __forceinline__ void gather_issue_map(const Problem &p, const WPlan &pl, const Geo &g, uint32_t nb_rk,
                                                 const uint32_t *faces, uint32_t face_stride, const uint32_t *cmap,
                                                 uint32_t rec[CPL], uint64_t face_words = ~0ull) {
    const uint32_t lane = threadIdx.x & 31, nb3 = pl.nb3;
    // the whole context layer lies in the volume unless the block reaches a high face
    const bool inner = g.ox + pl.B < p.X && g.oy + pl.B < p.Y && g.oz + pl.B < p.Z;
#pragma unroll
    for (uint32_t k = 0; k < CPL; ++k) {
        rec[k] = 0;
        if (k * 32 >= nb3) continue;  // warp-uniform
        const uint32_t j = k * 32 + lane;
        const uint32_t m = cmap[j < nb3 ? j : 0];
        const uint32_t c = j < nb3 ? (m & 7u) : 1u;
        const uint32_t rk = __shfl_sync(0xffffffffu, nb_rk, c);
        bool take = j < nb3 && rk != kNoVertex;
        if (!inner)
            take = take && g.ox + ((m >> 13) & 31u) < p.X && g.oy + ((m >> 18) & 31u) < p.Y &&
                   g.oz + ((m >> 23) & 31u) < p.Z;
        if (take && MTX_BC((uint64_t)rk * face_stride + ((m >> 3) & 1023u), face_words, kBcFaces))
            rec[k] = __ldg(faces + (uint64_t)rk * face_stride + ((m >> 3) & 1023u)) | 0x80000000u | (c << 27);
    }
}

// Turns the gathered records into first-vertex ids and owned-edge masks of the
// context layer (nb_vb: lane c holds neighbour c's first vertex id).
// PACKED (B <= 8, the unified table of build_utab): each entry keeps the
// neighbour-relative first vertex and the voxel's owned-edge mask, rel | m <<
// 11 (the neighbour's number comes from the context map), and lanes 0-7 store
// the first vertex of the block (vbase, entry 0) and of its neighbours into
// the plan's eight base words.
template <int CPL, bool PACKED = false>
__device__ __forceinline__ void gather_finish(const WPlan &pl, uint32_t nb_vb, const uint32_t rec[CPL],
                                              unsigned char *ws, uint32_t vbase = 0) {
    const uint32_t lane = threadIdx.x & 31, nb3 = pl.nb3;
    uint32_t *nvid = reinterpret_cast<uint32_t *>(ws + pl.off_nvid);
    uint16_t *nvid16 = reinterpret_cast<uint16_t *>(ws + pl.off_nvid);
    uint8_t *nm = ws + pl.off_nm;
    if constexpr (PACKED) {
        if (lane < 8) reinterpret_cast<uint32_t *>(ws + pl.off_bar + 16)[lane] = lane ? nb_vb : vbase;
    }
#pragma unroll
    for (uint32_t k = 0; k < CPL; ++k) {
        if (k * 32 >= nb3) continue;
        const uint32_t j = k * 32 + lane;
        const uint32_t vb = PACKED ? 0u : __shfl_sync(0xffffffffu, nb_vb, (rec[k] >> 27) & 7u);
        if (j < nb3) {
            const bool present = rec[k] >> 31;
            if constexpr (PACKED) {
                nvid16[j] = (uint16_t)((rec[k] & 0x7ffu) | (present ? ((rec[k] >> 24) & 7u) << 11 : 0u));
            } else {
                nvid[j] = present ? vb + (rec[k] & 0xffffffu) : kNoVertex;
                nm[j] = present ? (uint8_t)((rec[k] >> 24) & 7u) : (uint8_t)0;
            }
        }
    }
}

// The block's low-face records from its crossing rows and row prefixes:
// block-relative first vertex | owned-edge mask << 24 of the voxels with
// x == 0 (index z*B + y), y == 0 (BB + z*B + x) and z == 0 (2BB + y*B + x).
// SPREAD: each y == 0 / z == 0 record computed by its own lane from its row's
// prefix (coalesced stores; the single-volume count pass); otherwise 2B lanes
// walk those rows along x with a running first vertex (the batched count phase).
template <bool SPREAD = true>
__device__ __forceinline__ void write_face_records(const WPlan &pl, const unsigned char *ws, uint32_t *fr) {
    const uint32_t lane = threadIdx.x & 31, B = pl.B, BB = pl.BB;
    const uint32_t *cross = reinterpret_cast<const uint32_t *>(ws + pl.off_cross);
    const uint32_t *vp = reinterpret_cast<const uint32_t *>(ws + pl.off_vp);
    if constexpr (SPREAD) {
        // records BB + i for i < 2BB: record i is voxel x of row q (y == 0:
        // q = z*B; z == 0: q = y); consecutive lanes take consecutive records
        for (uint32_t i = lane; i < 2 * BB; i += 32) {
            const uint32_t face = i >= BB, rem = face ? i - BB : i;
            const uint32_t r = fdiv(rem, pl.rB), x = rem - r * B;
            const uint32_t q = face ? r : r * B;
            const uint32_t xc = cross[q], yc = cross[BB + q], zc = cross[2 * BB + q];
            const uint32_t below = (1u << x) - 1u;
            const uint32_t run = vp[q] + __popc(xc & below) + __popc(yc & below) + __popc(zc & below);
            const uint32_t m = ((xc >> x) & 1u) | (((yc >> x) & 1u) << 1) | (((zc >> x) & 1u) << 2);
            if (MTX_BC(BB + i, 3 * BB, kBcFaces)) fr[BB + i] = run | (m << 24);
        }
    } else if (lane < 2 * B) {
        // lane l < 2B walks row (y = 0, z = l) or (y = l - B, z = 0) along x
        const bool yface = lane < B;
        const uint32_t q = yface ? lane * B : lane - B;
        uint32_t *o = fr + (yface ? BB + lane * B : 2 * BB + (lane - B) * B);
        const uint32_t xc = cross[q], yc = cross[BB + q], zc = cross[2 * BB + q];
        uint32_t run = vp[q];
        for (uint32_t x = 0; x < B; ++x) {
            const uint32_t m = ((xc >> x) & 1u) | (((yc >> x) & 1u) << 1) | (((zc >> x) & 1u) << 2);
            if (MTX_BC((uint32_t)(o - fr) + x, 3 * BB, kBcFaces)) o[x] = run | (m << 24);
            run += __popc(m);
        }
    }
    // x == 0 face: record z*B + y is voxel (0, y, z), the first of row q = z*B + y
    for (uint32_t q = lane; q < BB; q += 32)
        fr[q] = vp[q] | (((cross[q] & 1u) | ((cross[BB + q] & 1u) << 1) | ((cross[2 * BB + q] & 1u) << 2)) << 24);
}

// Count body of one block whose tile is staged: the (vertices, triangles)
// counts into *dr and the low-face records -- block-relative prefix | mask
// << 24 of the voxels with x == 0 (index z*B+y), y == 0 (BB + z*B+x) and
// z == 0 (2BB + y*B+x) -- into fr.  The tile is dead once the inside rows
// are built: next (TMA, one tile buffer) is then issued into the same buffer,
// so that its load runs under the rest of this block.
template <typename T, bool TMA = false>
__device__ __forceinline__ void count_block(const Problem &p, const WPlan &pl, unsigned char *ws, uint32_t buf,
                                            const Geo &g, const uint8_t *ntab, uint8_t *cases_out,
                                            mtx_meshlet_descriptor *dr, uint32_t *fr, uint8_t *state,
                                            const Geo *next = nullptr, const CUtensorMap *map = nullptr) {
    const uint32_t lane = threadIdx.x & 31;
    build_rows<T>(p, pl, ws, buf, g);
    if (next) tile_issue<T, TMA>(pl, ws, buf, *next, map);
    uint32_t bnv, bnt;
    block_counts(p, pl, ws, g, ntab, true, cases_out, bnv, bnt, state != nullptr);
    if (lane == 0) *reinterpret_cast<uint2 *>(&dr->vertexCount) = make_uint2(bnv, bnt);
    if (state) {  // the block state for the emit pass: 16-byte words, coalesced
        const uint4 *src = reinterpret_cast<const uint4 *>(ws + pl.off_cross);
        uint4 *dst = reinterpret_cast<uint4 *>(state);
        for (uint32_t i = lane; i < pl.state_bytes / 16; i += 32) dst[i] = src[i];
    }
    write_face_records(pl, ws, fr);
}

// Emit body of one block whose tile is staged and whose context layer has
// been gathered: its own vertices (when `vertices` is set) and its triangles.
// ANY as in emit_vertices.  VT: resolve triangle corners through the voxel
// table (build_utab; B <= 8 only).  STATE: the count pass's block state came
// with the tile (tile_issue), so the rows and counts are not rebuilt.
template <typename T, bool GENERIC, bool ANY = false, bool VT = false, bool STATE = false>
__device__ __forceinline__ void emit_block(const Problem &p, const WPlan &pl, unsigned char *ws, uint32_t buf,
                                           const Geo &g, const mtx_meshlet_descriptor &d, const uint64_t *tab,
                                           const uint8_t *ntab, const uint8_t *owner, uint32_t *indices,
                                           uint64_t tcap, void *vertices, uint64_t vcap, uint32_t vfmt,
                                           uint32_t frame, uint32_t normals, DevStatus *st, uint32_t r,
                                           const uint32_t *cmap = nullptr) {
    const uint32_t lane = threadIdx.x & 31, B = pl.B, BB = pl.BB;
    const uint32_t *cross = reinterpret_cast<const uint32_t *>(ws + pl.off_cross);
    const uint32_t *vp = reinterpret_cast<const uint32_t *>(ws + pl.off_vp);
    const uint32_t *tp = reinterpret_cast<const uint32_t *>(ws + pl.off_tp);
    const uint32_t *nvid = reinterpret_cast<const uint32_t *>(ws + pl.off_nvid);
    const uint8_t *nm = ws + pl.off_nm;
    uint32_t *jobs = reinterpret_cast<uint32_t *>(ws + pl.off_jobs);
    const uint32_t tbase = d.indexOffset / 3u;
    if ((uint64_t)tbase + d.primitiveCount > tcap || (vertices && (uint64_t)d.vertexOffset + d.vertexCount > vcap)) {
        if (lane == 0) report(st, MTX_ERR_CAPACITY, kSiteEmitCapacity, r, 2);
        return;
    }
    if (!(d.primitiveCount || (vertices && d.vertexCount))) return;
    uint32_t bnv = d.vertexCount;
    if constexpr (!STATE) {
        uint32_t bnt;
        build_rows<T>(p, pl, ws, buf, g);
        block_counts(p, pl, ws, g, ntab, true, nullptr, bnv, bnt, true);
        if (lane == 0 && (bnv != d.vertexCount || bnt != d.primitiveCount))
            report(st, MTX_ERR_INTERNAL, kSiteEmitNeighbour, r, 2);
    }
    if (vertices && bnv)
        emit_vertices<T, GENERIC, ANY>(p, pl, ws, buf, g, d.vertexOffset, bnv, vertices, vfmt, frame, normals);
    // triangles in canonical order: each lane walks the mixed cells of its rows
    // (masks and case bytes kept by block_counts) and writes one job per
    // triangle (cell | t << 12 | case << 16) at the triangle's own position in
    // a window of kJobWin jobs; the warp resolves 32 triangles at a time.  With
    // the vertex table (VT) the cell is given by its low corner's table index
    // (z (B+1) + y) (B+1) + x, which the resolve uses as is.
    const uint16_t *mmk = reinterpret_cast<const uint16_t *>(ws + pl.off_mm);
    const uint8_t *ck = ws + pl.off_case;
    uint16_t *vt = reinterpret_cast<uint16_t *>(ws + pl.off_tile[buf]);  // the tile is dead past the vertices
    uint8_t *um = ws + pl.off_tile[buf] + 2 * pl.B1 * pl.B1 * pl.B1;
    const uint32_t *nbase = reinterpret_cast<const uint32_t *>(ws + pl.off_bar + 16);
    if constexpr (VT) build_utab(pl, ws, vt, um, cmap);
    const uint32_t R = (BB + 31) / 32, nt = d.primitiveCount;
    bool bad = false;
    for (uint32_t w0 = 0; w0 < nt; w0 += kJobWin) {
        const uint32_t w1 = w0 + kJobWin;
        if (nt <= kJobWin) {  // one window (the common case): no window checks
            for (uint32_t k = 0; k < R; ++k) {
                const uint32_t q = lane * R + k;
                if (q >= BB) break;
                uint32_t j = tp[q], mm = mmk[q];
                const uint32_t cell0 = VT ? (q + fdiv(q, pl.rB)) * pl.B1 : q * B;  // row q = z B + y
                while (mm) {
                    const uint32_t x = __ffs(mm) - 1;
                    mm &= mm - 1u;
                    const uint32_t cfg = ck[q * B + x];
                    const uint32_t n = ntab[cfg], job = (cell0 + x) | (cfg << 16);
#pragma unroll
                    for (uint32_t t = 0; t < 5; ++t)  // at most five triangles a case
                        if (t < n) jobs[j + t] = job | (t << 12);
                    j += n;
                }
            }
        } else {
            for (uint32_t k = 0; k < R; ++k) {
                const uint32_t q = lane * R + k;
                if (q >= BB) break;
                uint32_t j = tp[q];
                const uint32_t jend = (q + 1 < BB) ? tp[q + 1] : nt;
                if (j >= w1 || jend <= w0) continue;
                uint32_t mm = mmk[q];
                const uint32_t cell0 = VT ? (q + fdiv(q, pl.rB)) * pl.B1 : q * B;
                while (mm) {
                    const uint32_t x = __ffs(mm) - 1;
                    mm &= mm - 1u;
                    const uint32_t cfg = ck[q * B + x];
                    const uint32_t n = ntab[cfg];
                    for (uint32_t t = 0; t < n; ++t, ++j)
                        if (j >= w0 && j < w1) jobs[j - w0] = (cell0 + x) | (t << 12) | (cfg << 16);
                }
            }
        }
        __syncwarp();
        const uint32_t cnt = min(kJobWin, nt - w0);
        for (uint32_t b = 0; b < cnt; b += 32) {
            const uint32_t n = min(32u, cnt - b);
            if (lane < n && MTX_BC(w0 + b + lane, nt, kBcIndex)) {
                const uint32_t job = jobs[b + lane];
                const uint32_t i = job & 0xfffu, t = (job >> 12) & 7u;
                const uint64_t w = tab[job >> 16] >> (4 + 12 * t);
                uint32_t *o = indices + 3ull * (tbase + w0 + b + lane);  // each lane its own 12 bytes
                if constexpr (VT) {
                    const uint32_t ti = i;  // the cell's low corner in the vertex table
                    const uint16_t *eoff = reinterpret_cast<const uint16_t *>(owner + 16);  // edge_offsets
                    o[0] = edge_vertex_ut(ti, (uint32_t)(w & 0xFu), eoff, vt, um, nbase, pl.B1, bad);
                    o[1] = edge_vertex_ut(ti, (uint32_t)((w >> 4) & 0xFu), eoff, vt, um, nbase, pl.B1, bad);
                    o[2] = edge_vertex_ut(ti, (uint32_t)((w >> 8) & 0xFu), eoff, vt, um, nbase, pl.B1, bad);
                } else {
                    const uint32_t q = fdiv(i, pl.rB), x = i - q * B;
                    const uint32_t z = fdiv(q, pl.rB), y = q - z * B;
                    o[0] = edge_vertex(x, y, z, (uint32_t)(w & 0xFu), owner, cross, vp, nvid, nm, B, BB,
                                       d.vertexOffset, bad);
                    o[1] = edge_vertex(x, y, z, (uint32_t)((w >> 4) & 0xFu), owner, cross, vp, nvid, nm, B, BB,
                                       d.vertexOffset, bad);
                    o[2] = edge_vertex(x, y, z, (uint32_t)((w >> 8) & 0xFu), owner, cross, vp, nvid, nm, B, BB,
                                       d.vertexOffset, bad);
                }
            }
            __syncwarp();
        }
    }
    if (bad) report(st, MTX_ERR_INTERNAL, kSiteEmitNeighbour, r, 3);
}

// Exclusive scan of the per-block vertex and triangle counts in rank order,
// one tile of up to kScanTile descriptors per CTA of kScanThreads: the tile
// resolves its offset with a decoupled look-back over the tiles before it,
// then fills vertexOffset and indexOffset; the last tile writes the totals.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ void scan_tile(mtx_meshlet_descriptor *desc, uint32_t count, uint32_t t, uint64_t *status,
                                          uint32_t *totals, DevStatus *st, uint64_t *s_tmp, uint32_t *s_ok,
                                          uint64_t *s_pre, uint32_t spin_limit = kSpinLimit) {
    const uint32_t ntiles = (count + kScanTile - 1) / kScanTile;
    const uint32_t base = t * kScanTile + threadIdx.x * kScanItems;
    uint32_t nv[kScanItems], nt[kScanItems], sv = 0, stt = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        nv[i] = nt[i] = 0;
        if (base + i < count) {
            const uint2 c = *reinterpret_cast<const uint2 *>(&desc[base + i].vertexCount);
            nv[i] = c.x;
            nt[i] = c.y;
        }
        sv += nv[i];
        stt += nt[i];
    }
    uint64_t tot;
    const uint64_t pre = cta_exclusive_scan64<kScanThreads>(((uint64_t)stt << 32) | sv, s_tmp, &tot);
    if (threadIdx.x < 32) {
        uint64_t ev, et;
        const bool ok = lookback_counts(status, t, (uint32_t)tot, (uint32_t)(tot >> 32), ev, et, st, spin_limit);
        if (threadIdx.x == 0) {
            *s_ok = ok;
            s_pre[0] = ev;
            s_pre[1] = et;
            if (ok && t == ntiles - 1) {
                totals[0] = (uint32_t)(ev + (uint32_t)tot);
                totals[1] = 3u * (uint32_t)(et + (uint32_t)(tot >> 32));
                totals[2] = count;
                totals[3] = count;
            }
        }
    }
    __syncthreads();
    if (!*s_ok) return;
    uint32_t v = (uint32_t)s_pre[0] + (uint32_t)pre, tr = (uint32_t)s_pre[1] + (uint32_t)(pre >> 32);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < count) {
            *reinterpret_cast<uint2 *>(&desc[base + i].vertexOffset) = make_uint2(v, 3u * tr);
            v += nv[i];
            tr += nt[i];
        }
    }
}

}  // namespace mtx
