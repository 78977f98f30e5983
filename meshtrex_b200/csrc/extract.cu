// Stage 3: PMB marching cubes over the active blocks
// (meshtrex: marching_cubes_pmb.task.glsl:101-216 and
// marching_cubes_pmb.mesh.glsl:185-393, drawn by extractionManager.cpp:638-640).
//
// Two persistent kernels over the compacted block list:
//
//  count  stages the block's (B+1)^3 voxels in shared memory (a TMA 3D tile
//         or plain loads), turns every voxel row into an inside bitmask, and
//         from those bitmasks gets, per row, the crossed +x/+y/+z edges each
//         voxel owns (PMB ownership) and the case index of each cell.  It
//         scans the per-block vertex/triangle counts across blocks with a
//         decoupled look-back (blocks taken in rank order by ticket), and
//         records for the block's three low faces the vertex prefix and edge
//         mask of every face voxel: that is all a neighbouring block needs to
//         name this block's vertices.
//  emit   restages the tile, rebuilds the masks, writes each owned vertex
//         once at its final index, and writes triangles whose vertex ids come
//         from a shared table of the (B+1)^3 context: own voxels from the row
//         prefixes, the +x/+y/+z layer from the neighbours' face records.
//
// Output order is canonical (and equals the CPU oracle's): vertices by
// (block rank, owner voxel x-fastest in the block, axis x<y<z); triangles by
// (block rank, cell x-fastest in the block, triangle number in the case).
#include <algorithm>

#include "mtx_internal.h"

namespace mtx {

__constant__ uint64_t c_mc_cases[256];
__constant__ uint8_t c_mc_owner[12];

// ------------------------------------------------------------- smem plan
struct Plan {
    uint32_t B, B1, PX;        // block edge, B+1, tile row pitch (elements)
    uint32_t off_tile, off_rows, off_cross, off_vp, off_tp, off_vid, off_vm, off_tab, off_misc;
    uint32_t bytes;
    uint32_t tile_bytes;       // TMA transaction size
};

__host__ __device__ inline uint32_t align_up(uint32_t v, uint32_t a) { return (v + a - 1) / a * a; }

__host__ __device__ inline Plan make_plan(uint32_t B, uint32_t esz, bool tma, bool emit) {
    Plan p{};
    p.B = B;
    p.B1 = B + 1;
    const uint32_t A = 16 / esz;  // elements per 16 bytes
    if (tma) {
        uint32_t g = 1;
        for (uint32_t d = 1; d <= A; ++d)
            if (B % d == 0 && A % d == 0) g = d;
        uint32_t xoff_max = (B % A == 0) ? 0 : A - g;
        p.PX = align_up(xoff_max + B + 1, A);
    } else {
        p.PX = B + 1;
    }
    uint32_t o = 0;
    p.off_tile = o;
    p.tile_bytes = p.PX * p.B1 * p.B1 * esz;
    o = align_up(o + p.tile_bytes, 128);
    p.off_rows = o;                       // (B+1)^2 inside masks
    o = align_up(o + 4 * p.B1 * p.B1, 16);
    p.off_cross = o;                      // 3 * B^2 crossing masks
    o = align_up(o + 12 * B * B, 16);
    p.off_vp = o;                         // B^2 vertex prefixes (per owned row)
    o = align_up(o + 4 * B * B, 16);
    p.off_tp = o;                         // B^2 triangle prefixes (per cell row)
    o = align_up(o + 4 * B * B, 16);
    if (emit) {
        p.off_vid = o;                    // (B+1)^3 first-vertex ids
        o = align_up(o + 4 * p.B1 * p.B1 * p.B1, 16);
        p.off_vm = o;                     // (B+1)^3 owned-edge masks
        o = align_up(o + p.B1 * p.B1 * p.B1, 16);
        p.off_tab = o;                    // packed case table
        o = align_up(o + 8 * 256, 16);
    } else {
        p.off_tab = o;                    // triangle counts only
        o = align_up(o + 256, 16);
    }
    p.off_misc = o;                       // scan scratch, neighbour info, mbarrier
    o += 512;
    p.bytes = align_up(o, 128);
    return p;
}

struct Geo {
    uint32_t ox, oy, oz;  // block origin (voxels)
    uint32_t bx, by, bz;
    uint32_t nx;          // voxels of the block inside the volume along x (<= B)
    uint32_t xoff;        // tile column of the block's first voxel
};

__device__ __forceinline__ Geo block_geo(uint32_t id, uint32_t B, uint32_t GX, uint32_t GY, uint32_t X, bool tma,
                                         uint32_t esz) {
    Geo g;
    g.bx = id % GX;
    g.by = (id / GX) % GY;
    g.bz = id / (GX * GY);
    g.ox = g.bx * B;
    g.oy = g.by * B;
    g.oz = g.bz * B;
    g.nx = min(B, X - g.ox);
    const uint32_t A = 16 / esz;
    g.xoff = tma ? (g.ox % A) : 0u;
    return g;
}

// Stage the (B+1)^3 voxels at the block origin into the tile.  TMA fills
// voxels outside the volume with zeros; plain loads do the same explicitly.
template <typename T>
__device__ __forceinline__ bool stage_tile(const Problem &p, const CUtensorMap *map, const Plan &pl, const Geo &g,
                                           unsigned char *smem, uint64_t *bar, uint32_t &phase, bool tma,
                                           DevStatus *st) {
    T *tile = reinterpret_cast<T *>(smem + pl.off_tile);
    if (tma) {
        if (threadIdx.x == 0) {
            mbar_arrive_expect_tx(bar, pl.tile_bytes);
            tma_load_3d(tile, map, bar, (int)(g.ox - g.xoff), (int)g.oy, (int)g.oz);
        }
        const bool ok = mbar_wait_bounded(bar, phase);
        phase ^= 1u;
        // every thread must take the same branch before the next barrier
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) report(st, MTX_ERR_TIMEOUT, kSiteTmaWait, g.ox, g.oy);
            return false;
        }
        return true;
    }
    const T *vol = reinterpret_cast<const T *>(p.vol);
    const uint32_t n = pl.B1 * pl.B1 * pl.B1;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        uint32_t x = i % pl.B1, y = (i / pl.B1) % pl.B1, z = i / (pl.B1 * pl.B1);
        uint32_t gx = g.ox + x, gy = g.oy + y, gz = g.oz + z;
        T v = T(0);
        if (gx < p.X && gy < p.Y && gz < p.Z) v = __ldg(vol + ((uint64_t)gz * p.Y + gy) * p.X + gx);
        tile[(z * pl.B1 + y) * pl.PX + x] = v;
    }
    __syncthreads();
    return true;
}

// Inside bitmask of every tile row (bit x <=> voxel at or below iso and in the volume).
template <typename T>
__device__ __forceinline__ void row_masks(const Problem &p, const Plan &pl, const Geo &g, unsigned char *smem) {
    const T *tile = reinterpret_cast<const T *>(smem + pl.off_tile);
    uint32_t *rows = reinterpret_cast<uint32_t *>(smem + pl.off_rows);
    const uint32_t nrows = pl.B1 * pl.B1;
    const uint32_t xin = min(pl.B1, p.X - g.ox);  // voxels of the row inside the volume
    for (uint32_t q = threadIdx.x; q < nrows; q += blockDim.x) {
        uint32_t y = q % pl.B1, z = q / pl.B1;
        uint32_t m = 0;
        if (g.oy + y < p.Y && g.oz + z < p.Z) {
            const T *r = tile + (z * pl.B1 + y) * pl.PX + g.xoff;
            for (uint32_t x = 0; x < xin; ++x) m |= (Vox<T>::val(r[x]) <= p.iso ? 1u : 0u) << x;
        }
        rows[q] = m;
    }
}

// Crossing masks of the owned voxel row (y, z): bit x of Xc/Yc/Zc set when
// the owned +x/+y/+z edge of voxel (x, y, z) is cut.
__device__ __forceinline__ void row_cross(const Problem &p, const Plan &pl, const Geo &g, const uint32_t *rows,
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

__device__ __forceinline__ uint32_t cell_case(uint32_t r00, uint32_t r01, uint32_t r10, uint32_t r11, uint32_t x) {
    // corners (marching_cubes_pmb.mesh.glsl:84-93): r00 = row (y,z), r01 = (y+1,z),
    // r10 = (y,z+1), r11 = (y+1,z+1)
    return ((r00 >> x) & 1u) | (((r00 >> (x + 1)) & 1u) << 1) | (((r01 >> (x + 1)) & 1u) << 2) |
           (((r01 >> x) & 1u) << 3) | (((r10 >> x) & 1u) << 4) | (((r10 >> (x + 1)) & 1u) << 5) |
           (((r11 >> (x + 1)) & 1u) << 6) | (((r11 >> x) & 1u) << 7);
}

// Number of cells of row (y, z) that lie inside the volume (0 if the row does not).
__device__ __forceinline__ uint32_t cells_in_row(const Problem &p, const Plan &pl, const Geo &g, uint32_t y,
                                                 uint32_t z) {
    if (g.oy + y + 1 >= p.Y || g.oz + z + 1 >= p.Z || g.ox + 1 >= p.X) return 0;
    return min(pl.B, p.X - 1 - g.ox);
}

// ------------------------------------------------------------- count pass
constexpr uint64_t kCnt31 = 0x7fffffffull;

template <typename T, int NT>
__global__ void __launch_bounds__(NT) count_kernel(Problem p, const __grid_constant__ CUtensorMap map, bool tma,
                                                   const uint32_t *__restrict__ ids,
                                                   const uint32_t *__restrict__ count_ptr,
                                                   mtx_meshlet_descriptor *__restrict__ desc,
                                                   uint64_t desc_capacity, uint32_t *__restrict__ faces,
                                                   uint64_t *status, uint32_t *ticket, uint32_t *totals,
                                                   uint8_t *__restrict__ cell_cases, uint64_t block_cap,
                                                   DevStatus *st) {
    extern __shared__ __align__(128) unsigned char smem[];
    const Plan pl = make_plan(p.B, sizeof(T), tma, false);
    uint32_t *rows = reinterpret_cast<uint32_t *>(smem + pl.off_rows);
    uint32_t *cross = reinterpret_cast<uint32_t *>(smem + pl.off_cross);
    uint32_t *vp = reinterpret_cast<uint32_t *>(smem + pl.off_vp);
    uint32_t *tp = reinterpret_cast<uint32_t *>(smem + pl.off_tp);
    uint8_t *ntab = smem + pl.off_tab;
    uint32_t *misc = reinterpret_cast<uint32_t *>(smem + pl.off_misc);
    uint64_t *misc64 = reinterpret_cast<uint64_t *>(smem + pl.off_misc);
    // misc layout: [0..15] u64 scan scratch, [32] u32 rank, [33] abort, [34..35] u64 prefix, bar at +448
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + pl.off_misc + 448);

    for (uint32_t i = threadIdx.x; i < 256; i += NT) ntab[i] = (uint8_t)(c_mc_cases[i] & 0xFu);
    if (threadIdx.x == 0 && tma) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    if (tma && threadIdx.x == 0) prefetch_tensormap(&map);
    __syncthreads();
    const uint32_t count = *count_ptr;
    const uint32_t B = p.B, BB = B * B;
    uint32_t phase = 0;
    if (count > block_cap || count > desc_capacity) {
        // scratch sized for fewer active blocks: report the needed count, do nothing
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            report(st, MTX_ERR_CAPACITY, kSiteEmitCapacity, count, 3);
            totals[3] = count;
        }
        return;
    }

    while (true) {
        if (threadIdx.x == 0) misc[32] = atomicAdd(ticket, 1u);
        __syncthreads();
        const uint32_t r = misc[32];
        __syncthreads();
        if (r >= count) break;
        const uint32_t id = ids[r];
        const Geo g = block_geo(id, B, p.GX, p.GY, p.X, tma, sizeof(T));
        bool ok = stage_tile<T>(p, &map, pl, g, smem, bar, phase, tma, st);
        if (ok) row_masks<T>(p, pl, g, smem);
        __syncthreads();

        // per-row vertex and triangle counts; thread t owns a contiguous run of rows
        constexpr int RPT_MAX = 4;  // rows per thread for B <= 16 with NT >= 64
        const uint32_t rpt = (BB + NT - 1) / NT;
        uint32_t nv_t = 0, nt_t = 0;
        uint32_t rv[RPT_MAX], rt[RPT_MAX];
#pragma unroll
        for (int k = 0; k < RPT_MAX; ++k) {
            rv[k] = rt[k] = 0;
            const uint32_t q = threadIdx.x * rpt + k;
            if (!ok || (uint32_t)k >= rpt || q >= BB) continue;
            const uint32_t y = q % B, z = q / B;
            uint32_t xc, yc, zc;
            row_cross(p, pl, g, rows, y, z, xc, yc, zc);
            cross[q] = xc;
            cross[BB + q] = yc;
            cross[2 * BB + q] = zc;
            rv[k] = __popc(xc) + __popc(yc) + __popc(zc);
            const uint32_t ncell = cells_in_row(p, pl, g, y, z);
            uint32_t ntr = 0;
            if (ncell) {
                const uint32_t r00 = rows[z * pl.B1 + y], r01 = rows[z * pl.B1 + y + 1];
                const uint32_t r10 = rows[(z + 1) * pl.B1 + y], r11 = rows[(z + 1) * pl.B1 + y + 1];
                const uint32_t span = (2u << ncell) - 1u;  // bits 0..ncell
                const uint32_t a = r00 & r01 & r10 & r11 & span, o = (r00 | r01 | r10 | r11) & span;
                const bool uniform = (a == span) || (o == 0);
                for (uint32_t x = 0; x < ncell; ++x) {
                    const uint32_t cfg = uniform ? (a ? 255u : 0u) : cell_case(r00, r01, r10, r11, x);
                    ntr += ntab[cfg];
                    if (cell_cases) cell_cases[(uint64_t)r * B * BB + q * B + x] = (uint8_t)cfg;
                }
            }
            if (cell_cases)
                for (uint32_t x = ncell; x < B; ++x) cell_cases[(uint64_t)r * B * BB + q * B + x] = 0;
            rt[k] = ntr;
            nv_t += rv[k];
            nt_t += ntr;
        }
        uint64_t tot64;
        const uint64_t pre =
            cta_exclusive_scan64<NT>(((uint64_t)nt_t << 32) | nv_t, reinterpret_cast<uint64_t *>(misc64), &tot64);
        uint32_t pv = (uint32_t)pre, pt = (uint32_t)(pre >> 32);
#pragma unroll
        for (int k = 0; k < RPT_MAX; ++k) {
            const uint32_t q = threadIdx.x * rpt + k;
            if ((uint32_t)k < rpt && q < BB) {
                vp[q] = pv;
                tp[q] = pt;
                pv += rv[k];
                pt += rt[k];
            }
        }
        const uint32_t bnv = (uint32_t)tot64, bnt = (uint32_t)(tot64 >> 32);

        // ---- decoupled look-back over ranks: status = [63:62] flag, [61:31] tris, [30:0] verts
        if (threadIdx.x < 32) {
            const uint32_t lane = threadIdx.x;
            uint64_t sv = 0, stt = 0;
            bool abort = !ok;
            const uint64_t agg = ((uint64_t)bnt << 31) | bnv;
            if (r == 0) {
                // nothing before
            } else {
                if (lane == 0 && !abort) st_volatile(&status[r], (1ull << 62) | agg);
                int64_t j = (int64_t)r - 1;
                uint32_t spins = 0;
                while (!abort) {
                    const int64_t k = j - (int64_t)lane;
                    const uint64_t w = k >= 0 ? ld_volatile(&status[k]) : (2ull << 62);
                    const uint32_t flag = (uint32_t)(w >> 62);
                    if (__any_sync(0xffffffffu, flag == 3u)) { abort = true; break; }
                    const uint32_t inc = __ballot_sync(0xffffffffu, flag == 2u);
                    const uint32_t emp = __ballot_sync(0xffffffffu, flag == 0u);
                    const uint32_t first = inc ? (uint32_t)(__ffs(inc) - 1) : 32u;
                    const uint32_t window = first >= 31 ? 0xffffffffu : ((2u << first) - 1u);
                    if (emp & window) {
                        if (++spins >= kSpinLimit) {
                            if (lane == 0) report(st, MTX_ERR_TIMEOUT, kSiteCountLookback, r, (uint32_t)j);
                            abort = true;
                            break;
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
                    sv += a;
                    stt += b;
                    if (first < 32) break;
                    j -= 32;
                }
            }
            const uint64_t iv = sv + bnv, it = stt + bnt;
            if (!abort && (iv > kCnt31 || it > kCnt31 || 3ull * it > 0xffffffffull)) {
                if (lane == 0) report(st, MTX_ERR_CAPACITY, kSiteCountOverflow, (uint32_t)(iv >> 32), (uint32_t)it);
                abort = true;
            }
            if (lane == 0) {
                st_volatile(&status[r], abort ? (3ull << 62) : ((2ull << 62) | (it << 31) | iv));
                misc[33] = abort ? 1u : 0u;
                misc64[17] = (stt << 32) | sv;
            }
        }
        __syncthreads();
        if (!misc[33]) {
            const uint64_t pre2 = misc64[17];
            const uint32_t vbase = (uint32_t)pre2, tbase = (uint32_t)(pre2 >> 32);
            if (threadIdx.x == 0) {
                if (r < desc_capacity) {
                    mtx_meshlet_descriptor d;
                    d.vertexOffset = vbase;
                    d.indexOffset = 3u * tbase;
                    d.vertexCount = bnv;
                    d.primitiveCount = bnt;
                    desc[r] = d;
                } else {
                    report(st, MTX_ERR_CAPACITY, kSiteEmitCapacity, r, 0);
                }
                if (r == count - 1) {
                    totals[0] = vbase + bnv;
                    totals[1] = 3u * (tbase + bnt);
                    totals[2] = count;
                    totals[3] = count;
                }
            }
            // low-face records: prefix | mask << 24 of voxels with x == 0, y == 0, z == 0
            uint32_t *fr = faces + (uint64_t)r * 3 * BB;
            for (uint32_t e = threadIdx.x; e < 3 * BB; e += NT) {
                const uint32_t f = e / BB, i = e % BB;
                const uint32_t a = i % B, b = i / B;
                uint32_t x, y, z;
                if (f == 0) { x = 0; y = a; z = b; }
                else if (f == 1) { x = a; y = 0; z = b; }
                else { x = a; y = b; z = 0; }
                const uint32_t q = z * B + y;
                const uint32_t below = (1u << x) - 1u;
                const uint32_t xc = cross[q], yc = cross[BB + q], zc = cross[2 * BB + q];
                const uint32_t pre = vp[q] + __popc(xc & below) + __popc(yc & below) + __popc(zc & below);
                const uint32_t m = ((xc >> x) & 1u) | (((yc >> x) & 1u) << 1) | (((zc >> x) & 1u) << 2);
                fr[e] = pre | (m << 24);
            }
        }
        const bool stop = misc[33] != 0;
        __syncthreads();
        if (stop) break;  // successors see the aborted status and stop too
    }
}

// -------------------------------------------------------------- emit pass
constexpr uint32_t kNoVertex = 0xffffffffu;

template <typename T>
__device__ __forceinline__ float tile_val(const Plan &pl, const Geo &g, const unsigned char *smem, uint32_t x,
                                          uint32_t y, uint32_t z) {
    const T *tile = reinterpret_cast<const T *>(smem + pl.off_tile);
    return Vox<T>::val(tile[(z * pl.B1 + y) * pl.PX + g.xoff + x]);
}

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

template <typename T, int NT>
__global__ void __launch_bounds__(NT) emit_kernel(Problem p, const __grid_constant__ CUtensorMap map, bool tma,
                                                  const uint32_t *__restrict__ ids,
                                                  const uint32_t *__restrict__ rank_map,
                                                  const uint32_t *__restrict__ count_ptr,
                                                  const mtx_meshlet_descriptor *__restrict__ desc,
                                                  const uint32_t *__restrict__ faces, void *__restrict__ vertices,
                                                  uint64_t vcap, uint32_t *__restrict__ indices, uint64_t tcap,
                                                  uint32_t vfmt, uint32_t frame, uint32_t normals,
                                                  uint64_t block_cap, DevStatus *st) {
    extern __shared__ __align__(128) unsigned char smem[];
    const Plan pl = make_plan(p.B, sizeof(T), tma, true);
    uint32_t *rows = reinterpret_cast<uint32_t *>(smem + pl.off_rows);
    uint32_t *cross = reinterpret_cast<uint32_t *>(smem + pl.off_cross);
    uint32_t *vp = reinterpret_cast<uint32_t *>(smem + pl.off_vp);
    uint32_t *tp = reinterpret_cast<uint32_t *>(smem + pl.off_tp);
    uint32_t *vid = reinterpret_cast<uint32_t *>(smem + pl.off_vid);
    uint8_t *vm = smem + pl.off_vm;
    uint64_t *tab = reinterpret_cast<uint64_t *>(smem + pl.off_tab);
    uint32_t *misc = reinterpret_cast<uint32_t *>(smem + pl.off_misc);
    uint64_t *misc64 = reinterpret_cast<uint64_t *>(smem + pl.off_misc);
    // misc: [0..15] u64 scan scratch; [40..47] neighbour vbase; [48..55] neighbour rank
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + pl.off_misc + 448);

    for (uint32_t i = threadIdx.x; i < 256; i += NT) tab[i] = c_mc_cases[i];
    if (threadIdx.x == 0 && tma) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    const uint32_t count = *count_ptr;
    if (count > block_cap) return;  // reported by the count pass
    const uint32_t B = p.B, BB = B * B, B1 = pl.B1;
    uint32_t phase = 0;
    const uint64_t nvert_cap = vcap, ntri_cap = tcap;

    for (uint32_t r = blockIdx.x; r < count; r += gridDim.x) {
        const mtx_meshlet_descriptor d = desc[r];
        if (d.vertexCount == 0 && d.primitiveCount == 0) continue;
        const uint32_t tbase = d.indexOffset / 3u;
        if ((uint64_t)d.vertexOffset + d.vertexCount > nvert_cap || (uint64_t)tbase + d.primitiveCount > ntri_cap) {
            if (threadIdx.x == 0) report(st, MTX_ERR_CAPACITY, kSiteEmitCapacity, r, 1);
            continue;
        }
        const uint32_t id = ids[r];
        const Geo g = block_geo(id, B, p.GX, p.GY, p.X, tma, sizeof(T));
        if (threadIdx.x < 7) {
            // neighbour (dx,dy,dz) = bits of threadIdx.x + 1
            const uint32_t c = threadIdx.x + 1, dx = c & 1u, dy = (c >> 1) & 1u, dz = c >> 2;
            uint32_t vb = kNoVertex, rk = kNoVertex;
            if (g.bx + dx < p.GX && g.by + dy < p.GY && g.bz + dz < p.GZ) {
                const uint32_t nid = id + dx + dy * p.GX + dz * p.GX * p.GY;
                const uint32_t cand = rank_map[nid];
                if (cand < count && ids[cand] == nid) {
                    rk = cand;
                    vb = desc[cand].vertexOffset;
                }
            }
            misc[40 + c] = vb;
            misc[48 + c] = rk;
        }
        if (!stage_tile<T>(p, &map, pl, g, smem, bar, phase, tma, st)) return;
        row_masks<T>(p, pl, g, smem);
        __syncthreads();

        constexpr int RPT_MAX = 4;
        const uint32_t rpt = (BB + NT - 1) / NT;
        uint32_t nv_t = 0, nt_t = 0;
        uint32_t rv[RPT_MAX], rt[RPT_MAX];
#pragma unroll
        for (int k = 0; k < RPT_MAX; ++k) {
            rv[k] = rt[k] = 0;
            const uint32_t q = threadIdx.x * rpt + k;
            if ((uint32_t)k >= rpt || q >= BB) continue;
            const uint32_t y = q % B, z = q / B;
            uint32_t xc, yc, zc;
            row_cross(p, pl, g, rows, y, z, xc, yc, zc);
            cross[q] = xc;
            cross[BB + q] = yc;
            cross[2 * BB + q] = zc;
            rv[k] = __popc(xc) + __popc(yc) + __popc(zc);
            const uint32_t ncell = cells_in_row(p, pl, g, y, z);
            uint32_t ntr = 0;
            if (ncell) {
                const uint32_t r00 = rows[z * B1 + y], r01 = rows[z * B1 + y + 1];
                const uint32_t r10 = rows[(z + 1) * B1 + y], r11 = rows[(z + 1) * B1 + y + 1];
                const uint32_t span = (2u << ncell) - 1u;
                const uint32_t a = r00 & r01 & r10 & r11 & span, o = (r00 | r01 | r10 | r11) & span;
                if (a != span && o != 0)
                    for (uint32_t x = 0; x < ncell; ++x) ntr += (uint32_t)(tab[cell_case(r00, r01, r10, r11, x)] & 0xFu);
            }
            rt[k] = ntr;
            nv_t += rv[k];
            nt_t += ntr;
        }
        uint64_t tot64;
        const uint64_t pre = cta_exclusive_scan64<NT>(((uint64_t)nt_t << 32) | nv_t, misc64, &tot64);
        uint32_t pv = (uint32_t)pre, pt = (uint32_t)(pre >> 32);
#pragma unroll
        for (int k = 0; k < RPT_MAX; ++k) {
            const uint32_t q = threadIdx.x * rpt + k;
            if ((uint32_t)k < rpt && q < BB) {
                vp[q] = pv;
                tp[q] = pt;
                pv += rv[k];
                pt += rt[k];
            }
        }
        if (threadIdx.x == 0 && ((uint32_t)tot64 != d.vertexCount || (uint32_t)(tot64 >> 32) != d.primitiveCount))
            report(st, MTX_ERR_INTERNAL, kSiteEmitNeighbour, r, 2);
        __syncthreads();

        // first-vertex id and owned-edge mask of every voxel of the (B+1)^3 context
        const uint32_t nctx = B1 * B1 * B1;
        for (uint32_t i = threadIdx.x; i < nctx; i += NT) {
            const uint32_t x = i % B1, y = (i / B1) % B1, z = i / (B1 * B1);
            uint32_t first = kNoVertex, mask = 0;
            if (x < B && y < B && z < B) {
                const uint32_t q = z * B + y, below = (1u << x) - 1u;
                const uint32_t xc = cross[q], yc = cross[BB + q], zc = cross[2 * BB + q];
                first = d.vertexOffset + vp[q] + __popc(xc & below) + __popc(yc & below) + __popc(zc & below);
                mask = ((xc >> x) & 1u) | (((yc >> x) & 1u) << 1) | (((zc >> x) & 1u) << 2);
            } else if (g.ox + x < p.X && g.oy + y < p.Y && g.oz + z < p.Z) {
                const uint32_t dx = x == B, dy = y == B, dz = z == B;
                const uint32_t c = dx | (dy << 1) | (dz << 2);
                const uint32_t rk = misc[48 + c];
                if (rk != kNoVertex) {
                    const uint32_t lx = dx ? 0 : x, ly = dy ? 0 : y, lz = dz ? 0 : z;
                    uint32_t e;
                    if (dx) e = lz * B + ly;
                    else if (dy) e = BB + lz * B + lx;
                    else e = 2 * BB + ly * B + lx;
                    const uint32_t rec = __ldg(faces + (uint64_t)rk * 3 * BB + e);
                    first = misc[40 + c] + (rec & 0xffffffu);
                    mask = rec >> 24;
                }
            }
            vid[i] = first;
            vm[i] = (uint8_t)mask;
        }
        __syncthreads();

        // vertices: one thread per owned voxel row
        for (uint32_t q = threadIdx.x; q < BB; q += NT) {
            const uint32_t y = q % B, z = q / B;
            const uint32_t xc = cross[q], yc = cross[BB + q], zc = cross[2 * BB + q];
            uint32_t any = xc | yc | zc;
            uint32_t idx = d.vertexOffset + vp[q];
            while (any) {
                const uint32_t x = __ffs(any) - 1;
                any &= any - 1;
                const uint32_t m = ((xc >> x) & 1u) | (((yc >> x) & 1u) << 1) | (((zc >> x) & 1u) << 2);
                const float fa = tile_val<T>(pl, g, smem, x, y, z);
#pragma unroll
                for (uint32_t a = 0; a < 3; ++a) {
                    if (!((m >> a) & 1u)) continue;
                    const float fb = tile_val<T>(pl, g, smem, x + (a == 0), y + (a == 1), z + (a == 2));
                    const float t = edge_t(fa, fb, p.iso);
                    float pos[3] = {(float)(g.ox + x), (float)(g.oy + y), (float)(g.oz + z)};
                    pos[a] = __fadd_rn(pos[a], t);
                    if (frame == MTX_FRAME_NDC) {
                        const float dims[3] = {(float)p.X, (float)p.Y, (float)p.Z};
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                            pos[k] = __fsub_rn(__fmul_rn(__fdiv_rn(pos[k], dims[k]), 2.0f), 1.0f);
                    }
                    if (vfmt == MTX_VERTEX_XYZ) {
                        float *v = reinterpret_cast<float *>(vertices) + 3ull * idx;
                        v[0] = pos[0];
                        v[1] = pos[1];
                        v[2] = pos[2];
                    } else {
                        float nrm[3] = {0.f, 0.f, 0.f};
                        if (normals) {
                            float n1[3], n2[3];
                            const uint32_t gx = g.ox + x, gy = g.oy + y, gz = g.oz + z;
                            voxel_normal<T>(p, gx, gy, gz, n1);
                            voxel_normal<T>(p, gx + (a == 0), gy + (a == 1), gz + (a == 2), n2);
                            const float omt = __fsub_rn(1.0f, t);
#pragma unroll
                            for (int k = 0; k < 3; ++k) nrm[k] = __fadd_rn(__fmul_rn(n1[k], omt), __fmul_rn(n2[k], t));
                            normalize3(nrm[0], nrm[1], nrm[2]);
                        }
                        float4 *v = reinterpret_cast<float4 *>(vertices) + 2ull * idx;
                        v[0] = make_float4(pos[0], pos[1], pos[2], 1.0f);
                        v[1] = make_float4(nrm[0], nrm[1], nrm[2], 0.0f);
                    }
                    ++idx;
                }
            }
        }

        // triangles: one thread per cell row
        for (uint32_t q = threadIdx.x; q < BB; q += NT) {
            const uint32_t y = q % B, z = q / B;
            const uint32_t ncell = cells_in_row(p, pl, g, y, z);
            if (!ncell) continue;
            const uint32_t r00 = rows[z * B1 + y], r01 = rows[z * B1 + y + 1];
            const uint32_t r10 = rows[(z + 1) * B1 + y], r11 = rows[(z + 1) * B1 + y + 1];
            const uint32_t span = (2u << ncell) - 1u;
            const uint32_t a = r00 & r01 & r10 & r11 & span, o = (r00 | r01 | r10 | r11) & span;
            if (a == span || o == 0) continue;
            uint64_t tri = (uint64_t)tbase + tp[q];
            for (uint32_t x = 0; x < ncell; ++x) {
                const uint32_t cfg = cell_case(r00, r01, r10, r11, x);
                const uint64_t w = tab[cfg];
                const uint32_t n = (uint32_t)(w & 0xFu);
                for (uint32_t t = 0; t < n; ++t, ++tri) {
                    uint32_t out[3];
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const uint32_t e = (uint32_t)((w >> (4 + 4 * (3 * t + k))) & 0xFu);
                        const uint32_t own = c_mc_owner[e];
                        const uint32_t ux = x + (own & 1u), uy = y + ((own >> 1) & 1u), uz = z + ((own >> 2) & 1u);
                        const uint32_t ax = own >> 3;
                        const uint32_t li = (uz * B1 + uy) * B1 + ux;
                        const uint32_t msk = vm[li];
                        uint32_t v = vid[li];
                        if (v == kNoVertex || !((msk >> ax) & 1u)) {
                            report(st, MTX_ERR_INTERNAL, kSiteEmitNeighbour, r, li);
                            v = 0;
                        } else {
                            v += __popc(msk & ((1u << ax) - 1u));
                        }
                        out[k] = v;
                    }
                    uint32_t *dst = indices + 3ull * tri;
                    dst[0] = out[0];
                    dst[1] = out[1];
                    dst[2] = out[2];
                }
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ host
static bool g_tables_loaded[64] = {false};

static mtx_status ensure_tables(mtx_context *c) {
    if (c->device < 64 && g_tables_loaded[c->device]) return MTX_OK;
    MTX_CUDA(c, cudaMemcpyToSymbol(c_mc_cases, MTX_MC_CASES, sizeof(MTX_MC_CASES)));
    MTX_CUDA(c, cudaMemcpyToSymbol(c_mc_owner, MTX_MC_EDGE_OWNER, sizeof(MTX_MC_EDGE_OWNER)));
    if (c->device < 64) g_tables_loaded[c->device] = true;
    return MTX_OK;
}

bool tma_ok(const Problem &p) {
    const uint32_t esz = dtype_size(p.dtype);
    return ((uintptr_t)p.vol % 16 == 0) && (((uint64_t)p.X * esz) % 16 == 0);
}

static bool use_tma(const Problem &p, uint32_t staging) {
    if (staging == MTX_STAGING_LDG) return false;
    return tma_ok(p);
}

template <typename T, int NT>
static mtx_status run_count(mtx_context *c, const Problem &p, const ExtractArgs &a, const CUtensorMap &map, bool tma,
                            cudaStream_t s) {
    const Plan pl = make_plan(p.B, sizeof(T), tma, false);
    auto k = count_kernel<T, NT>;
    MTX_CUDA(c, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.bytes));
    int per_sm = 0;
    MTX_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, pl.bytes));
    uint64_t grid = (uint64_t)std::max(per_sm, 1) * c->sm_count;
    if (a.host_count) grid = std::min<uint64_t>(grid, a.host_count);
    grid = std::max<uint64_t>(grid, 1);
    k<<<(unsigned)grid, NT, pl.bytes, s>>>(p, map, tma, a.ids, a.count, a.desc, a.desc_capacity, a.faces,
                                          a.count_status, &c->ctrl->count_ticket, a.totals, a.cell_cases,
                                          a.block_capacity, &c->ctrl->status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "count launch");
    return MTX_OK;
}

template <typename T, int NT>
static mtx_status run_emit(mtx_context *c, const Problem &p, const ExtractArgs &a, const CUtensorMap &map, bool tma,
                           cudaStream_t s) {
    const Plan pl = make_plan(p.B, sizeof(T), tma, true);
    auto k = emit_kernel<T, NT>;
    MTX_CUDA(c, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.bytes));
    int per_sm = 0;
    MTX_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, pl.bytes));
    uint64_t grid = (uint64_t)std::max(per_sm, 1) * c->sm_count;
    if (a.host_count) grid = std::min<uint64_t>(grid, a.host_count);
    grid = std::max<uint64_t>(grid, 1);
    k<<<(unsigned)grid, NT, pl.bytes, s>>>(p, map, tma, a.ids, a.rank_map, a.count, a.desc, a.faces, a.vertices,
                                          a.vertex_capacity, a.indices, a.tri_capacity, a.vertex_format, a.frame,
                                          a.normals, a.block_capacity, &c->ctrl->status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "emit launch");
    return MTX_OK;
}

static int pick_threads(uint32_t B, uint32_t req) {
    if (req == 64 || req == 128 || req == 256) {
        // rows per thread must stay <= 4
        if ((B * B + req - 1) / req <= 4) return (int)req;
    }
    return B * B <= 64 ? 64 : (B * B <= 128 ? 128 : 256);
}

template <int NT, bool EMIT>
static mtx_status dispatch_nt(mtx_context *c, const Problem &p, const ExtractArgs &a, const CUtensorMap &map, bool tma,
                              cudaStream_t s) {
    switch (p.dtype) {
    case MTX_DTYPE_U8: return EMIT ? run_emit<uint8_t, NT>(c, p, a, map, tma, s) : run_count<uint8_t, NT>(c, p, a, map, tma, s);
    case MTX_DTYPE_U16: return EMIT ? run_emit<uint16_t, NT>(c, p, a, map, tma, s) : run_count<uint16_t, NT>(c, p, a, map, tma, s);
    default: return EMIT ? run_emit<float, NT>(c, p, a, map, tma, s) : run_count<float, NT>(c, p, a, map, tma, s);
    }
}

template <bool EMIT>
static mtx_status launch_stage(mtx_context *c, const Problem &p, const ExtractArgs &a, cudaStream_t s) {
    if (p.B < 2 || p.B > MTX_MAX_BLOCK_EDGE) return fail(c, MTX_ERR_UNSUPPORTED, "block edge must be in [2, 16]");
    mtx_status rs = ensure_tables(c);
    if (rs != MTX_OK) return rs;
    const bool tma = use_tma(p, a.staging);
    CUtensorMap map;
    memset(&map, 0, sizeof(map));
    if (tma) {
        const Plan pl = make_plan(p.B, dtype_size(p.dtype), true, EMIT);
        rs = make_volume_tensor_map(c, p, pl.PX, &map);
        if (rs != MTX_OK) return rs;
    }
    switch (pick_threads(p.B, a.threads)) {
    case 64: return dispatch_nt<64, EMIT>(c, p, a, map, tma, s);
    case 128: return dispatch_nt<128, EMIT>(c, p, a, map, tma, s);
    default: return dispatch_nt<256, EMIT>(c, p, a, map, tma, s);
    }
}

mtx_status launch_count(mtx_context *c, const Problem &p, const ExtractArgs &a, cudaStream_t s) {
    MTX_CUDA(c, cudaMemsetAsync(&c->ctrl->count_ticket, 0, sizeof(uint32_t), s));
    MTX_CUDA(c, cudaMemsetAsync(a.totals, 0, 4 * sizeof(uint32_t), s));
    if (a.host_count) MTX_CUDA(c, cudaMemsetAsync(a.count_status, 0, sizeof(uint64_t) * a.host_count, s));
    return launch_stage<false>(c, p, a, s);
}

mtx_status launch_emit(mtx_context *c, const Problem &p, const ExtractArgs &a, cudaStream_t s) {
    return launch_stage<true>(c, p, a, s);
}

}  // namespace mtx
