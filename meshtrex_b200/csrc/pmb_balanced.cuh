// Balanced block bodies for dense blocks, used by the batched kernel.
//
// The single-volume bodies (pmb_device.cuh) let each lane walk its own rows
// of the block, which costs little when a block has few mixed cells but
// leaves lanes idle behind the busiest one when it has many.  Here a block's
// mixed cells (and cut voxels) are first listed in canonical order, then the
// warp takes them 32 at a time, one per lane: a warp scan of their triangle
// (vertex) counts queues the jobs in a ring, which the warp resolves 32 at a
// time.  Triangle corners resolve through a per-block vertex table: the first
// vertex id and owned-edge mask of every voxel of the (B+1)^3 tile.
//
// Layout (make_wplan_balanced): a single float tile, which the vertex table
// takes over once the block's vertices are written; the context layer of the
// table is gathered from the neighbours' face records at that point.  The
// row prefixes live in the job ring (dead until the first job is queued),
// and outputs go straight from the lanes to global memory, so that four CTAs
// of eight warps fit an SM at B = 8.  Same output as the row bodies, bit for
// bit.
#pragma once

#include "pmb_device.cuh"

namespace mtx {

constexpr uint32_t kRing = 256;  // queued jobs (a power of two): at most 31 left + 32 cells x 5 triangles

__host__ __device__ inline WPlan make_wplan_balanced(uint32_t B) {
    WPlan p{};
    p.B = B;
    p.B1 = B + 1;
    p.BB = B * B;
    p.nb3 = 3 * B * B + 3 * B + 1;
    p.rB = (uint32_t)((0x100000000ull + B - 1) / B);
    p.rB1 = (uint32_t)((0x100000000ull + B) / (B + 1));
    p.rBB = (uint32_t)((0x100000000ull + B * B - 1) / (B * B));
    p.R = 32 / B;
    p.PX = B + 1;
    const uint32_t T3 = p.B1 * p.B1 * p.B1;
    p.tile_bytes = 4 * T3;
    p.nbuf = 1;
    uint32_t o = 0;
    p.off_tile[0] = p.off_tile[1] = o;
    p.off_vtab = o;  // the vertex table replaces the tile (same size)
    o = align_up(o + p.tile_bytes, 16);
    p.off_bar = 0;   // unused: tiles are staged by plain loads
    p.off_rows = o;
    o = align_up(o + 4 * p.B1 * p.B1, 16);
    p.off_cross = o;
    o = align_up(o + 12 * p.BB, 16);
    p.off_list = o;  // uint16 cell or voxel indices, canonical order
    o = align_up(o + 2 * B * B * B, 16);
    p.off_vmsk = o;
    o = align_up(o + T3, 16);
    p.off_jobs = o;
    o = align_up(o + 4 * kRing, 16);
    p.off_vp = p.off_jobs;  // 4 * BB <= 4 * kRing for B <= 16
    p.off_tp = p.off_tile[0];  // the count phase's triangle prefixes: the tile is dead there
    p.off_nvid = p.off_nm = 0;  // unused
    p.bytes = o;
    return p;
}

// Plain loads of a block's (B+1)^3 tile as float (tile_load_float) that also
// build its inside masks (build_rows<float>): the inside bits of 32
// consecutive tile voxels -- in the volume and at or below the isovalue --
// are one warp ballot, a word of the tile's bitstream (kept in the list
// region, which is free until the block's cells are listed), and row (y, z)
// is the B+1 bits from bit (z*(B+1) + y)*(B+1) on.  The layout's tile pitch
// is B+1, so voxel i of the tile is tile[i].
template <typename S>
__device__ __forceinline__ void tile_load_rows_from(const Problem &p, const WPlan &pl, unsigned char *ws,
                                                    const Geo &g) {
    // four loads a lane in flight: the loop is inlined six times (three
    // dtypes, count and emit phases) and a smaller kernel keeps the
    // instruction cache from stalling the warps (batched mix: 35.7 ms at
    // eight, 33.5 ms at four, 34.7 ms at two; one loop for all dtypes with a
    // per-load branch, 34.6 ms)
    constexpr uint32_t kLdgBatch = 4;
    const S *vol = reinterpret_cast<const S *>(p.vol);
    float *tile = reinterpret_cast<float *>(ws + pl.off_tile[0]);
    uint32_t *words = reinterpret_cast<uint32_t *>(ws + pl.off_list);
    uint32_t *rows = reinterpret_cast<uint32_t *>(ws + pl.off_rows);
    const uint32_t lane = threadIdx.x & 31, B1 = pl.B1, n = B1 * B1 * B1, nw = (n + 31) / 32;
    for (uint32_t i0 = 0; i0 < n; i0 += 32 * kLdgBatch) {
        float v[kLdgBatch];
        bool in[kLdgBatch];
#pragma unroll
        for (uint32_t k = 0; k < kLdgBatch; ++k) {
            const uint32_t i = i0 + k * 32 + lane;
            const uint32_t iq = fdiv(i, pl.rB1);
            const uint32_t x = i - iq * B1, z = fdiv(iq, pl.rB1), y = iq - z * B1;
            const uint32_t gx = g.ox + x, gy = g.oy + y, gz = g.oz + z;
            in[k] = i < n && gx < p.X && gy < p.Y && gz < p.Z;
            v[k] = in[k] ? Vox<S>::val(__ldg(vol + ((uint64_t)gz * p.Y + gy) * p.X + gx)) : 0.0f;
        }
#pragma unroll
        for (uint32_t k = 0; k < kLdgBatch; ++k) {
            const uint32_t i = i0 + k * 32 + lane, w = (i0 >> 5) + k;
            if (i < n) tile[i] = v[k];
            const uint32_t bal = __ballot_sync(0xffffffffu, in[k] && v[k] <= p.iso);
            if (lane == 0 && w < nw) words[w] = bal;
        }
    }
    __syncwarp();
    const uint32_t mask = (1u << B1) - 1u;
    for (uint32_t q = lane; q < B1 * B1; q += 32) {
        const uint32_t bit = q * B1, w = bit >> 5;
        const uint64_t two = (uint64_t)words[w] | (w + 1 < nw ? (uint64_t)words[w + 1] << 32 : 0ull);
        rows[q] = (uint32_t)(two >> (bit & 31)) & mask;
    }
    __syncwarp();
}

__device__ __forceinline__ void tile_load_rows(const Problem &p, const WPlan &pl, unsigned char *ws, const Geo &g) {
    if (p.dtype == MTX_DTYPE_U8) tile_load_rows_from<uint8_t>(p, pl, ws, g);
    else if (p.dtype == MTX_DTYPE_U16) tile_load_rows_from<uint16_t>(p, pl, ws, g);
    else tile_load_rows_from<float>(p, pl, ws, g);
}

// Cell (x, y, z) of linear index c (x fastest) of a B^3 block.
__device__ __forceinline__ void cell_xyz(const WPlan &pl, uint32_t c, uint32_t &x, uint32_t &y, uint32_t &z) {
    const uint32_t q = fdiv(c, pl.rB);
    x = c - q * pl.B;
    z = fdiv(q, pl.rB);
    y = q - z * pl.B;
}

// Row masks of the block: MIXED cells (mixed_cells) or CUT voxels (a cut
// owned edge, from the crossing rows).
enum RowSet { kMixedCells = 0, kCutVoxels = 1 };

template <RowSet S>
__device__ __forceinline__ uint32_t row_set(const Problem &p, const WPlan &pl, const Geo &g, const uint32_t *rows,
                                            const uint32_t *cross, uint32_t q) {
    if constexpr (S == kCutVoxels) {
        return cross[q] | cross[pl.BB + q] | cross[2 * pl.BB + q];
    } else {
        const uint32_t z = fdiv(q, pl.rB), y = q - z * pl.B;
        uint32_t inside;
        return mixed_cells(p, pl, g, rows, y, z, inside);
    }
}

// Writes the linear indices (q*B + x) of the block's cells or voxels in set S
// to the warp's list in canonical order and returns their number.  Lane l
// owns rows [l*R, l*R + R); a warp scan of the rows' counts gives each lane
// its place in the list.
template <RowSet S>
__device__ __forceinline__ uint32_t list_block(const Problem &p, const WPlan &pl, const Geo &g, unsigned char *ws) {
    const uint32_t lane = threadIdx.x & 31, B = pl.B, BB = pl.BB, R = (BB + 31) / 32;
    const uint32_t *rows = reinterpret_cast<const uint32_t *>(ws + pl.off_rows);
    const uint32_t *cross = reinterpret_cast<const uint32_t *>(ws + pl.off_cross);
    uint16_t *list = reinterpret_cast<uint16_t *>(ws + pl.off_list);
    uint32_t cnt = 0;
    for (uint32_t k = 0; k < R; ++k) {
        const uint32_t q = lane * R + k;
        if (q >= BB) break;
        cnt += __popc(row_set<S>(p, pl, g, rows, cross, q));
    }
    uint32_t total;
    uint32_t pos = warp_excl_scan(cnt, total);
    for (uint32_t k = 0; k < R; ++k) {
        const uint32_t q = lane * R + k;
        if (q >= BB) break;
        uint32_t m = row_set<S>(p, pl, g, rows, cross, q);
        while (m) {
            const uint32_t x = __ffs(m) - 1;
            m &= m - 1u;
            list[pos++] = (uint16_t)(q * B + x);
        }
    }
    __syncwarp();
    return total;
}

// Case index of listed cell c (a mixed cell, so inside the volume) and its
// position in the (B+1)^3 tile.
__device__ __forceinline__ uint32_t listed_case(const WPlan &pl, const uint32_t *rows, uint32_t c,
                                                uint32_t &tile_index) {
    uint32_t x, y, z;
    cell_xyz(pl, c, x, y, z);
    tile_index = (z * pl.B1 + y) * pl.B1 + x;
    return cell_case(rows, pl.B1, x, y, z);
}

// Crossing masks and vertex prefixes per row (block_counts), and with
// want_tris the block's triangle count by the row walk of block_counts (the
// count phase; its triangle prefixes land in the tile, dead by then).  The
// walk takes fewer instructions and less code than listing the mixed cells
// and counting them 32 at a time (batched mix 33.5 -> 32.6 ms).
__device__ __forceinline__ void block_counts_balanced(const Problem &p, const WPlan &pl, unsigned char *ws,
                                                      const Geo &g, const uint8_t *ntab, bool want_tris,
                                                      uint32_t &nv, uint32_t &nt) {
    block_counts(p, pl, ws, g, ntab, want_tris, nullptr, nv, nt);
    if (!want_tris) nt = 0;
}

// Count body (count_block) of the batched kernel, for a block whose tile and
// inside masks tile_load_rows staged.
__device__ __forceinline__ void count_block_balanced(const Problem &p, const WPlan &pl, unsigned char *ws,
                                                     const Geo &g, const uint8_t *ntab, mtx_meshlet_descriptor *dr,
                                                     uint32_t *fr) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t bnv, bnt;
    block_counts_balanced(p, pl, ws, g, ntab, true, bnv, bnt);
    if (lane == 0) *reinterpret_cast<uint2 *>(&dr->vertexCount) = make_uint2(bnv, bnt);
    write_face_records<false>(pl, ws, fr);
}

// ---------------------------------------------------------- vertex table
// The context layer's entries (some coordinate == B), straight from the
// gathered face records (gather_issue; nb_vb: lane c holds neighbour c's
// first vertex id).
template <int CPL>
__device__ __forceinline__ void fill_context_vertices(const WPlan &pl, unsigned char *ws, uint32_t nb_vb,
                                                      const uint32_t rec[CPL]) {
    const uint32_t lane = threadIdx.x & 31, B = pl.B, B1 = pl.B1, nb3 = pl.nb3;
    uint32_t *vtab = reinterpret_cast<uint32_t *>(ws + pl.off_vtab);
    uint8_t *vmsk = ws + pl.off_vmsk;
#pragma unroll
    for (uint32_t k = 0; k < CPL; ++k) {
        if (k * 32 >= nb3) continue;  // warp-uniform
        const uint32_t j = k * 32 + lane;
        uint32_t x, y, z;
        ctx_voxel(pl, j < nb3 ? j : 0, x, y, z);
        const uint32_t c = j < nb3 ? ((x == B) | ((y == B) << 1) | ((z == B) << 2)) : 1u;
        const uint32_t vb = __shfl_sync(0xffffffffu, nb_vb, c);
        if (j < nb3) {
            const bool present = rec[k] >> 31;
            const uint32_t i = (z * B1 + y) * B1 + x;
            vtab[i] = present ? vb + (rec[k] & 0xffffffu) : kNoVertex;
            vmsk[i] = present ? (uint8_t)((rec[k] >> 24) & 7u) : (uint8_t)0;
        }
    }
}

// The block's own voxels, from the crossing rows.  Lane l owns rows
// [l*R, l*R + R), as in block_counts, so one warp scan of the rows' vertex
// counts gives every row its first vertex.
__device__ __forceinline__ void fill_own_vertices(const WPlan &pl, unsigned char *ws, uint32_t vbase) {
    const uint32_t lane = threadIdx.x & 31, B = pl.B, BB = pl.BB, B1 = pl.B1, R = (BB + 31) / 32;
    const uint32_t *cross = reinterpret_cast<const uint32_t *>(ws + pl.off_cross);
    uint32_t *vtab = reinterpret_cast<uint32_t *>(ws + pl.off_vtab);
    uint8_t *vmsk = ws + pl.off_vmsk;
    uint32_t cnt = 0;
    for (uint32_t k = 0; k < R; ++k) {
        const uint32_t q = lane * R + k;
        if (q >= BB) break;
        cnt += __popc(cross[q]) + __popc(cross[BB + q]) + __popc(cross[2 * BB + q]);
    }
    uint32_t tot;
    uint32_t run = vbase + warp_excl_scan(cnt, tot);
    for (uint32_t k = 0; k < R; ++k) {
        const uint32_t q = lane * R + k;
        if (q >= BB) break;
        const uint32_t z = fdiv(q, pl.rB), y = q - z * B, row = (z * B1 + y) * B1;
        const uint32_t xc = cross[q], yc = cross[BB + q], zc = cross[2 * BB + q];
        for (uint32_t x = 0; x < B; ++x) {
            const uint32_t m = ((xc >> x) & 1u) | (((yc >> x) & 1u) << 1) | (((zc >> x) & 1u) << 2);
            vmsk[row + x] = (uint8_t)m;
            vtab[row + x] = run;
            run += __popc(m);
        }
    }
    __syncwarp();
}

// Vertex id of cube edge e of the cell at tile index c: the owner voxel
// (c + dx + dy*B1 + dz*B1^2, owner byte dx | dy << 1 | dz << 2 | axis << 3)
// and the owned edges of lower axes before it.  EO: the CTA's edge-offset
// table (edge_offsets, after the owner bytes) holds offset | axis << 8 for a
// block edge known at compile time.
template <bool EO = false>
__device__ __forceinline__ uint32_t table_vertex(uint32_t c, uint32_t e, const uint8_t *owner, uint32_t B1,
                                                 const uint32_t *vtab, const uint8_t *vmsk, bool &bad) {
    uint32_t i, ax;
    if constexpr (EO) {
        const uint32_t eo = reinterpret_cast<const uint16_t *>(owner + 16)[e];
        i = c + (eo & 0xffu);
        ax = eo >> 8;
    } else {
        const uint32_t o = owner[e];
        i = c + (o & 1u) + ((o >> 1) & 1u) * B1 + ((o >> 2) & 1u) * B1 * B1;
        ax = o >> 3;
    }
    const uint32_t m = vmsk[i];
    bad |= !((m >> ax) & 1u);
    return vtab[i] + __popc(m & ((1u << ax) - 1u));
}

// ---------------------------------------------------------- resolution
// Vertex jobs [done, done + n), n <= 32, one per lane: job = tile index of
// the owner voxel | axis << 13, at jobs[i & (kRing - 1)].
template <bool GENERIC>
__device__ __forceinline__ void resolve_vertices(const Problem &p, const WPlan &pl, unsigned char *ws, const Geo &g,
                                                 uint32_t done, uint32_t n, uint32_t vbase, void *vertices,
                                                 uint32_t vfmt, uint32_t frame, uint32_t normals) {
    const uint32_t lane = threadIdx.x & 31, B1 = pl.B1;
    const float *tile = reinterpret_cast<const float *>(ws + pl.off_tile[0]);
    const uint32_t *jobs = reinterpret_cast<const uint32_t *>(ws + pl.off_jobs);
    const bool xyz = !GENERIC || vfmt == MTX_VERTEX_XYZ;
    if (lane < n) {
        const uint32_t job = jobs[(done + lane) & (kRing - 1)];
        const uint32_t t3 = job & 0x1fffu, a = job >> 13;
        const uint32_t iq = fdiv(t3, pl.rB1);
        const uint32_t x = t3 - iq * B1, z = fdiv(iq, pl.rB1), y = iq - z * B1;
        float t;
        const float3 pos = vertex_pos<float>(p, pl, tile, g, x, y, z, a, GENERIC && frame == MTX_FRAME_NDC, &t);
        if (xyz) {  // each lane its own 12 bytes, as the triangles
            float *o = reinterpret_cast<float *>(vertices) + 3ull * (vbase + done + lane);
            o[0] = pos.x;
            o[1] = pos.y;
            o[2] = pos.z;
        } else {
            float3 nn = make_float3(0.0f, 0.0f, 0.0f);
            if (normals) nn = vertex_normal_any(p, g.ox + x, g.oy + y, g.oz + z, a, t);
            float4 *o = reinterpret_cast<float4 *>(vertices) + 2ull * (vbase + done + lane);
            o[0] = make_float4(pos.x, pos.y, pos.z, 1.0f);
            o[1] = make_float4(nn.x, nn.y, nn.z, 0.0f);
        }
    }
    __syncwarp();
}

// Triangle jobs [done, done + n), n <= 32, one per lane: job = tile index of
// the cell | t << 13 | case << 16; writes the n triangles from dst on.
template <bool EO = false>
__device__ __forceinline__ void resolve_triangles(const WPlan &pl, unsigned char *ws, const uint64_t *tab,
                                                  const uint8_t *owner, uint32_t done, uint32_t n, uint32_t *dst,
                                                  bool &bad) {
    const uint32_t lane = threadIdx.x & 31, B1 = pl.B1;
    const uint32_t *vtab = reinterpret_cast<const uint32_t *>(ws + pl.off_vtab);
    const uint8_t *vmsk = ws + pl.off_vmsk;
    const uint32_t *jobs = reinterpret_cast<const uint32_t *>(ws + pl.off_jobs);
    // each lane stores its own 12 bytes: the warp's stores cover one 384-byte
    // span, which L2 merges, and no staging round trip is spent
    if (lane < n) {
        const uint32_t job = jobs[(done + lane) & (kRing - 1)];
        const uint32_t cell = job & 0x1fffu, t = (job >> 13) & 7u;
        const uint64_t w = tab[job >> 16] >> (4 + 12 * t);
        dst[3 * lane + 0] = table_vertex<EO>(cell, (uint32_t)(w & 0xFu), owner, B1, vtab, vmsk, bad);
        dst[3 * lane + 1] = table_vertex<EO>(cell, (uint32_t)((w >> 4) & 0xFu), owner, B1, vtab, vmsk, bad);
        dst[3 * lane + 2] = table_vertex<EO>(cell, (uint32_t)((w >> 8) & 0xFu), owner, B1, vtab, vmsk, bad);
    }
    __syncwarp();
}

// ---------------------------------------------------------- emit body
// First half of the emit body (emit_block) for a block whose float tile is
// staged: checks the capacities, writes the block's vertices and returns
// whether its triangles are still to be written (emit_triangles_balanced,
// after the caller has put the context layer into the vertex table).
template <bool GENERIC>
__device__ __forceinline__ bool emit_vertices_balanced(const Problem &p, const WPlan &pl, unsigned char *ws,
                                                       const Geo &g, const mtx_meshlet_descriptor &d,
                                                       const uint8_t *ntab, uint64_t tcap, void *vertices,
                                                       uint64_t vcap, uint32_t vfmt, uint32_t frame,
                                                       uint32_t normals, DevStatus *st, uint32_t r) {
    const uint32_t lane = threadIdx.x & 31, B = pl.B, BB = pl.BB, B1 = pl.B1;
    const uint32_t *cross = reinterpret_cast<const uint32_t *>(ws + pl.off_cross);
    const uint16_t *list = reinterpret_cast<const uint16_t *>(ws + pl.off_list);
    uint32_t *jobs = reinterpret_cast<uint32_t *>(ws + pl.off_jobs);
    const uint32_t tbase = d.indexOffset / 3u;
    if ((uint64_t)tbase + d.primitiveCount > tcap || (vertices && (uint64_t)d.vertexOffset + d.vertexCount > vcap)) {
        if (lane == 0) report(st, MTX_ERR_CAPACITY, kSiteEmitCapacity, r, 2);
        return false;
    }
    if (!(d.primitiveCount || (vertices && d.vertexCount))) return false;
    uint32_t bnv, bnt;
    block_counts_balanced(p, pl, ws, g, ntab, false, bnv, bnt);
    if (lane == 0 && bnv != d.vertexCount) report(st, MTX_ERR_INTERNAL, kSiteEmitNeighbour, r, 2);

    // vertices: the cut voxels 32 at a time; a warp scan of their cut-edge
    // counts queues the jobs (tile index | axis << 13) in the ring
    if (vertices && bnv) {
        const uint32_t nc = list_block<kCutVoxels>(p, pl, g, ws);
        uint32_t top = 0, done = 0;  // vertices queued, vertices written
        for (uint32_t v0 = 0; v0 < nc; v0 += 32) {
            uint32_t m = 0, ti = 0;
            if (v0 + lane < nc) {
                uint32_t x, y, z;
                cell_xyz(pl, list[v0 + lane], x, y, z);
                const uint32_t q = z * B + y;
                m = ((cross[q] >> x) & 1u) | (((cross[BB + q] >> x) & 1u) << 1) |
                    (((cross[2 * BB + q] >> x) & 1u) << 2);
                ti = (z * B1 + y) * B1 + x;
            }
            uint32_t tot;
            uint32_t j = top + warp_excl_scan(__popc(m), tot);
            for (uint32_t a = 0; a < 3; ++a)
                if ((m >> a) & 1u) jobs[(j++) & (kRing - 1)] = ti | (a << 13);
            top += tot;
            __syncwarp();
            const bool last = v0 + 32 >= nc;
            while (top - done >= (last ? 1u : 32u)) {
                const uint32_t n = min(32u, top - done);
                resolve_vertices<GENERIC>(p, pl, ws, g, done, n, d.vertexOffset, vertices, vfmt, frame, normals);
                done += n;
            }
        }
    }
    return d.primitiveCount != 0;
}

// Second half: the block's own voxels into the vertex table, then its
// triangles.
template <bool EO = false>
__device__ __forceinline__ void emit_triangles_balanced(const Problem &p, const WPlan &pl, unsigned char *ws,
                                                        const Geo &g, const mtx_meshlet_descriptor &d,
                                                        const uint64_t *tab, const uint8_t *ntab,
                                                        const uint8_t *owner, uint32_t *indices, DevStatus *st,
                                                        uint32_t r) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t *rows = reinterpret_cast<const uint32_t *>(ws + pl.off_rows);
    const uint16_t *list = reinterpret_cast<const uint16_t *>(ws + pl.off_list);
    uint32_t *jobs = reinterpret_cast<uint32_t *>(ws + pl.off_jobs);
    const uint32_t tbase = d.indexOffset / 3u;
    fill_own_vertices(pl, ws, d.vertexOffset);
    // triangles: the mixed cells 32 at a time; a warp scan of their triangle
    // counts queues the jobs (tile index | t << 13 | case << 16) in the ring
    const uint32_t nt = d.primitiveCount;
    const uint32_t nmix = list_block<kMixedCells>(p, pl, g, ws);
    bool bad = false;
    uint32_t top = 0, done = 0;  // triangles queued, triangles written
    for (uint32_t c0 = 0; c0 < nmix; c0 += 32) {
        uint32_t n = 0, cfg = 0, ti = 0;
        if (c0 + lane < nmix) {
            cfg = listed_case(pl, rows, list[c0 + lane], ti);
            n = ntab[cfg];
        }
        uint32_t tot;
        const uint32_t j = top + warp_excl_scan(n, tot);
        for (uint32_t t = 0; t < n; ++t) jobs[(j + t) & (kRing - 1)] = ti | (t << 13) | (cfg << 16);
        top += tot;
        __syncwarp();
        const bool last = c0 + 32 >= nmix;
        const uint32_t avail = min(top, nt);  // never write past the block's triangles
        while (avail - done >= (last ? 1u : 32u)) {
            const uint32_t n32 = min(32u, avail - done);
            resolve_triangles<EO>(pl, ws, tab, owner, done, n32, indices + 3ull * (tbase + done), bad);
            done += n32;
        }
    }
    bad |= top != nt;
    if (bad) report(st, MTX_ERR_INTERNAL, kSiteEmitNeighbour, r, 3);
}

}  // namespace mtx
