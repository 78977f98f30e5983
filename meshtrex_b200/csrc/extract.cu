// Stage 3: PMB marching cubes over the active blocks of one volume
// (meshtrex: marching_cubes_pmb.task.glsl:101-216 and
// marching_cubes_pmb.mesh.glsl:185-393, drawn by extractionManager.cpp:638-640).
//
// One warp owns one active block at a time; a CTA runs several such warps
// that share only the case tables (and, in the emit pass, the context-layer
// map).  Each warp stages the (B+1)^3 voxel tile of its block in shared
// memory (a TMA 3D tile, or plain loads when the volume's rows are not
// 16-byte aligned); the next block's tile is issued as soon as the current
// block is done.
//
//  count pass  per-block vertex/triangle counts, low-face records and, for
//              B <= 8, the block state the emit pass takes over
//  scan pass   decoupled look-back scan of the counts -> meshlet descriptors, totals
//  emit pass   vertices (each exactly once) and triangles, indices resolved
//              through the block's voxel table and the neighbours' face records
#include "pmb_device.cuh"

namespace mtx {

// One tile buffer a warp in the count and emit passes: without the second
// (prefetch) buffer a warp's region shrinks by a tile (2.7 KB for uint16 at
// B = 8), more CTAs fit an SM (emit: seven instead of five), and the other
// warps hide a tile's latency better than the prefetch did (per 1024^3
// extraction: emit 0.41 -> 0.33 ms, count 0.101 -> 0.095 ms).
constexpr bool kSingleBuffer = true;

// ------------------------------------------------------------- count pass
// BC: the block edge at compile time (0: p.B at run time).  The bench's edge 8
// has its own instantiation, in which the warp's shared-memory plan and every
// division by the edge fold to constants (48 registers).  The run-time form is
// held to 64 registers (no spills), where it would otherwise take up to 128.
template <typename T, bool TMA, int BC>
__global__ void __launch_bounds__(kMaxWarps * 32, BC ? 0 : 4)
    pmb_count_kernel(Problem p_, const __grid_constant__ CUtensorMap map, const uint32_t *__restrict__ ids,
                     const uint32_t *__restrict__ count_ptr, mtx_meshlet_descriptor *__restrict__ desc,
                     uint64_t desc_cap, uint32_t *__restrict__ faces, uint8_t *__restrict__ state,
                     uint32_t *totals, uint8_t *__restrict__ cell_cases, uint64_t block_cap, DevStatus *st) {
    extern __shared__ __align__(128) unsigned char smem[];
    Problem p = p_;
    if (BC) p.B = BC;
    const WPlan pl = make_wplan(p.B, sizeof(T), TMA, false, kSingleBuffer, p.B <= 8);
    const GridDiv dv = grid_div(p);
    uint8_t *ntab = smem + 2048;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = blockDim.x >> 5;
    unsigned char *ws = smem + kTableBytes + warp * pl.bytes;
    for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) ntab[i] = (uint8_t)(c_mc_cases[i] & 0xFu);
    if (lane == 0 && TMA) {
        uint64_t *bar = reinterpret_cast<uint64_t *>(ws + pl.off_bar);
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        fence_mbar_init();
    }
    __syncthreads();
    const uint32_t count = *count_ptr;
    if (count > block_cap || count > desc_cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            report(st, MTX_ERR_CAPACITY, kSiteEmitCapacity, count, 3);
            totals[3] = count;
        }
        return;
    }
    const uint32_t B3 = pl.BB * pl.B;
    const uint32_t gw = blockIdx.x * W + warp, nw = gridDim.x * W;
    uint32_t parity = 0, buf = 0;

    uint32_t r = gw;
    Geo g{};
    if (r < count) {
        g = block_geo(__ldg(ids + r), p, TMA, sizeof(T), dv);
        tile_issue<T, TMA>(pl, ws, buf, g, &map);
    }
    while (r < count) {
        const uint32_t rn = r + nw;
        Geo gn{};
        const bool have_next = rn < count;
        if (have_next) {
            gn = block_geo(__ldg(ids + rn), p, TMA, sizeof(T), dv);
            if (pl.nbuf == 2) tile_issue<T, TMA>(pl, ws, buf ^ 1u, gn, &map);
        }
        if (!tile_wait<T, TMA>(p, pl, ws, buf, g, parity, st)) {
            if (have_next && pl.nbuf == 2) tile_drain<TMA>(pl, ws, buf ^ 1u, parity);
            break;
        }
        // one tile buffer: the next tile is issued as soon as this block's rows are built
        const bool early = have_next && pl.nbuf == 1;
        count_block<T, TMA>(p, pl, ws, buf, g, ntab, cell_cases ? cell_cases + (uint64_t)r * B3 : nullptr, desc + r,
                            faces + (uint64_t)r * 3 * pl.BB,
                            (state && pl.state_bytes) ? state + (uint64_t)r * pl.state_bytes : nullptr,
                            early ? &gn : nullptr, &map);
        if (!have_next) break;
        if (pl.nbuf != 1) buf ^= 1u;
        r = rn;
        g = gn;
    }
}

// -------------------------------------------------------------- scan pass
__global__ void __launch_bounds__(kScanThreads)
    pmb_scan_kernel(mtx_meshlet_descriptor *__restrict__ desc, const uint32_t *__restrict__ count_ptr,
                    uint64_t *tile_status, uint32_t *ticket, uint32_t *totals, DevStatus *st, uint32_t spin_limit) {
    __shared__ uint32_t s_tile, s_ok;
    __shared__ uint64_t s_tmp[kScanThreads / 32 + 1];
    __shared__ uint64_t s_pre[2];
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    const uint32_t count = *count_ptr;
    if (t >= (count + kScanTile - 1) / kScanTile) return;
    scan_tile(desc, count, t, tile_status, totals, st, s_tmp, &s_ok, s_pre, spin_limit);
}

// -------------------------------------------------------------- emit pass
// CPL: context voxels per lane, ceil((3B^2 + 3B + 1) / 32): 8 covers B <= 8, 32 covers B <= 16.
// The xyz form of B <= 8 is bounded to 85 registers (three CTAs of 256
// threads); it uses 60 at the compile-time edge 8 and about 68 otherwise, with
// no spills; with 27.9 KB of shared memory a CTA of four warps (8- and 16-bit
// voxels) eight CTAs share an SM at edge 8.  The other forms would spill
// under that bound.
template <typename T, int CPL, bool TMA, bool GENERIC, int BC>
__global__ void __launch_bounds__(kMaxWarps * 32, (!GENERIC && CPL == 8) ? 3 : 1)
    pmb_emit_kernel(Problem p_, const __grid_constant__ CUtensorMap map, const uint32_t *__restrict__ ids,
                    const uint32_t *__restrict__ rank_map, const uint32_t *__restrict__ count_ptr,
                    const mtx_meshlet_descriptor *__restrict__ desc, const uint32_t *__restrict__ faces,
                    const uint8_t *__restrict__ state, uint32_t *__restrict__ indices, uint64_t tcap,
                    uint64_t block_cap, void *__restrict__ vertices, uint64_t vcap, uint32_t vfmt, uint32_t frame,
                    uint32_t normals, DevStatus *st) {
    // B <= 8 with TMA: the count pass's block state comes with each tile
    constexpr bool STATE = TMA && CPL == 8;
    extern __shared__ __align__(128) unsigned char smem[];
    Problem p = p_;
    if (BC) p.B = BC;
    const WPlan pl = make_wplan(p.B, sizeof(T), TMA, true, kSingleBuffer);
    const GridDiv dv = grid_div(p);
    uint64_t *tab = reinterpret_cast<uint64_t *>(smem);
    uint8_t *ntab = smem + 2048;
    uint8_t *owner = smem + 2048 + 256;
    uint32_t *cmap = reinterpret_cast<uint32_t *>(smem + kTableBytes);
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = blockDim.x >> 5;
    unsigned char *ws = smem + cta_fixed_bytes(p.B, true) + warp * pl.bytes;
    for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
        tab[i] = c_mc_cases[i];
        ntab[i] = (uint8_t)(c_mc_cases[i] & 0xFu);
    }
    for (uint32_t j = threadIdx.x; j < pl.nb3; j += blockDim.x) cmap[j] = ctx_map_entry(pl, j);
    if (threadIdx.x < 12) owner[threadIdx.x] = c_mc_owner[threadIdx.x];
    if (CPL == 8) edge_offsets(reinterpret_cast<uint16_t *>(owner + 16), pl.B1);
    if (lane == 0 && TMA) {
        uint64_t *bar = reinterpret_cast<uint64_t *>(ws + pl.off_bar);
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        fence_mbar_init();
    }
    __syncthreads();
    const uint32_t count = *count_ptr;
    if (count > block_cap) return;  // reported by the count pass
    const uint32_t gw = blockIdx.x * W + warp, nw = gridDim.x * W;
    uint32_t parity = 0, buf = 0;

    uint32_t r = gw;
    Geo g{};
    mtx_meshlet_descriptor d{};
    uint32_t nb_rk = kNoVertex;
    auto state_of = [&](uint32_t rr) -> const unsigned char * {
        return STATE ? state + (uint64_t)rr * pl.state_bytes : nullptr;
    };
    if (r < count) {
        const uint32_t id = __ldg(ids + r);
        g = block_geo(id, p, TMA, sizeof(T), dv);
        tile_issue<T, TMA>(pl, ws, buf, g, &map, state_of(r));
        d = desc[r];
        nb_rk = neighbour_rank(p, g, id, rank_map);
    }
    while (r < count) {
        // prefetch the next block: its tile, descriptor and neighbour ranks
        const uint32_t rn = r + nw;
        const bool have_next = rn < count;
        Geo gn{};
        mtx_meshlet_descriptor dn{};
        uint32_t nb_rk_n = kNoVertex;
        if (have_next) {
            const uint32_t idn = __ldg(ids + rn);
            gn = block_geo(idn, p, TMA, sizeof(T), dv);
            if (pl.nbuf == 2) tile_issue<T, TMA>(pl, ws, buf ^ 1u, gn, &map, state_of(rn));
            dn = desc[rn];
            nb_rk_n = neighbour_rank(p, gn, idn, rank_map);
        }
        const uint32_t nb_vb =
            (nb_rk != kNoVertex && MTX_BC(nb_rk, count, kBcDesc)) ? __ldg(&desc[nb_rk].vertexOffset) : kNoVertex;
        uint32_t rec[CPL];
        gather_issue_map<CPL>(p, pl, g, nb_rk, faces, 3 * pl.BB, cmap, rec, block_cap * 3 * pl.BB);
        if (!tile_wait<T, TMA>(p, pl, ws, buf, g, parity, st)) {
            if (have_next && pl.nbuf == 2) tile_drain<TMA>(pl, ws, buf ^ 1u, parity);
            break;
        }
        gather_finish<CPL, CPL == 8>(pl, nb_vb, rec, ws, d.vertexOffset);
        emit_block<T, GENERIC, false, CPL == 8, STATE>(p, pl, ws, buf, g, d, tab, ntab, owner, indices, tcap,
                                                       vertices, vcap, vfmt, frame, normals, st, r, cmap);
        if (!have_next) break;
        if (pl.nbuf == 1) tile_issue<T, TMA>(pl, ws, buf, gn, &map, state_of(rn));
        else buf ^= 1u;
        r = rn;
        d = dn;
        g = gn;
        nb_rk = nb_rk_n;
    }
}

// ------------------------------------------------------------------ host

bool tma_ok(const Problem &p) {
    const uint32_t esz = dtype_size(p.dtype);
    return ((uintptr_t)p.vol % 16 == 0) && (((uint64_t)p.X * esz) % 16 == 0);
}

static bool use_tma(const Problem &p, uint32_t staging) {
    if (staging == MTX_STAGING_LDG) return false;
    return tma_ok(p);
}

template <typename K>
static mtx_status grid_for(mtx_context *c, K kernel, int threads, uint32_t smem, uint32_t host_count, int warps,
                           unsigned &grid) {
    MTX_CUDA(c, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    MTX_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    if (per_sm < 1) return fail(c, MTX_ERR_UNSUPPORTED, "extraction kernel does not fit on an SM");
    if (c->tuning.extractCtasPerSm) per_sm = std::min(per_sm, (int)c->tuning.extractCtasPerSm);
    uint64_t g = (uint64_t)per_sm * c->sm_count;
    if (host_count) g = std::min<uint64_t>(g, (host_count + warps - 1) / warps);
    grid = (unsigned)std::max<uint64_t>(g, 1);
    return MTX_OK;
}

template <typename T>
static mtx_status run_count(mtx_context *c, const Problem &p, const ExtractArgs &a, const CUtensorMap &map, bool tma,
                            uint32_t W, cudaStream_t s) {
    const WPlan pl = make_wplan(p.B, sizeof(T), tma, false, kSingleBuffer, p.B <= 8);
    const uint32_t smem = kTableBytes + W * pl.bytes;
    auto k = tma ? (p.B == 8 ? pmb_count_kernel<T, true, 8> : pmb_count_kernel<T, true, 0>)
                 : pmb_count_kernel<T, false, 0>;
    unsigned grid;
    mtx_status r = grid_for(c, k, W * 32, smem, a.host_count, W, grid);
    if (r != MTX_OK) return r;
    k<<<grid, W * 32, smem, s>>>(p, map, a.ids, a.count, a.desc, a.desc_capacity, a.faces, a.state, a.totals,
                                 a.cell_cases, a.block_capacity, &c->ctrl->status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "count launch");
    return MTX_OK;
}

template <typename T, int CPL, bool TMA, int BC = 0>
static void (*emit_fn(bool generic))(Problem, CUtensorMap, const uint32_t *, const uint32_t *, const uint32_t *,
                                     const mtx_meshlet_descriptor *, const uint32_t *, const uint8_t *, uint32_t *,
                                     uint64_t, uint64_t, void *, uint64_t, uint32_t, uint32_t, uint32_t, DevStatus *) {
    return generic ? pmb_emit_kernel<T, CPL, TMA, true, BC> : pmb_emit_kernel<T, CPL, TMA, false, BC>;
}

template <typename T>
static mtx_status run_emit(mtx_context *c, const Problem &p, const ExtractArgs &a, const CUtensorMap &map, bool tma,
                           uint32_t W, cudaStream_t s) {
    const WPlan pl = make_wplan(p.B, sizeof(T), tma, true, kSingleBuffer);
    const uint32_t smem = cta_fixed_bytes(p.B, true) + W * pl.bytes;
    const bool generic = a.vertices && (a.vertex_format != MTX_VERTEX_XYZ || a.frame != MTX_FRAME_VOXEL);
    auto k = p.B == 8 && tma ? emit_fn<T, 8, true, 8>(generic)
             : p.B <= 8    ? (tma ? emit_fn<T, 8, true>(generic) : emit_fn<T, 8, false>(generic))
                           : (tma ? emit_fn<T, 32, true>(generic) : emit_fn<T, 32, false>(generic));
    unsigned grid;
    mtx_status r = grid_for(c, k, W * 32, smem, a.host_count, W, grid);
    if (r != MTX_OK) return r;
    k<<<grid, W * 32, smem, s>>>(p, map, a.ids, a.rank_map, a.count, a.desc, a.faces, a.state, a.indices,
                                 a.tri_capacity, a.block_capacity, a.vertices, a.vertex_capacity, a.vertex_format,
                                 a.frame, a.normals, &c->ctrl->status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "emit launch");
    return MTX_OK;
}

template <bool EMIT>
static mtx_status launch_stage(mtx_context *c, const Problem &p, const ExtractArgs &a, cudaStream_t s) {
    if (p.B < 2 || p.B > MTX_MAX_BLOCK_EDGE) return fail(c, MTX_ERR_UNSUPPORTED, "block edge must be in [2, 16]");
    mtx_status rs = load_case_tables(c);
    if (rs != MTX_OK) return rs;
    const uint32_t staging = a.staging ? a.staging : c->tuning.staging;
    const bool tma = use_tma(p, staging);
    CUtensorMap map;
    memset(&map, 0, sizeof(map));
    if (tma) {
        rs = make_volume_tensor_map(c, p, tile_pitch(p.B, dtype_size(p.dtype), true), &map);
        if (rs != MTX_OK) return rs;
    }
    // warps per CTA: threads/32 of the options, else the context's tuning, else 4
    uint32_t W = a.threads ? a.threads / 32 : (c->tuning.extractWarps ? c->tuning.extractWarps : 4);
    W = std::min<uint32_t>(std::max<uint32_t>(W, 1), kMaxWarps);
    // no more warps than the shared memory holds (16^3 float tiles fit 7, not 8)
    const WPlan pl = make_wplan(p.B, dtype_size(p.dtype), tma, EMIT, kSingleBuffer, p.B <= 8);
    // the emit pass with TMA and B <= 8 reads the block state the count pass wrote
    if (EMIT && tma && pl.state_bytes && !a.state) return fail(c, MTX_ERR_INTERNAL, "emit without block state");
    const uint32_t fixed = cta_fixed_bytes(p.B, EMIT);
    const uint32_t room = c->max_smem_optin > (int)fixed ? (uint32_t)c->max_smem_optin - fixed : 0u;
    W = std::min<uint32_t>(W, std::max<uint32_t>(1, room / pl.bytes));
    switch (p.dtype) {
    case MTX_DTYPE_U8: return EMIT ? run_emit<uint8_t>(c, p, a, map, tma, W, s) : run_count<uint8_t>(c, p, a, map, tma, W, s);
    case MTX_DTYPE_U16: return EMIT ? run_emit<uint16_t>(c, p, a, map, tma, W, s) : run_count<uint16_t>(c, p, a, map, tma, W, s);
    default: return EMIT ? run_emit<float>(c, p, a, map, tma, W, s) : run_count<float>(c, p, a, map, tma, W, s);
    }
}

uint32_t block_state_bytes(uint32_t B) { return make_wplan(B, 2, true, false, kSingleBuffer, B <= 8).state_bytes; }

// Counts, faces and the scan: after this the descriptors and totals are final.
mtx_status launch_count(mtx_context *c, const Problem &p, const ExtractArgs &a, cudaStream_t s) {
    const uint64_t cap = std::min<uint64_t>(a.block_capacity, a.desc_capacity);
    const uint32_t ntiles = (uint32_t)std::max<uint64_t>(1, (cap + kScanTile - 1) / kScanTile);
    mtx_status r = scratch_reserve(c, c->count_status, sizeof(uint64_t) * (size_t)ntiles);
    if (r != MTX_OK) return r;
    MTX_CUDA(c, cudaMemsetAsync(&c->ctrl->count_ticket, 0, sizeof(uint32_t), s));
    MTX_CUDA(c, cudaMemsetAsync(a.totals, 0, 4 * sizeof(uint32_t), s));
    MTX_CUDA(c, cudaMemsetAsync(c->count_status.ptr, 0, sizeof(uint64_t) * ntiles, s));
    if ((r = launch_stage<false>(c, p, a, s)) != MTX_OK) return r;
    if (c->withhold & 2u) {  // failure injection: scan tile 0 is never handed out
        static const uint32_t kOne = 1;
        MTX_CUDA(c, cudaMemcpyAsync(&c->ctrl->count_ticket, &kOne, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    }
    pmb_scan_kernel<<<ntiles, kScanThreads, 0, s>>>(a.desc, a.count, (uint64_t *)c->count_status.ptr,
                                                    &c->ctrl->count_ticket, a.totals, &c->ctrl->status,
                                                    c->wait_polls ? c->wait_polls : kSpinLimit);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "scan launch");
    return MTX_OK;
}

// The descriptor scan on its own: vertexOffset / indexOffset of count
// descriptors from their vertexCount / primitiveCount (totals as launch_count).
mtx_status launch_desc_scan(mtx_context *c, mtx_meshlet_descriptor *desc, const uint32_t *count, uint64_t capacity,
                            uint32_t *totals, cudaStream_t s) {
    const uint32_t ntiles = (uint32_t)std::max<uint64_t>(1, (capacity + kScanTile - 1) / kScanTile);
    mtx_status r = scratch_reserve(c, c->count_status, sizeof(uint64_t) * (size_t)ntiles);
    if (r != MTX_OK) return r;
    MTX_CUDA(c, cudaMemsetAsync(&c->ctrl->count_ticket, 0, sizeof(uint32_t), s));
    MTX_CUDA(c, cudaMemsetAsync(totals, 0, 4 * sizeof(uint32_t), s));
    MTX_CUDA(c, cudaMemsetAsync(c->count_status.ptr, 0, sizeof(uint64_t) * ntiles, s));
    pmb_scan_kernel<<<ntiles, kScanThreads, 0, s>>>(desc, count, (uint64_t *)c->count_status.ptr,
                                                    &c->ctrl->count_ticket, totals, &c->ctrl->status,
                                                    c->wait_polls ? c->wait_polls : kSpinLimit);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "scan launch");
    return MTX_OK;
}

// Vertices (when a.vertices is set) and triangles.
mtx_status launch_emit(mtx_context *c, const Problem &p, const ExtractArgs &a, cudaStream_t s) {
    return launch_stage<true>(c, p, a, s);
}

MTX_BC_READER(bc_take_extract)

}  // namespace mtx
