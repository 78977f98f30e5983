// Adjoint of the PMB extraction with the topology held fixed: dL/dvertex ->
// dL/dfield (dense) and dL/diso.  meshtrex has no backward pass; the forward
// this differentiates is the vertex placement of marching_cubes_pmb.mesh.glsl:
// 122-141, p = u + t * e_axis with t = (iso - f(u)) / (f(u + e_axis) - f(u)).
//
// One warp per active block restages the block's (B+1)^3 tile as float,
// rebuilds the crossing masks and vertex prefixes exactly as the forward
// passes do (so vertex ids follow the forward's canonical order), and for
// each of the block's vertices recomputes t's inputs from the volume:
//   dL/df(u)  = g (iso - f(v)) / d^2,  dL/df(v) = g (f(u) - iso) / d^2,
//   dL/diso   = g / d,                 d = f(v) - f(u), v = u + e_axis.
// ATOMIC mode adds the field terms into dL/dfield with FP32 atomics.
// DETERMINISTIC mode accumulates them into a private (B+1)^3 tile in shared
// memory in six sweeps (axis x, y, z; the edge's first, then second voxel),
// in each of which every tile voxel has at most one writer, writes the tile
// out as the block's partial, and a gather pass then gives every voxel one
// designated block that sums the partials of the up to 8 blocks whose tiles
// hold it, in a fixed order.  dL/diso is summed per block and then over
// blocks in rank order in both modes.
#include "pmb_device.cuh"

namespace mtx {

constexpr uint32_t kAdjWarps = 4;
constexpr uint32_t kIsoThreads = 1024;

struct AdjArgs {
    Problem p;
    const uint32_t *ids;
    const uint32_t *rank_map;
    const mtx_meshlet_descriptor *desc;
    uint32_t n;           // active blocks
    uint32_t vcount;      // vertices of the forward mesh
    const float *g;       // dL/dvertex, gstride floats per vertex
    uint32_t gstride;
    float gscale[3];      // d(position)/dt per axis: 1 (voxel frame) or 2 / extent (NDC)
    float *dfield;
    float *partial;       // DETERMINISTIC: T3 floats per active block
    float *iso_part;      // dL/diso of each active block
    uint32_t T3;          // (B+1)^3
    uint32_t ws_bytes;    // shared memory per warp
    uint32_t off_acc;     // accumulation tile inside the warp's shared memory
    DevStatus *st;
};

template <bool DET>
__global__ void __launch_bounds__(kAdjWarps * 32) adjoint_block_kernel(const __grid_constant__ AdjArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    const Problem &p = a.p;
    const WPlan pl = make_wplan(p.B, 4, false, false, true);
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = blockDim.x >> 5;
    unsigned char *ws = smem + warp * a.ws_bytes;
    float *tile = reinterpret_cast<float *>(ws + pl.off_tile[0]);
    float *acc = reinterpret_cast<float *>(ws + a.off_acc);
    const uint32_t *cross = reinterpret_cast<const uint32_t *>(ws + pl.off_cross);
    const uint32_t *vp = reinterpret_cast<const uint32_t *>(ws + pl.off_vp);
    const uint32_t B = pl.B, BB = pl.BB, B1 = pl.B1, R = (BB + 31) / 32;
    const float iso = p.iso;
    for (uint32_t r = blockIdx.x * W + warp; r < a.n; r += gridDim.x * W) {
        const uint32_t id = __ldg(a.ids + r);
        const Geo g = block_geo(id, p, false, 4);
        const uint4 dq = __ldg(reinterpret_cast<const uint4 *>(a.desc + r));
        const uint32_t vbase = dq.x, nv = dq.z;
        tile_load_float(p, pl, tile, g);
        build_rows<float>(p, pl, ws, 0, g);
        uint32_t bnv, bnt;
        block_counts(p, pl, ws, g, nullptr, false, nullptr, bnv, bnt);
        const bool ok = bnv == nv && (uint64_t)vbase + nv <= a.vcount;
        if (!ok && lane == 0) report(a.st, MTX_ERR_INTERNAL, kSiteAdjoint, r, bnv);
        if (DET) {
            for (uint32_t i = lane; i < a.T3; i += 32) acc[i] = 0.0f;
            __syncwarp();
        }
        float diso = 0.0f;
        if (ok) {
            for (uint32_t ax = 0; ax < 3; ++ax) {
                const uint32_t step = ax == 0 ? 1u : ax == 1 ? B1 : B1 * B1;
                const uint64_t gstep = ax == 0 ? 1ull : ax == 1 ? (uint64_t)p.X : (uint64_t)p.X * p.Y;
                for (uint32_t role = 0; role < (DET ? 2u : 1u); ++role) {
                    for (uint32_t k = 0; k < R; ++k) {
                        const uint32_t q = lane * R + k;
                        if (q >= BB) break;
                        const uint32_t z = fdiv(q, pl.rB), y = q - z * B;
                        uint32_t m = cross[ax * BB + q];
                        while (m) {
                            const uint32_t x = __ffs(m) - 1;
                            m &= m - 1u;
                            uint32_t vid = vbase + voxel_prefix(cross, vp, BB, q, x);
                            for (uint32_t b = 0; b < ax; ++b) vid += (cross[b * BB + q] >> x) & 1u;
                            const uint32_t i0 = (z * B1 + y) * B1 + x, i1 = i0 + step;
                            const float fa = tile[i0], fb = tile[i1];
                            const float den = __fsub_rn(fb, fa);
                            if (!(fabsf(den) > 1e-5f)) continue;  // t = 0.5: no gradient
                            const float gv = __fmul_rn(__ldg(a.g + (uint64_t)vid * a.gstride + ax), a.gscale[ax]);
                            const float s = __fdiv_rn(gv, den);
                            if (DET) {
                                if (role == 0) {
                                    acc[i0] = __fadd_rn(acc[i0], __fdiv_rn(__fmul_rn(s, __fsub_rn(iso, fb)), den));
                                    diso = __fadd_rn(diso, s);
                                } else {
                                    acc[i1] = __fadd_rn(acc[i1], __fdiv_rn(__fmul_rn(s, __fsub_rn(fa, iso)), den));
                                }
                            } else {
                                const uint64_t v0 = ((uint64_t)(g.oz + z) * p.Y + (g.oy + y)) * p.X + (g.ox + x);
                                atomicAdd(a.dfield + v0, __fdiv_rn(__fmul_rn(s, __fsub_rn(iso, fb)), den));
                                atomicAdd(a.dfield + v0 + gstep, __fdiv_rn(__fmul_rn(s, __fsub_rn(fa, iso)), den));
                                diso = __fadd_rn(diso, s);
                            }
                        }
                    }
                    if (DET) __syncwarp();
                }
            }
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) diso = __fadd_rn(diso, __shfl_xor_sync(0xffffffffu, diso, o));
        if (lane == 0) a.iso_part[r] = diso;
        if (DET) {
            float *dst = a.partial + (uint64_t)r * a.T3;
            for (uint32_t i = lane; i < a.T3; i += 32) dst[i] = acc[i];
        }
        __syncwarp();
    }
}

// DETERMINISTIC: each voxel of an active block's (B+1)^3 tile is written by
// one designated block, the first active block in the order
// c(w) - (0,0,0), -(1,0,0), -(0,1,0), -(1,1,0), -(0,0,1), ... among those
// whose tiles hold w (c(w) the block containing w), as the sum of their
// partials in that order.
__global__ void __launch_bounds__(kAdjWarps * 32) adjoint_gather_kernel(const __grid_constant__ AdjArgs a) {
    const Problem &p = a.p;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = blockDim.x >> 5;
    const uint32_t B = p.B, B1 = B + 1;
    const uint32_t rB1 = (uint32_t)((0x100000000ull + B) / B1);
    for (uint32_t r = blockIdx.x * W + warp; r < a.n; r += gridDim.x * W) {
        const uint32_t id = __ldg(a.ids + r);
        const Geo g = block_geo(id, p, false, 4);
        for (uint32_t i = lane; i < a.T3; i += 32) {
            const uint32_t iq = fdiv(i, rB1);
            const uint32_t lx = i - iq * B1, lz = fdiv(iq, rB1), ly = iq - lz * B1;
            const uint32_t wx = g.ox + lx, wy = g.oy + ly, wz = g.oz + lz;
            if (wx >= p.X || wy >= p.Y || wz >= p.Z) continue;
            // containing block and the coordinates of w in it
            const uint32_t cx = g.bx + (lx == B), cy = g.by + (ly == B), cz = g.bz + (lz == B);
            const uint32_t ux = lx == B ? 0 : lx, uy = ly == B ? 0 : ly, uz = lz == B ? 0 : lz;
            uint32_t first = kNoVertex;
            float sum = 0.0f;
            for (uint32_t d = 0; d < 8; ++d) {
                const uint32_t dx = d & 1u, dy = (d >> 1) & 1u, dz = d >> 2;
                if ((dx && (ux || !cx)) || (dy && (uy || !cy)) || (dz && (uz || !cz))) continue;
                const uint32_t bx = cx - dx, by = cy - dy, bz = cz - dz;
                if (bx >= p.GX || by >= p.GY || bz >= p.GZ) continue;
                const uint32_t rk = __ldg(a.rank_map + ((uint64_t)bz * p.GY + by) * p.GX + bx);
                if (rk == kNoVertex) continue;
                if (first == kNoVertex) {
                    first = rk;
                    if (first != r) break;
                }
                const uint32_t j = ((uz + dz * B) * B1 + (uy + dy * B)) * B1 + (ux + dx * B);
                sum = __fadd_rn(sum, __ldcg(a.partial + (uint64_t)rk * a.T3 + j));
            }
            if (first == r) a.dfield[((uint64_t)wz * p.Y + wy) * p.X + wx] = sum;
        }
    }
}

// dL/diso: the per-block sums added in rank order (double accumulation, one CTA).
__global__ void __launch_bounds__(kIsoThreads) adjoint_iso_kernel(const float *__restrict__ part, uint32_t n,
                                                                  float *out) {
    __shared__ double s[kIsoThreads];
    double acc = 0.0;
    const uint32_t per = (n + kIsoThreads - 1) / kIsoThreads;
    const uint32_t b0 = threadIdx.x * per, b1 = min(n, b0 + per);
    for (uint32_t i = b0; i < b1; ++i) acc += (double)part[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (uint32_t h = kIsoThreads / 2; h; h >>= 1) {
        if (threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = (float)s[0];
}

MTX_BC_READER(bc_take_adjoint)

}  // namespace mtx

using namespace mtx;

extern "C" mtx_status mtx_extract_backward(mtx_context_t c, const mtx_volume *vol, const mtx_push_constants *pc,
                                           const mtx_filtering_output *filt, const mtx_meshlet_descriptor *meshlets,
                                           uint32_t vertexCount, const float *dl_dvertex, uint32_t vertexStride,
                                           uint32_t frame, float *dl_dfield, float *dl_diso, uint32_t mode) {
    if (!c) return MTX_ERR_INVALID_ARG;
    DeviceGuard dg(c->device);
    join_extract(c);
    if (!vol || !pc || !filt || !dl_dfield || !dl_diso) return fail(c, MTX_ERR_INVALID_ARG, "null argument");
    if (mode > MTX_ADJOINT_DETERMINISTIC || frame > MTX_FRAME_NDC || vertexStride < 3)
        return fail(c, MTX_ERR_INVALID_ARG, "bad adjoint mode, frame or vertex stride");
    mtx_status rs = check_volume(c, vol);
    if (rs != MTX_OK) return rs;
    if ((rs = check_pc(c, vol, pc)) != MTX_OK) return rs;
    const Problem p = make_problem(vol, pc->blockDim[0], pc->isovalue);
    const uint32_t n = filt->activeBlockCount;
    if (filt->totalBlocks != p.nblocks || n > p.nblocks)
        return fail(c, MTX_ERR_INVALID_ARG, "filtering output does not match the volume and block edge");
    if (n && (!meshlets || !filt->compactedBlockIdBuffer.ptr || !filt->blockRankBuffer.ptr ||
              (vertexCount && !dl_dvertex)))
        return fail(c, MTX_ERR_INVALID_ARG, "forward outputs are missing");
    if ((rs = load_case_tables(c)) != MTX_OK) return rs;
    cudaStream_t s = c->stream;
    mtx_profiler *prof = c->prof;
    prof_begin(prof, "Mesh_Extraction_Backward", s);
    MTX_CUDA(c, cudaMemsetAsync(dl_dfield, 0, nvox(vol->dims) * sizeof(float), s));
    if (n == 0) {
        MTX_CUDA(c, cudaMemsetAsync(dl_diso, 0, sizeof(float), s));
        prof_end(prof, s);
        return MTX_OK;
    }
    const bool det = mode == MTX_ADJOINT_DETERMINISTIC;
    const uint32_t B = p.B, T3 = (B + 1) * (B + 1) * (B + 1);
    if ((rs = scratch_reserve(c, c->adj_iso, sizeof(float) * (size_t)n)) != MTX_OK) return rs;
    if (det && (rs = scratch_reserve(c, c->adj_partial, sizeof(float) * (size_t)n * T3)) != MTX_OK) return rs;

    AdjArgs a{};
    a.p = p;
    a.ids = (const uint32_t *)filt->compactedBlockIdBuffer.ptr;
    a.rank_map = (const uint32_t *)filt->blockRankBuffer.ptr;
    a.desc = meshlets;
    a.n = n;
    a.vcount = vertexCount;
    a.g = dl_dvertex;
    a.gstride = vertexStride;
    for (int k = 0; k < 3; ++k) a.gscale[k] = frame == MTX_FRAME_NDC ? 2.0f / (float)vol->dims[k] : 1.0f;
    a.dfield = dl_dfield;
    a.partial = det ? (float *)c->adj_partial.ptr : nullptr;
    a.iso_part = (float *)c->adj_iso.ptr;
    a.T3 = T3;
    a.st = &c->ctrl->status;
    const WPlan pl = make_wplan(B, 4, false, false, true);
    a.off_acc = pl.bytes;
    a.ws_bytes = pl.bytes + (det ? align_up(4 * T3, 128) : 0u);
    const uint32_t smem = kAdjWarps * a.ws_bytes;
    auto kern = det ? adjoint_block_kernel<true> : adjoint_block_kernel<false>;
    MTX_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    MTX_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kAdjWarps * 32, smem));
    if (occ < 1) return fail(c, MTX_ERR_UNSUPPORTED, "adjoint warp layout does not fit shared memory");
    const uint32_t grid = std::min<uint32_t>((n + kAdjWarps - 1) / kAdjWarps, (uint32_t)(occ * c->sm_count));
    kern<<<grid, kAdjWarps * 32, smem, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "adjoint launch");
    if (det) {
        const uint32_t gg = std::min<uint32_t>((n + kAdjWarps - 1) / kAdjWarps, (uint32_t)(16 * c->sm_count));
        adjoint_gather_kernel<<<gg, kAdjWarps * 32, 0, s>>>(a);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "adjoint gather launch");
    }
    adjoint_iso_kernel<<<1, kIsoThreads, 0, s>>>(a.iso_part, n, dl_diso);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "adjoint isovalue launch");
    prof_end(prof, s);
    return MTX_OK;
}
