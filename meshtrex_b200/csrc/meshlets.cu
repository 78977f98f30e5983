// Meshlet split: a post-pass over the canonical mesh that cuts each block's
// triangles into meshlets of at most maxVertices vertices and maxPrimitives
// triangles, each with its own copy of the vertices it uses -- the contract of
// meshtrex's renderer (render.task.glsl:55-250 accepts a triangle only if its
// three vertices lie in its meshlet's [vertexOffset, vertexOffset +
// vertexCount); the limits 64 / 126 are those of pmb.task.glsl:24-25).
//
// Rule (deterministic, the oracle's orc_meshlets): a block's triangles are
// taken in canonical order; a triangle joins the current meshlet unless its
// new vertices would take it past maxVertices or the meshlet already has
// maxPrimitives triangles, in which case a new meshlet starts with it.
// Meshlets never span blocks, and a meshlet's vertices are listed in the
// order its triangles first use them.
//
// One warp per block: lane k holds entries k and k + 32 of the current
// meshlet's vertex list, so a membership test is one compare and one ballot.
// A count pass sizes every block's meshlets, the descriptor scan places them,
// and the emit pass writes descriptors, meshlet vertex ids and indices.
#include <algorithm>

#include "mtx_internal.h"

namespace mtx {

constexpr uint32_t kMeshletWarps = 4;
constexpr uint32_t kMaxMeshletVertices = 64;

template <bool EMIT>
__global__ void __launch_bounds__(kMeshletWarps * 32)
    meshlet_kernel(const mtx_meshlet_descriptor *__restrict__ blocks, const uint32_t *__restrict__ count_ptr,
                   const uint32_t *__restrict__ indices, uint32_t maxV, uint32_t maxP,
                   mtx_meshlet_descriptor *__restrict__ per_block, mtx_meshlet_descriptor *__restrict__ meshlets,
                   uint32_t *__restrict__ mverts, uint32_t *__restrict__ midx) {
    __shared__ uint32_t s_list[kMeshletWarps][kMaxMeshletVertices];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *list = s_list[warp];
    const uint32_t n = *count_ptr;
    for (uint32_t r = blockIdx.x * kMeshletWarps + warp; r < n; r += gridDim.x * kMeshletWarps) {
        const mtx_meshlet_descriptor b = blocks[r];
        const uint32_t t0 = b.indexOffset / 3u, t1 = t0 + b.primitiveCount;
        uint32_t mbase = 0, vbase = 0;  // EMIT: the block's first meshlet and first meshlet vertex
        if (EMIT) {
            mbase = per_block[r].indexOffset / 3u;
            vbase = per_block[r].vertexOffset;
        }
        uint32_t mcount = 0, vused = 0;  // meshlets closed, their vertices
        uint32_t cur_v = 0, cur_p = 0, first_t = t0;
        for (uint32_t t = t0; t < t1; ++t) {
            const uint32_t c = lane < 3 ? __ldg(indices + 3ull * t + lane) : 0u;
            uint32_t id[3], loc[3];
            for (uint32_t k = 0; k < 3; ++k) id[k] = __shfl_sync(0xffffffffu, c, k);
            // local index of each corner in the current meshlet, or ~0
            for (uint32_t k = 0; k < 3; ++k) {
                const uint32_t m0 = __ballot_sync(0xffffffffu, lane < cur_v && list[lane] == id[k]);
                const uint32_t m1 = __ballot_sync(0xffffffffu, lane + 32 < cur_v && list[lane + 32] == id[k]);
                loc[k] = m0 ? (uint32_t)(__ffs(m0) - 1) : m1 ? 32u + (uint32_t)(__ffs(m1) - 1) : ~0u;
            }
            const bool n1 = loc[1] == ~0u && id[1] != id[0];
            const bool n2 = loc[2] == ~0u && id[2] != id[0] && id[2] != id[1];
            uint32_t fresh = (loc[0] == ~0u) + n1 + n2;
            if (cur_p > 0 && (cur_v + fresh > maxV || cur_p >= maxP)) {  // close the meshlet
                if (EMIT && lane == 0)
                    meshlets[mbase + mcount] = mtx_meshlet_descriptor{vbase + vused, 3u * first_t, cur_v, cur_p};
                vused += cur_v;
                ++mcount;
                cur_v = cur_p = 0;
                first_t = t;
                loc[0] = loc[1] = loc[2] = ~0u;
                fresh = 1u + (id[1] != id[0]) + (id[2] != id[0] && id[2] != id[1]);
            }
            // append the new corners in order (a repeated corner reuses its first slot)
            for (uint32_t k = 0; k < 3; ++k) {
                if (loc[k] != ~0u) continue;
                const uint32_t same = k > 0 && id[k] == id[0] ? loc[0] : (k > 1 && id[k] == id[1] ? loc[1] : ~0u);
                if (same != ~0u) {
                    loc[k] = same;
                    continue;
                }
                loc[k] = cur_v++;
                if (lane == 0) list[loc[k]] = id[k];
                if (EMIT && lane == 0) mverts[vbase + vused + loc[k]] = id[k];
            }
            __syncwarp();
            if (EMIT && lane < 3) midx[3ull * t + lane] = vbase + vused + (lane == 0 ? loc[0] : lane == 1 ? loc[1] : loc[2]);
            ++cur_p;
        }
        if (cur_p > 0) {
            if (EMIT && lane == 0)
                meshlets[mbase + mcount] = mtx_meshlet_descriptor{vbase + vused, 3u * first_t, cur_v, cur_p};
            vused += cur_v;
            ++mcount;
        }
        if (!EMIT && lane == 0) per_block[r] = mtx_meshlet_descriptor{0u, 0u, vused, mcount};
        __syncwarp();
    }
}

// vertexData[j] = vertices[mverts[j]], stride floats per record.
__global__ void gather_vertices_kernel(const float *__restrict__ vertices, const uint32_t *__restrict__ mverts,
                                       uint64_t n, uint32_t stride, float *__restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * stride;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t j = i / stride, k = i - j * stride;
        out[i] = __ldg(vertices + (uint64_t)__ldg(mverts + j) * stride + k);
    }
}

}  // namespace mtx

using namespace mtx;

extern "C" mtx_status mtx_build_meshlets(mtx_context_t c, const mtx_extraction_output *ext, uint32_t maxVertices,
                                         uint32_t maxPrimitives, mtx_meshlet_output *out) {
    if (!c) return MTX_ERR_INVALID_ARG;
    DeviceGuard dg(c->device);
    join_extract(c);
    if (!ext || !out) return fail(c, MTX_ERR_INVALID_ARG, "null argument");
    memset(out, 0, sizeof(*out));
    if (maxVertices < 3 || maxVertices > kMaxMeshletVertices || maxPrimitives < 1 || maxPrimitives > 1024)
        return fail(c, MTX_ERR_INVALID_ARG, "meshlet limits: 3 <= maxVertices <= 64, 1 <= maxPrimitives <= 1024");
    const uint32_t nb = ext->meshletCount, T = ext->indexCount / 3u;
    const uint32_t stride = ext->vertexStride ? ext->vertexStride / 4u : 3u;
    out->vertexStride = 4u * stride;
    if (nb == 0 || T == 0) return MTX_OK;
    if (!ext->meshletDescriptorBuffer.ptr || !ext->indexBuffer.ptr || !ext->vertexBuffer.ptr ||
        !ext->meshletDescriptorCountBuffer.ptr)
        return fail(c, MTX_ERR_INVALID_ARG, "extraction output is incomplete");
    cudaStream_t s = c->stream;
    void *per_block = nullptr, *counters = nullptr;
    mtx_status r;
    if ((r = dev_alloc(c, &per_block, sizeof(mtx_meshlet_descriptor) * (size_t)nb)) != MTX_OK) return r;
    auto bail = [&](mtx_status st) {
        dev_free(c, per_block);
        dev_free(c, counters);
        mtx_meshlet_output_free(c, out);
        return st;
    };
    if ((r = dev_alloc(c, &counters, 16)) != MTX_OK) return bail(r);
    const auto *blocks = (const mtx_meshlet_descriptor *)ext->meshletDescriptorBuffer.ptr;
    const auto *count = (const uint32_t *)ext->meshletDescriptorCountBuffer.ptr;
    const auto *indices = (const uint32_t *)ext->indexBuffer.ptr;
    const uint32_t grid = std::min<uint32_t>((nb + kMeshletWarps - 1) / kMeshletWarps, 16u * c->sm_count);
    meshlet_kernel<false><<<grid, kMeshletWarps * 32, 0, s>>>(blocks, count, indices, maxVertices, maxPrimitives,
                                                              (mtx_meshlet_descriptor *)per_block, nullptr, nullptr,
                                                              nullptr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return bail(cuda_fail(c, e, "meshlet count launch"));
    if ((r = launch_desc_scan(c, (mtx_meshlet_descriptor *)per_block, count, nb, (uint32_t *)counters, s)) != MTX_OK)
        return bail(r);
    uint32_t tot[4];
    if ((e = cudaMemcpyAsync(tot, counters, sizeof(tot), cudaMemcpyDeviceToHost, s)) == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bail(cuda_fail(c, e, "meshlet totals"));
    const uint32_t MV = tot[0], M = tot[1] / 3u;
    void *p_desc, *p_mv, *p_idx, *p_vd;
    if ((r = dev_alloc(c, &p_desc, sizeof(mtx_meshlet_descriptor) * (size_t)M)) != MTX_OK) return bail(r);
    out->meshletDescriptorBuffer = {p_desc, sizeof(mtx_meshlet_descriptor) * (uint64_t)M};
    if ((r = dev_alloc(c, &p_mv, 4ull * MV)) != MTX_OK) return bail(r);
    out->meshletVertexBuffer = {p_mv, 4ull * MV};
    if ((r = dev_alloc(c, &p_idx, 12ull * T)) != MTX_OK) return bail(r);
    out->indexBuffer = {p_idx, 12ull * T};
    if ((r = dev_alloc(c, &p_vd, 4ull * stride * MV)) != MTX_OK) return bail(r);
    out->vertexBuffer = {p_vd, 4ull * stride * MV};
    meshlet_kernel<true><<<grid, kMeshletWarps * 32, 0, s>>>(blocks, count, indices, maxVertices, maxPrimitives,
                                                             (mtx_meshlet_descriptor *)per_block,
                                                             (mtx_meshlet_descriptor *)p_desc, (uint32_t *)p_mv,
                                                             (uint32_t *)p_idx);
    if ((e = cudaGetLastError()) != cudaSuccess) return bail(cuda_fail(c, e, "meshlet emit launch"));
    const uint64_t work = (uint64_t)MV * stride;
    const uint32_t ggrid = (uint32_t)std::min<uint64_t>((work + 255) / 256, 8ull * c->sm_count);
    gather_vertices_kernel<<<std::max(1u, ggrid), 256, 0, s>>>((const float *)ext->vertexBuffer.ptr,
                                                               (const uint32_t *)p_mv, MV, stride, (float *)p_vd);
    if ((e = cudaGetLastError()) != cudaSuccess) return bail(cuda_fail(c, e, "meshlet gather launch"));
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return bail(cuda_fail(c, e, "meshlet build"));
    dev_free(c, per_block);
    dev_free(c, counters);
    out->meshletCount = M;
    out->vertexCount = MV;
    out->indexCount = 3u * T;
    return MTX_OK;
}

extern "C" mtx_status mtx_meshlet_output_free(mtx_context_t c, mtx_meshlet_output *out) {
    if (!c || !out) return MTX_ERR_INVALID_ARG;
    DeviceGuard dg(c->device);
    join_extract(c);
    dev_free(c, out->meshletDescriptorBuffer.ptr);
    dev_free(c, out->meshletVertexBuffer.ptr);
    dev_free(c, out->vertexBuffer.ptr);
    dev_free(c, out->indexBuffer.ptr);
    const uint32_t stride = out->vertexStride;
    memset(out, 0, sizeof(*out));
    out->vertexStride = stride;
    return MTX_OK;
}
