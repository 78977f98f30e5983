// Volume ingest and mesh export around the extraction path: meshtrex's
// loadVolume (src/volume.h:14-43) and writeGPUExtractionToOBJ
// (src/extractionTestUtils.cpp:203-369).  Host code only.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <regex>
#include <string>
#include <vector>

#include "mtx_internal.h"

using namespace mtx;

namespace {

constexpr size_t kStageBytes = 64ull << 20;  // one pinned staging buffer of the streamed upload

struct File {
    FILE *f = nullptr;
    explicit File(const char *path, const char *mode) { f = fopen(path, mode); }
    ~File() {
        if (f) fclose(f);
    }
};

}  // namespace

extern "C" {

mtx_status mtx_parse_volume_name(const char *path, uint32_t dims[3], uint32_t *dtype) {
    if (!path || !dims || !dtype) return MTX_ERR_INVALID_ARG;
    const std::string p(path);
    const size_t slash = p.find_last_of('/');
    const std::string base = slash == std::string::npos ? p : p.substr(slash + 1);
    // <name>_<X>x<Y>x<Z>_<type>.raw, the scheme of src/volume.h:18
    static const std::regex scheme(R"(^(\w+)_(\d+)x(\d+)x(\d+)_(.+)\.raw$)");
    std::smatch m;
    if (!std::regex_match(base, m, scheme)) return MTX_ERR_INVALID_ARG;
    for (int a = 0; a < 3; ++a) {
        const unsigned long v = std::stoul(m[2 + a].str());
        if (v == 0 || v > 0xffffffffull) return MTX_ERR_INVALID_ARG;
        dims[a] = (uint32_t)v;
    }
    const std::string t = m[5].str();
    if (t == "uint8") *dtype = MTX_DTYPE_U8;
    else if (t == "uint16") *dtype = MTX_DTYPE_U16;
    else if (t == "float32" || t == "float") *dtype = MTX_DTYPE_F32;
    else return MTX_ERR_UNSUPPORTED;
    return MTX_OK;
}

mtx_status mtx_volume_load(mtx_context_t c, const char *path, mtx_volume *out) {
    if (!c || !path || !out) return c ? fail(c, MTX_ERR_INVALID_ARG, "null argument") : MTX_ERR_INVALID_ARG;
    DeviceGuard dg(c->device);
    join_extract(c);
    memset(out, 0, sizeof(*out));
    uint32_t dims[3], dtype;
    mtx_status rs = mtx_parse_volume_name(path, dims, &dtype);
    if (rs != MTX_OK)
        return fail(c, rs, std::string("'") + path + "' does not follow <name>_<X>x<Y>x<Z>_<uint8|uint16|float32>.raw");
    const size_t bytes = nvox(dims) * dtype_size(dtype);
    File in(path, "rb");
    if (!in.f) return fail(c, MTX_ERR_INVALID_ARG, std::string("cannot open ") + path);
    void *dev = nullptr;
    if ((rs = dev_alloc(c, &dev, bytes)) != MTX_OK) return rs;
    // two pinned buffers: reading chunk k + 1 overlaps the copy of chunk k
    void *stage[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    const size_t chunk = std::min(bytes, kStageBytes);
    auto cleanup = [&](bool keep) {
        for (int i = 0; i < 2; ++i) {
            if (done[i]) cudaEventDestroy(done[i]);
            if (stage[i]) cudaFreeHost(stage[i]);
        }
        if (!keep) dev_free(c, dev);
    };
    for (int i = 0; i < 2; ++i) {
        cudaError_t e = cudaHostAlloc(&stage[i], chunk, cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming);
        if (e != cudaSuccess) {
            cleanup(false);
            return cuda_fail(c, e, "pinned staging for volume load");
        }
    }
    size_t off = 0;
    for (int k = 0; off < bytes; ++k) {
        const int i = k & 1;
        const size_t n = std::min(chunk, bytes - off);
        cudaError_t e = cudaEventSynchronize(done[i]);  // the copy that last used this buffer
        if (e == cudaSuccess && fread(stage[i], 1, n, in.f) != n) {
            cudaStreamSynchronize(c->stream);  // the other buffer's copy may be in flight
            cleanup(false);
            return fail(c, MTX_ERR_INVALID_ARG, std::string(path) + " is shorter than its name says");
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync((char *)dev + off, stage[i], n, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(done[i], c->stream);
        if (e != cudaSuccess) {
            cudaStreamSynchronize(c->stream);
            cleanup(false);
            return cuda_fail(c, e, "volume load copy");
        }
        off += n;
    }
    cudaError_t e = cudaStreamSynchronize(c->stream);
    cleanup(e == cudaSuccess);
    if (e != cudaSuccess) return cuda_fail(c, e, "volume load");
    out->data.ptr = dev;
    out->data.size = bytes;
    memcpy(out->dims, dims, sizeof(dims));
    out->dtype = dtype;
    out->owned = 1;
    return MTX_OK;
}

mtx_status mtx_write_obj(const char *path, const float *vertices, uint32_t vertexCount, uint32_t vertexStride,
                         const uint32_t *indices, uint32_t indexCount, mtx_obj_stats *stats) {
    if (!path || (vertexCount && !vertices) || (indexCount && !indices) || indexCount % 3 ||
        (vertexStride != 3 && vertexStride != 8))
        return MTX_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < indexCount; ++i)
        if (indices[i] >= vertexCount) return MTX_ERR_INVALID_ARG;
    // weld check: vertices with identical position (and normal) bits, and
    // triangles that repeat a vertex or a position
    const uint32_t key_words = vertexStride == 8 ? 6u : 3u;
    std::vector<uint32_t> order(vertexCount), canon(vertexCount);
    auto key = [&](uint32_t v, uint32_t w) {
        uint32_t b;
        memcpy(&b, vertices + (size_t)v * vertexStride + (w < 3 ? w : w + 1), 4);
        return b;
    };
    for (uint32_t v = 0; v < vertexCount; ++v) order[v] = v;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        for (uint32_t w = 0; w < key_words; ++w)
            if (key(a, w) != key(b, w)) return key(a, w) < key(b, w);
        return a < b;
    });
    uint32_t unique = 0;
    for (uint32_t i = 0; i < vertexCount; ++i) {
        bool same = i > 0;
        for (uint32_t w = 0; same && w < key_words; ++w) same = key(order[i], w) == key(order[i - 1], w);
        if (!same) ++unique;
        canon[order[i]] = same ? canon[order[i - 1]] : order[i];
    }
    uint32_t degenerate = 0;
    for (uint32_t t = 0; t < indexCount; t += 3) {
        const uint32_t a = canon[indices[t]], b = canon[indices[t + 1]], d = canon[indices[t + 2]];
        if (a == b || b == d || a == d) ++degenerate;
    }
    if (stats) {
        stats->vertexCount = vertexCount;
        stats->triangleCount = indexCount / 3;
        stats->uniqueVertexCount = unique;
        stats->degenerateTriangleCount = degenerate;
    }
    File out(path, "w");
    if (!out.f) return MTX_ERR_INVALID_ARG;
    FILE *f = out.f;
    fprintf(f, "# Generated by meshtrex-b200 (PMB: every vertex written once)\n");
    fprintf(f, "# %u vertices (%u distinct positions), %u triangles (%u degenerate)\n\n", vertexCount, unique,
            indexCount / 3, degenerate);
    fprintf(f, "# Vertex positions\n");
    for (uint32_t v = 0; v < vertexCount; ++v) {
        const float *p = vertices + (size_t)v * vertexStride;
        fprintf(f, "v %.9g %.9g %.9g\n", p[0], p[1], p[2]);
    }
    if (vertexStride == 8) {
        fprintf(f, "\n# Vertex normals\n");
        for (uint32_t v = 0; v < vertexCount; ++v) {
            const float *n = vertices + (size_t)v * 8 + 4;
            fprintf(f, "vn %.9g %.9g %.9g\n", n[0], n[1], n[2]);
        }
    }
    fprintf(f, "\n# Faces\n");
    for (uint32_t t = 0; t < indexCount; t += 3) {
        const uint32_t a = indices[t] + 1, b = indices[t + 1] + 1, d = indices[t + 2] + 1;
        if (vertexStride == 8) fprintf(f, "f %u//%u %u//%u %u//%u\n", a, a, b, b, d, d);
        else fprintf(f, "f %u %u %u\n", a, b, d);
    }
    if (ferror(f)) return MTX_ERR_INVALID_ARG;
    return MTX_OK;
}

}  // extern "C"
