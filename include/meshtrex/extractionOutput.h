// ExtractionOutput, MeshletDescriptor and VertexData of the C++ drop-in facade
// (meshtrex: src/extractionOutput.h:10-134).
#pragma once

#include "meshtrex/context.h"

namespace meshtrex {

using MeshletDescriptor = mtx_meshlet_descriptor;  // {vertexOffset, indexOffset, vertexCount, primitiveCount}

struct vec4 {
    float x, y, z, w;
};
// The 32-byte vertex of the MTX_VERTEX_DATA format.
struct VertexData {
    vec4 position;
    vec4 normal;
};

// Buffers are sized exactly; the counts are on the host after
// extractMeshletDescriptors returns.  The destructor frees, as meshtrex's does.
struct ExtractionOutput {
    Buffer vertexBuffer;
    Buffer vertexCountBuffer;
    Buffer indexBuffer;
    Buffer indexCountBuffer;
    Buffer meshletDescriptorBuffer;
    Buffer meshletDescriptorCountBuffer;
    uint32_t meshletCount = 0;
    uint32_t vertexCount = 0;
    uint32_t indexCount = 0;
    uint32_t vertexStride = 0;  // 12 (xyz) or 32 (VertexData) bytes

    mtx_extraction_output raw{};
    mtx_context_t ctx = nullptr;

    ExtractionOutput() = default;
    ExtractionOutput(ExtractionOutput &&o) noexcept { *this = std::move(o); }
    ExtractionOutput &operator=(ExtractionOutput &&o) noexcept {
        if (this != &o) {
            cleanup();
            raw = o.raw;
            ctx = std::exchange(o.ctx, nullptr);
            refresh();
        }
        return *this;
    }
    ExtractionOutput(const ExtractionOutput &) = delete;
    ExtractionOutput &operator=(const ExtractionOutput &) = delete;
    ~ExtractionOutput() { cleanup(); }

    void cleanup() noexcept {
        if (ctx) mtx_extraction_free(ctx, &raw);
        ctx = nullptr;
        raw = mtx_extraction_output{};
        refresh();
    }

    void refresh() noexcept {
        vertexBuffer = toBuffer(raw.vertexBuffer);
        vertexCountBuffer = toBuffer(raw.vertexCountBuffer);
        indexBuffer = toBuffer(raw.indexBuffer);
        indexCountBuffer = toBuffer(raw.indexCountBuffer);
        meshletDescriptorBuffer = toBuffer(raw.meshletDescriptorBuffer);
        meshletDescriptorCountBuffer = toBuffer(raw.meshletDescriptorCountBuffer);
        meshletCount = raw.meshletCount;
        vertexCount = raw.vertexCount;
        indexCount = raw.indexCount;
        vertexStride = raw.vertexStride;
    }
};

}  // namespace meshtrex
