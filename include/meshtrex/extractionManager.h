// extractMeshletDescriptors of the C++ drop-in facade (meshtrex:
// src/extractionManager.h:10-11), and writeGPUExtractionToOBJ
// (src/extractionTestUtils.cpp:203-369).
#pragma once

#include <vector>

#include "meshtrex/extractionOutput.h"
#include "meshtrex/filteringOutput.h"
#include "meshtrex/minMaxOutput.h"
#include "meshtrex/volume.h"

namespace meshtrex {

// options: vertex format, frame and normals (default: 12-byte xyz in the voxel
// frame; meshtrex's own layout is MTX_VERTEX_DATA in MTX_FRAME_NDC with normals).
inline ExtractionOutput extractMeshletDescriptors(Context &context, MinMaxOutput &minMax, FilteringOutput &filtering,
                                                  PushConstants &pushConstants, void *externalStream = nullptr,
                                                  GPUProfiler *profiler = nullptr,
                                                  const mtx_extract_options *options = nullptr) {
    StreamScope scope(context, externalStream);
    ExtractionOutput out;
    check(mtx_extract_meshlet_descriptors(context.handle(), &minMax.raw, &filtering.raw, &pushConstants, options,
                                          profilerHandle(profiler), &out.raw),
          context.handle(), "extractMeshletDescriptors");
    out.ctx = context.handle();
    out.refresh();
    return out;
}

// Copies the mesh back and writes it as OBJ; returns the weld check.
inline mtx_obj_stats writeGPUExtractionToOBJ(Context &context, ExtractionOutput &extraction, const char *filePath) {
    const uint32_t stride = extraction.vertexStride ? extraction.vertexStride / 4 : 3;
    std::vector<float> v((size_t)extraction.vertexCount * stride);
    std::vector<uint32_t> idx(extraction.indexCount);
    check(mtx_read_buffer(context.handle(), &extraction.raw.vertexBuffer, 0, v.data(), v.size() * 4),
          context.handle(), "writeGPUExtractionToOBJ: vertices");
    check(mtx_read_buffer(context.handle(), &extraction.raw.indexBuffer, 0, idx.data(), idx.size() * 4),
          context.handle(), "writeGPUExtractionToOBJ: indices");
    mtx_obj_stats stats{};
    check(mtx_write_obj(filePath, v.data(), extraction.vertexCount, stride, idx.data(), extraction.indexCount, &stats),
          nullptr, "writeGPUExtractionToOBJ");
    return stats;
}

}  // namespace meshtrex
