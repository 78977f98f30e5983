// computeMinMaxMip of the C++ drop-in facade (meshtrex: src/minMaxManager.h:20-21).
#pragma once

#include "meshtrex/minMaxOutput.h"
#include "meshtrex/volume.h"

namespace meshtrex {

// On a device-resident volume (no copy; it must outlive the output).
inline MinMaxOutput computeMinMaxMip(Context &context, const mtx_volume &volume, PushConstants &pushConstants,
                                     void *externalStream = nullptr, GPUProfiler *profiler = nullptr) {
    StreamScope scope(context, externalStream);
    MinMaxOutput out;
    check(mtx_compute_min_max_mip(context.handle(), &volume, &pushConstants, profilerHandle(profiler), &out.raw),
          context.handle(), "computeMinMaxMip");
    out.ctx = context.handle();
    out.refresh();
    return out;
}

// On host voxels, uploaded first (meshtrex passes Volume by value and stages it
// into volumeImage, minMaxManager.cpp:115-125); the output owns the upload.
inline MinMaxOutput computeMinMaxMip(Context &context, const Volume &volume, PushConstants &pushConstants,
                                     void *externalStream = nullptr, GPUProfiler *profiler = nullptr) {
    StreamScope scope(context, externalStream);
    const uint32_t dims[3] = {volume.volume_dims.x, volume.volume_dims.y, volume.volume_dims.z};
    mtx_volume dev{};
    check(mtx_volume_upload(context.handle(), volume.volume_data.data(), dims, volumeDtype(volume.volume_type), &dev),
          context.handle(), "computeMinMaxMip: upload");
    MinMaxOutput out;
    out.ownedVolume = dev;
    out.ctx = context.handle();
    check(mtx_compute_min_max_mip(context.handle(), &out.ownedVolume, &pushConstants, profilerHandle(profiler),
                                  &out.raw),
          context.handle(), "computeMinMaxMip");
    out.refresh();
    return out;
}

}  // namespace meshtrex
