// MinMaxOutput of the C++ drop-in facade (meshtrex: src/minMaxOutput.h:10-65).
#pragma once

#include <vector>

#include "meshtrex/context.h"

namespace meshtrex {

// One mip level of the min/max image: meshtrex's minMaxMipViews entry.
struct MipView {
    uint64_t offset = 0;  // texel offset of the level in minMaxImage (8 bytes per texel)
    uint32_t extent[3] = {0, 0, 0};
};

// Move-only, like meshtrex's.  cleanup() releases the device memory (meshtrex's
// cleanup(VkDevice)); the destructor calls it too.
struct MinMaxOutput {
    Buffer volumeImage;                  // the volume on the device
    Buffer minMaxImage;                  // {min,max} uint32 keys of every level, back to back
    std::vector<MipView> minMaxMipViews;
    uint32_t mipLevels = 0;

    mtx_minmax_output raw{};             // the C ABI view the next stages take
    mtx_volume ownedVolume{};            // set when computeMinMaxMip uploaded a host Volume
    mtx_context_t ctx = nullptr;

    MinMaxOutput() = default;
    MinMaxOutput(MinMaxOutput &&o) noexcept { *this = std::move(o); }
    MinMaxOutput &operator=(MinMaxOutput &&o) noexcept {
        if (this != &o) {
            cleanup();
            volumeImage = o.volumeImage;
            minMaxImage = o.minMaxImage;
            minMaxMipViews = std::move(o.minMaxMipViews);
            mipLevels = o.mipLevels;
            raw = o.raw;
            ownedVolume = o.ownedVolume;
            ctx = std::exchange(o.ctx, nullptr);
        }
        return *this;
    }
    MinMaxOutput(const MinMaxOutput &) = delete;
    MinMaxOutput &operator=(const MinMaxOutput &) = delete;
    ~MinMaxOutput() { cleanup(); }

    void cleanup() noexcept {
        if (!ctx) return;
        mtx_minmax_free(ctx, &raw);
        if (ownedVolume.owned) mtx_volume_free(ctx, &ownedVolume);
        ctx = nullptr;
        volumeImage = minMaxImage = Buffer{};
        minMaxMipViews.clear();
    }

    void refresh() {
        volumeImage = toBuffer(raw.volumeImage.data);
        minMaxImage = toBuffer(raw.minMaxImage);
        mipLevels = raw.mipLevels;
        minMaxMipViews.assign(mipLevels, MipView{});
        for (uint32_t l = 0; l < mipLevels; ++l) {
            minMaxMipViews[l].offset = raw.levelOffset[l];
            for (int a = 0; a < 3; ++a) minMaxMipViews[l].extent[a] = raw.levelExtent[l][a];
        }
    }
};

}  // namespace meshtrex
