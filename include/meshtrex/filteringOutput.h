// FilteringOutput of the C++ drop-in facade (meshtrex: src/filteringOutput.h:11-74).
#pragma once

#include "meshtrex/context.h"

namespace meshtrex {

struct FilteringOutput {
    Buffer compactedBlockIdBuffer;  // ascending ids of the active blocks
    Buffer activeBlockCountBuffer;  // one uint32
    Buffer blockRankBuffer;         // rank of every block (0xffffffff if inactive); not in meshtrex
    uint32_t activeBlockCount = 0;  // host copy, filled by readActiveBlockCount

    mtx_filtering_output raw{};
    mtx_context_t ctx = nullptr;

    FilteringOutput() = default;
    FilteringOutput(FilteringOutput &&o) noexcept { *this = std::move(o); }
    FilteringOutput &operator=(FilteringOutput &&o) noexcept {
        if (this != &o) {
            cleanup();
            compactedBlockIdBuffer = o.compactedBlockIdBuffer;
            activeBlockCountBuffer = o.activeBlockCountBuffer;
            blockRankBuffer = o.blockRankBuffer;
            activeBlockCount = o.activeBlockCount;
            raw = o.raw;
            ctx = std::exchange(o.ctx, nullptr);
        }
        return *this;
    }
    FilteringOutput(const FilteringOutput &) = delete;
    FilteringOutput &operator=(const FilteringOutput &) = delete;
    ~FilteringOutput() { cleanup(); }

    void cleanup() noexcept {
        if (!ctx) return;
        mtx_filtering_free(ctx, &raw);
        ctx = nullptr;
        compactedBlockIdBuffer = activeBlockCountBuffer = blockRankBuffer = Buffer{};
    }

    void refresh() {
        compactedBlockIdBuffer = toBuffer(raw.compactedBlockIdBuffer);
        activeBlockCountBuffer = toBuffer(raw.activeBlockCountBuffer);
        blockRankBuffer = toBuffer(raw.blockRankBuffer);
        activeBlockCount = raw.activeBlockCount;
    }
};

}  // namespace meshtrex
