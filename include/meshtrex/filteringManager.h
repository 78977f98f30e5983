// filterActiveBlocks and readActiveBlockCount of the C++ drop-in facade
// (meshtrex: src/filteringManager.h:9-13).
#pragma once

#include "meshtrex/filteringOutput.h"
#include "meshtrex/minMaxOutput.h"
#include "meshtrex/volume.h"

namespace meshtrex {

inline FilteringOutput filterActiveBlocks(Context &context, MinMaxOutput &minMax, PushConstants &pushConstants,
                                          void *externalStream = nullptr, GPUProfiler *profiler = nullptr) {
    StreamScope scope(context, externalStream);
    FilteringOutput out;
    check(mtx_filter_active_blocks(context.handle(), &minMax.raw, &pushConstants, profilerHandle(profiler), &out.raw),
          context.handle(), "filterActiveBlocks");
    out.ctx = context.handle();
    out.refresh();
    return out;
}

inline void readActiveBlockCount(Context &context, FilteringOutput &filtering) {
    check(mtx_read_active_block_count(context.handle(), &filtering.raw), context.handle(), "readActiveBlockCount");
    filtering.refresh();
}

}  // namespace meshtrex
