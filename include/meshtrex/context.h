// Context, errors and profiler of the C++ drop-in facade.  These stand in for
// meshtrex's VulkanContext (src/vulkan_context.h:7-45) in its compute role,
// its Buffer (src/buffer.h:3-8) and its GPUProfiler (src/gpuProfiler.h:11-160),
// on top of the C ABI in meshtrex/mtx.h.  Header only; link libmeshtrex_b200.
#pragma once

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>

#include "meshtrex/mtx.h"

namespace meshtrex {

// meshtrex throws std::runtime_error (extractionManager.cpp:276-356); so does the facade.
class Error : public std::runtime_error {
   public:
    Error(mtx_status s, const std::string &what) : std::runtime_error(what), status(s) {}
    mtx_status status;
};

inline void check(mtx_status s, mtx_context_t ctx, const char *what) {
    if (s == MTX_OK) return;
    std::string msg = std::string(what) + ": " + mtx_status_string(s);
    if (ctx) {
        const char *detail = mtx_context_last_error(ctx);
        if (detail && *detail) msg += std::string(" (") + detail + ")";
    }
    throw Error(s, msg);
}

// Buffer (src/buffer.h:3-8): `buffer` is the device pointer; device memory is
// not mapped, so `data` stays null.
struct Buffer {
    void *buffer = nullptr;
    void *data = nullptr;
    size_t size = 0;
};

inline Buffer toBuffer(const mtx_buffer &b) { return Buffer{b.ptr, nullptr, (size_t)b.size}; }

// The compute role of VulkanContext: one CUDA device and the stream work is
// issued on (meshtrex's queue and command pool).
class Context {
   public:
    explicit Context(int device = 0, void *stream = nullptr) : stream_(stream) {
        check(mtx_context_create(device, stream, &h_), nullptr, "mtx_context_create");
    }
    ~Context() {
        if (h_) mtx_context_destroy(h_);
    }
    Context(Context &&o) noexcept : h_(std::exchange(o.h_, nullptr)), stream_(o.stream_) {}
    Context &operator=(Context &&o) noexcept {
        if (this != &o) {
            if (h_) mtx_context_destroy(h_);
            h_ = std::exchange(o.h_, nullptr);
            stream_ = o.stream_;
        }
        return *this;
    }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;

    mtx_context_t handle() const { return h_; }
    void *stream() const { return stream_; }
    void setStream(void *stream) {
        check(mtx_context_set_stream(h_, stream), h_, "mtx_context_set_stream");
        stream_ = stream;
    }
    // For destructors: never throws (the call cannot fail for a live context).
    void restoreStream(void *stream) noexcept {
        if (mtx_context_set_stream(h_, stream) == MTX_OK) stream_ = stream;
    }
    // Waits for the stream and reports any error a kernel recorded.
    void synchronize() { check(mtx_synchronize(h_), h_, "mtx_synchronize"); }

   private:
    mtx_context_t h_ = nullptr;
    void *stream_ = nullptr;
};

// meshtrex's `VkCommandBuffer externalCmd` argument: work is recorded into the
// caller's stream for the duration of one call.
class StreamScope {
   public:
    StreamScope(Context &ctx, void *external) : ctx_(ctx), prev_(ctx.stream()), on_(external != nullptr) {
        if (on_) ctx_.setStream(external);
    }
    ~StreamScope() {
        if (on_) ctx_.restoreStream(prev_);
    }

   private:
    Context &ctx_;
    void *prev_;
    bool on_;
};

// GPUProfiler (src/gpuProfiler.h:11-160): CUDA events around the stages, under
// meshtrex's stage names.
class GPUProfiler {
   public:
    explicit GPUProfiler(Context &ctx) { check(mtx_profiler_create(ctx.handle(), &h_), ctx.handle(), "mtx_profiler_create"); }
    ~GPUProfiler() {
        if (h_) mtx_profiler_destroy(h_);
    }
    GPUProfiler(const GPUProfiler &) = delete;
    GPUProfiler &operator=(const GPUProfiler &) = delete;
    mtx_profiler_t handle() const { return h_; }
    void beginFrame() { check(mtx_profiler_begin_frame(h_), nullptr, "mtx_profiler_begin_frame"); }
    void endFrame() { check(mtx_profiler_end_frame(h_), nullptr, "mtx_profiler_end_frame"); }
    // Last frame's time of a stage in ms, or -1 if it did not run.
    double lastMs(const std::string &name) const {
        const uint32_t n = mtx_profiler_region_count(h_);
        for (uint32_t i = 0; i < n; ++i) {
            char nm[64];
            double last, avg;
            uint32_t frames;
            if (mtx_profiler_region(h_, i, nm, &last, &avg, &frames) == MTX_OK && name == nm) return last;
        }
        return -1.0;
    }
    void printResults() const {
        const uint32_t n = mtx_profiler_region_count(h_);
        for (uint32_t i = 0; i < n; ++i) {
            char nm[64];
            double last, avg;
            uint32_t frames;
            if (mtx_profiler_region(h_, i, nm, &last, &avg, &frames) == MTX_OK)
                std::printf("%-28s %10.4f ms (avg %.4f over %u)\n", nm, last, avg, frames);
        }
    }
    void exportCSV(const char *path) const { check(mtx_profiler_export_csv(h_, path), nullptr, "mtx_profiler_export_csv"); }

   private:
    mtx_profiler_t h_ = nullptr;
};

inline mtx_profiler_t profilerHandle(GPUProfiler *p) { return p ? p->handle() : nullptr; }

}  // namespace meshtrex
