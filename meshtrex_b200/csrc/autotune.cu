// Autotuner of the plain path's launch shape.  meshtrex fixes its workgroup
// sizes and block edge at compile time (specialization constants,
// extractionPipeline.cpp:238-256, and the 4^3 cap of pmb.task.glsl:19,27);
// here they are run-time knobs, and mtx_autotune picks them for a volume by
// timing the whole plain extraction of each candidate on the device.
//
// The score of a candidate is the sum of the stage times the profiler's CUDA
// events record (leaf min/max, octree, filter, extraction), the best of a few
// repetitions, so host-side allocation and the count read-back do not count.
// Results are cached per (dims, dtype, device name): in memory for the
// process and, given a path, in a text file with one line per entry
//   X Y Z dtype B zchunk slices warps staging ms device-name
// that later processes read.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "mtx_internal.h"

using namespace mtx;

namespace {

using Key = std::tuple<uint32_t, uint32_t, uint32_t, uint32_t, std::string>;

struct Entry {
    uint32_t B;
    mtx_tuning t;
    double ms;
};

std::mutex g_mu;
std::map<Key, Entry> g_cache;

bool read_file(const char *path, const Key &k, Entry &e) {
    FILE *f = path ? fopen(path, "r") : nullptr;
    if (!f) return false;
    char line[512];
    bool found = false;
    while (fgets(line, sizeof(line), f)) {
        unsigned X, Y, Z, dt, B, zc, sl, w, st;
        double ms;
        char name[256] = {0};
        if (sscanf(line, "%u %u %u %u %u %u %u %u %u %lf %255[^\n]", &X, &Y, &Z, &dt, &B, &zc, &sl, &w, &st, &ms,
                   name) != 11)
            continue;
        if (Key(X, Y, Z, dt, std::string(name)) == k) {  // the last matching line wins
            e = Entry{B, mtx_tuning{zc, sl, w, st}, ms};
            found = true;
        }
    }
    fclose(f);
    return found;
}

void append_file(const char *path, const Key &k, const Entry &e) {
    FILE *f = path ? fopen(path, "a") : nullptr;
    if (!f) return;
    fprintf(f, "%u %u %u %u %u %u %u %u %u %.6f %s\n", std::get<0>(k), std::get<1>(k), std::get<2>(k),
            std::get<3>(k), e.B, e.t.minmaxZChunk, e.t.minmaxSlices, e.t.extractWarps, e.t.staging, e.ms,
            std::get<4>(k).c_str());
    fclose(f);
}

// Device time of one plain extraction with the context's current tuning:
// the sum of the profiler's stage times, best of `reps`.
mtx_status time_plain(mtx_context *c, const mtx_volume *vol, uint32_t B, float iso, uint32_t reps, double &best) {
    mtx_push_constants pc;
    mtx_status rs = mtx_push_constants_init(vol->dims, B, iso, &pc);
    if (rs != MTX_OK) return fail(c, rs, "autotune: push constants");
    mtx_profiler_t prof = nullptr;
    if ((rs = mtx_profiler_create(c, &prof)) != MTX_OK) return rs;
    best = 1e30;
    for (uint32_t r = 0; r < reps && rs == MTX_OK; ++r) {
        mtx_minmax_output mm{};
        mtx_filtering_output f{};
        mtx_extraction_output x{};
        mtx_profiler_begin_frame(prof);
        rs = mtx_compute_min_max_mip(c, vol, &pc, prof, &mm);
        if (rs == MTX_OK) rs = mtx_filter_active_blocks(c, &mm, &pc, prof, &f);
        if (rs == MTX_OK) rs = mtx_read_active_block_count(c, &f);
        if (rs == MTX_OK) rs = mtx_extract_meshlet_descriptors(c, &mm, &f, &pc, nullptr, prof, &x);
        if (rs == MTX_OK) rs = mtx_synchronize(c);
        if (rs == MTX_OK) rs = mtx_profiler_end_frame(prof);
        if (rs == MTX_OK) {
            double sum = 0.0;
            const uint32_t n = mtx_profiler_region_count(prof);
            for (uint32_t i = 0; i < n; ++i) {
                char name[64];
                double last, avg;
                uint32_t frames;
                if (mtx_profiler_region(prof, i, name, &last, &avg, &frames) == MTX_OK) sum += last;
            }
            best = std::min(best, sum);
        }
        mtx_extraction_free(c, &x);
        mtx_filtering_free(c, &f);
        mtx_minmax_free(c, &mm);
    }
    mtx_profiler_destroy(prof);
    return rs;
}

}  // namespace

extern "C" mtx_status mtx_autotune(mtx_context_t c, const mtx_volume *vol, float isovalue, const char *cache_path,
                                   uint32_t flags, mtx_autotune_result *out) {
    if (!c || !vol || !out) return c ? fail(c, MTX_ERR_INVALID_ARG, "null argument") : MTX_ERR_INVALID_ARG;
    DeviceGuard dg(c->device);
    join_extract(c);
    mtx_status rs = check_volume(c, vol);
    if (rs != MTX_OK) return rs;
    memset(out, 0, sizeof(*out));
    cudaDeviceProp prop;
    MTX_CUDA(c, cudaGetDeviceProperties(&prop, c->device));
    const Key key(vol->dims[0], vol->dims[1], vol->dims[2], vol->dtype, std::string(prop.name));
    const bool fresh = flags & MTX_AUTOTUNE_IGNORE_CACHE;
    Entry e{};
    bool hit = false;
    if (!fresh) {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_cache.find(key);
        if (it != g_cache.end()) {
            e = it->second;
            hit = true;
        } else if (read_file(cache_path, key, e)) {
            g_cache[key] = e;
            hit = true;
        }
    }
    if (hit) {
        out->blockEdge = e.B;
        out->tuning = e.t;
        out->ms = e.ms;
        out->fromCache = 1;
        return MTX_OK;
    }

    const mtx_tuning saved = c->tuning;
    const uint32_t reps = (flags & MTX_AUTOTUNE_QUICK) ? 1u : 3u;
    // stage 1: block edge x warps x staging, min/max at its default
    Entry best{0, mtx_tuning{0, 0, 0, 0}, 1e30};
    uint32_t tried = 0;
    for (uint32_t B : {4u, 8u, 16u}) {
        for (uint32_t warps : {2u, 4u, 8u}) {
            for (uint32_t staging : {(uint32_t)MTX_STAGING_TMA, (uint32_t)MTX_STAGING_LDG}) {
                c->tuning = mtx_tuning{0, 0, warps, staging};
                double ms;
                rs = time_plain(c, vol, B, isovalue, reps, ms);
                if (rs != MTX_OK) break;
                ++tried;
                if (ms < best.ms) best = Entry{B, c->tuning, ms};
            }
            if (rs != MTX_OK) break;
        }
        if (rs != MTX_OK) break;
    }
    // stage 2: the load-based min/max pass with 1, 2 or 4 z slices in flight
    // against the default (the TMA ring where the dtype allows it), at the chosen shape
    for (uint32_t slices : {1u, 2u, 4u}) {
        if (rs != MTX_OK) break;
        c->tuning = best.t;
        c->tuning.minmaxSlices = slices;
        double ms;
        rs = time_plain(c, vol, best.B, isovalue, reps, ms);
        if (rs != MTX_OK) break;
        ++tried;
        if (ms < best.ms) best = Entry{best.B, c->tuning, ms};
    }
    c->tuning = saved;
    if (rs != MTX_OK) return rs;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_cache[key] = best;
        append_file(cache_path, key, best);
    }
    out->blockEdge = best.B;
    out->tuning = best.t;
    out->ms = best.ms;
    out->fromCache = 0;
    out->candidates = tried;
    return MTX_OK;
}
