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

// ------------------------------------------------------------- batches
// mtx_autotune_batch: the block edge of every volume of a batch and the
// batched kernel's block warps, by timing the batched run itself (the plain
// path's best edge does not carry over: the batched bodies at edge 4 take
// twice the time of edge 8 on dense blob volumes).  Candidates: one edge for
// every volume (4, 8, 16) at 8 and 6 block warps; then, from the best, each
// dtype's volumes moved to the other edges in turn.  A candidate is run once
// with small capacities to learn the sizes it needs, then created with those,
// run once to warm up and timed (CUDA events on the context's stream), best
// of `reps`.  Cached per (the batch's sorted (dims, dtype) list, device name):
// in memory and, given a path, as lines
//   batch <edges of the volumes in the order of the list> <warps> <ms> <key>
namespace {

struct BatchEntry {
    std::vector<uint32_t> edges;  // per volume, in the order of the sorted key
    uint32_t warps;
    double ms;
};
std::map<std::string, BatchEntry> g_batch_cache;

// The key: "X,Y,Z,dtype;" per volume in sorted order, then the device name;
// order[i] is the volume behind the i-th entry.
std::string batch_key(const mtx_batch_desc *d, const char *device, std::vector<uint32_t> &order) {
    std::vector<std::pair<std::string, uint32_t>> v;
    for (uint32_t i = 0; i < d->volumeCount; ++i) {
        const mtx_volume &m = d->volumes[i];
        v.push_back({std::to_string(m.dims[0]) + "," + std::to_string(m.dims[1]) + "," + std::to_string(m.dims[2]) +
                         "," + std::to_string(m.dtype) + ";",
                     i});
    }
    std::stable_sort(v.begin(), v.end());
    std::string k;
    order.clear();
    for (auto &e : v) {
        k += e.first;
        order.push_back(e.second);
    }
    return k + device;
}

bool read_batch_file(const char *path, const std::string &key, size_t n, BatchEntry &e) {
    FILE *f = path ? fopen(path, "r") : nullptr;
    if (!f) return false;
    std::string line;
    bool found = false;
    char buf[1 << 16];
    while (fgets(buf, sizeof(buf), f)) {
        line = buf;
        if (line.compare(0, 6, "batch ") != 0) continue;
        if (!line.empty() && line.back() == '\n') line.pop_back();
        const char *s = line.c_str() + 6;
        BatchEntry t;
        bool ok = true;
        for (size_t i = 0; i < n && ok; ++i) {
            char *end;
            const unsigned long x = strtoul(s, &end, 10);
            ok = end != s;
            t.edges.push_back((uint32_t)x);
            s = end;
        }
        char *end;
        t.warps = ok ? (uint32_t)strtoul(s, &end, 10) : 0;
        if (ok) {
            s = end;
            t.ms = strtod(s, &end);
            s = end;
            while (*s == ' ') ++s;
            if (key == s) {
                e = t;
                found = true;
            }
        }
    }
    fclose(f);
    return found;
}

void append_batch_file(const char *path, const std::string &key, const BatchEntry &e) {
    FILE *f = path ? fopen(path, "a") : nullptr;
    if (!f) return;
    fprintf(f, "batch");
    for (uint32_t x : e.edges) fprintf(f, " %u", x);
    fprintf(f, " %u %.6f %s\n", e.warps, e.ms, key.c_str());
    fclose(f);
}

// Device time of one batched run of `d` with these block edges and warps.
mtx_status time_batch(mtx_context *c, const mtx_batch_desc *d, const std::vector<uint32_t> &edges, uint32_t warps,
                      uint32_t reps, double &best) {
    mtx_batch_desc t = *d;
    t.blockEdges = edges.data();
    t.blockWarps = warps;
    t.useGraph = 0;
    // sizes: runs with small capacities report what the run needs -- the
    // active blocks first, then (with room for those) the vertices and triangles
    t.maxActiveBlocks = 1u << 16;
    t.vertexCapacity = t.triangleCapacity = 1u << 16;
    mtx_batch_t b = nullptr;
    mtx_status rs = MTX_OK;
    mtx_batch_totals tot{};
    for (int pass = 0; pass < 2 && rs == MTX_OK; ++pass) {
        if ((rs = mtx_batch_create(c, &t, &b)) != MTX_OK) return rs;
        rs = mtx_batch_run(b);
        if (rs == MTX_OK) {
            rs = mtx_batch_read_results(b, nullptr, &tot);
            if (rs == MTX_ERR_CAPACITY) rs = MTX_OK;
        }
        mtx_batch_destroy(b);
        t.maxActiveBlocks = std::max<uint64_t>(tot.activeBlocks, 1);
    }
    if (rs != MTX_OK) return rs;
    t.maxActiveBlocks = std::max<uint64_t>(tot.activeBlocks, 1);
    t.vertexCapacity = std::max<uint64_t>(tot.vertexCount, 1);
    t.triangleCapacity = std::max<uint64_t>(tot.triangleCount, 1);
    if ((rs = mtx_batch_create(c, &t, &b)) != MTX_OK) return rs;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    best = 1e30;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rs = MTX_ERR_CUDA;
    if (rs == MTX_OK) rs = mtx_batch_run(b);  // warm-up
    for (uint32_t r = 0; r < reps && rs == MTX_OK; ++r) {
        cudaEventRecord(e0, c->stream);
        rs = mtx_batch_run(b);
        cudaEventRecord(e1, c->stream);
        if (rs == MTX_OK) rs = mtx_batch_read_results(b, nullptr, nullptr);
        float ms = 0.0f;
        if (rs == MTX_OK && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) best = std::min(best, (double)ms);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    mtx_batch_destroy(b);
    return rs;
}

}  // namespace

extern "C" mtx_status mtx_autotune_batch(mtx_context_t c, const mtx_batch_desc *d, const char *cache_path,
                                         uint32_t flags, uint32_t *blockEdges, mtx_batch_autotune_result *out) {
    if (!c || !d || !blockEdges || !out || !d->volumes || !d->volumeCount || !d->jobs || !d->jobCount)
        return c ? fail(c, MTX_ERR_INVALID_ARG, "null argument") : MTX_ERR_INVALID_ARG;
    DeviceGuard dg(c->device);
    join_extract(c);
    memset(out, 0, sizeof(*out));
    cudaDeviceProp prop;
    MTX_CUDA(c, cudaGetDeviceProperties(&prop, c->device));
    std::vector<uint32_t> order;
    const std::string key = batch_key(d, prop.name, order);
    const uint32_t n = d->volumeCount;
    BatchEntry e;
    bool hit = false;
    if (!(flags & MTX_AUTOTUNE_IGNORE_CACHE)) {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_batch_cache.find(key);
        if (it != g_batch_cache.end()) {
            e = it->second;
            hit = true;
        } else if (read_batch_file(cache_path, key, n, e)) {
            g_batch_cache[key] = e;
            hit = true;
        }
    }
    if (hit) {
        for (uint32_t i = 0; i < n; ++i) blockEdges[order[i]] = e.edges[i];
        out->blockWarps = e.warps;
        out->ms = e.ms;
        out->fromCache = 1;
        return MTX_OK;
    }
    const uint32_t reps = (flags & MTX_AUTOTUNE_QUICK) ? 1u : 3u;
    mtx_status rs = MTX_OK;
    std::vector<uint32_t> best_edges(n, 8), edges(n);
    uint32_t best_warps = 0, tried = 0;
    double best = 1e30;
    auto consider = [&](const std::vector<uint32_t> &ed, uint32_t w) {
        double ms;
        rs = time_batch(c, d, ed, w, reps, ms);
        if (rs != MTX_OK) return;
        ++tried;
        if (ms < best) {
            best = ms;
            best_edges = ed;
            best_warps = w;
        }
    };
    // one edge for every volume, at 8 (as many as fit) and 6 block warps
    for (uint32_t B : {4u, 8u, 16u})
        for (uint32_t w : {0u, 6u}) {
            if (rs != MTX_OK) break;
            std::fill(edges.begin(), edges.end(), B);
            consider(edges, w);
        }
    // then each dtype's volumes at the other edges
    for (uint32_t dt = 0; dt <= MTX_DTYPE_F32 && rs == MTX_OK; ++dt) {
        bool any = false;
        for (uint32_t i = 0; i < n; ++i) any |= d->volumes[i].dtype == dt;
        if (!any) continue;
        const std::vector<uint32_t> base = best_edges;
        for (uint32_t B : {4u, 8u, 16u}) {
            edges = base;
            bool changed = false;
            for (uint32_t i = 0; i < n; ++i)
                if (d->volumes[i].dtype == dt && edges[i] != B) {
                    edges[i] = B;
                    changed = true;
                }
            if (changed) consider(edges, best_warps);
            if (rs != MTX_OK) break;
        }
    }
    if (rs != MTX_OK) return rs;
    e.edges.resize(n);
    for (uint32_t i = 0; i < n; ++i) e.edges[i] = best_edges[order[i]];
    e.warps = best_warps;
    e.ms = best;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_batch_cache[key] = e;
        append_batch_file(cache_path, key, e);
    }
    for (uint32_t i = 0; i < n; ++i) blockEdges[i] = best_edges[i];
    out->blockWarps = best_warps;
    out->ms = best;
    out->candidates = tried;
    return MTX_OK;
}
