// Batched extraction: every (volume, isovalue) job of a batch in two
// launches.  The leaf min/max of all volumes runs as one kernel (a volume's
// min/max serves all of its isovalues); one persistent kernel then takes all
// jobs through filtering with ordered compaction, per-block counts, the
// offset scan and emission.  meshtrex extracts one volume at one isovalue per
// call (src/meshtrex.cpp:107-141); each job here gives exactly what that
// sequence gives for its volume, block edge and isovalue.
//
// The persistent kernel hands out work by ticket and a CTA only ever waits
// for work that was handed out before its own (to CTAs that are running), so
// it needs neither a co-residency guarantee nor a grid barrier:
//
//  filter   1024-block tiles of every job in job order, under one decoupled
//           look-back: pooled rank = (job, block id) order.  Each job's rank
//           map holds pooled ranks.
//  count    one active block per warp item, as in the single-volume count pass
//  scan     1024-descriptor tiles under a segmented look-back: a job's
//           offsets restart at its first block
//  bases    one CTA: each job's first vertex and index in the pooled buffers,
//           capacity checks
//  emit     one active block per warp item; indices count from the job's
//           first vertex
//
// Data written by an earlier phase of the same launch is read with L2-only
// loads (never the read-only cache), after a fenced hand-over counter.
#include <algorithm>
#include <vector>

#include "minmax_device.cuh"
#include "pmb_balanced.cuh"

namespace mtx {

constexpr uint32_t kBThreads = 256;
constexpr uint32_t kBItems = 4;
constexpr uint32_t kBTile = kBThreads * kBItems;
constexpr uint32_t kBWarps = kBThreads / 32;
constexpr uint32_t kBChunk = 2;                 // active blocks per warp ticket
constexpr uint32_t kPhaseSpinLimit = 1u << 26;  // about 17 s of polling at the longest back-off

struct BVol {
    Problem p;      // isovalue unset
    WPlan pl;       // region sizes of this volume, offsets of the batch's shared warp layout
    GridDiv dv;     // reciprocals of the grid's row and slice sizes (block_geo)
    uint32_t vec;   // min/max by 16-byte vector warps (1) or one thread per block (0)
    uint32_t nXS, zchunk, pad;
    uint64_t leaf_off;  // first leaf entry of the volume in the pooled leaf array
    uint64_t mm_begin;  // first min/max warp of the volume
};

struct BJob {
    uint32_t vol;
    float iso;
    uint32_t tile_begin, ntiles;  // filter tiles of the job
    uint64_t rank_off;            // first word of the job's rank map
};

// Zeroed before every run.
struct BCtrl {
    uint32_t filter_ticket, filter_done, total_active, count_ticket;
    uint32_t count_done, scan_ticket, scan_done, bases_ticket;
    uint32_t bases_ready, emit_ok, emit_ticket, pad;
    uint64_t total_vertices, total_triangles;
    DevStatus status;
};

struct BatchArgs {
    const BVol *vols;
    const BJob *jobs;
    const uint32_t *tile_job;
    const uint2 *leaf;
    uint32_t njobs, n_ftiles;
    uint32_t ws_bytes, face_stride;
    uint32_t block_warps, pad0;  // warps of a CTA that take count/emit work (the layout fits that many)
    uint32_t *rank_pool;
    uint32_t *ids, *job_of;
    uint64_t block_cap;
    mtx_meshlet_descriptor *desc;
    uint32_t *faces;
    uint32_t *filter_status;
    uint64_t *scan_status;
    mtx_batch_job_result *res;
    uint32_t *job_end;
    void *vertices;
    uint64_t vcap;
    uint32_t *indices;
    uint64_t tcap;
    uint32_t vfmt, frame, normals, vsz;
    BCtrl *ctrl;
};

// ------------------------------------------------------------ min/max
// Every volume's leaf min/max in one launch; warp w belongs to the last
// volume whose mm_begin <= w.
template <int ZU>
__global__ void __launch_bounds__(128) batch_minmax_kernel(const BVol *__restrict__ vols, uint32_t nvol,
                                                           uint64_t nwarps, uint2 *__restrict__ leaf) {
    const uint64_t w = (uint64_t)blockIdx.x * 4 + (threadIdx.x >> 5);
    if (w >= nwarps) return;  // uniform per warp
    uint32_t lo = 0, hi = nvol - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (vols[mid].mm_begin <= w) lo = mid;
        else hi = mid - 1;
    }
    const BVol &v = vols[lo];
    const Problem &p = v.p;
    const uint64_t lw = w - v.mm_begin;
    uint2 *out = leaf + v.leaf_off;
    if (!v.vec) {
        const uint64_t b = lw * 32 + (threadIdx.x & 31);
        if (b >= p.nblocks) return;
        switch (p.dtype) {
        case MTX_DTYPE_U8: minmax_leaf_one<uint8_t>((const uint8_t *)p.vol, p.X, p.Y, p.Z, p.B, p.GX, p.GY, b, out); break;
        case MTX_DTYPE_U16: minmax_leaf_one<uint16_t>((const uint16_t *)p.vol, p.X, p.Y, p.Z, p.B, p.GX, p.GY, b, out); break;
        default: minmax_leaf_one<float>((const float *)p.vol, p.X, p.Y, p.Z, p.B, p.GX, p.GY, b, out); break;
        }
        return;
    }
#define MTX_MM(T, BE) \
    minmax_leaf_vec_warp<T, BE, ZU>((const T *)p.vol, p.X, p.Y, p.Z, p.GX, p.GY, p.GZ, v.nXS, v.zchunk, lw, out)
    switch (p.dtype * 32 + p.B) {
    case MTX_DTYPE_U8 * 32 + 4: MTX_MM(uint8_t, 4); break;
    case MTX_DTYPE_U8 * 32 + 8: MTX_MM(uint8_t, 8); break;
    case MTX_DTYPE_U8 * 32 + 16: MTX_MM(uint8_t, 16); break;
    case MTX_DTYPE_U16 * 32 + 4: MTX_MM(uint16_t, 4); break;
    case MTX_DTYPE_U16 * 32 + 8: MTX_MM(uint16_t, 8); break;
    case MTX_DTYPE_U16 * 32 + 16: MTX_MM(uint16_t, 16); break;
    case MTX_DTYPE_F32 * 32 + 4: MTX_MM(float, 4); break;
    case MTX_DTYPE_F32 * 32 + 8: MTX_MM(float, 8); break;
    default: MTX_MM(float, 16); break;
    }
#undef MTX_MM
}

// ------------------------------------------------------------ hand-over
// CTA-wide bounded wait until *word >= target.  Thread 0 polls, then fences
// so that what the producers wrote before their counter update is visible.
__device__ __forceinline__ bool cta_wait_geq(const uint32_t *word, uint32_t target, DevStatus *st, uint32_t phase,
                                             uint32_t *s_flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t ok = 1, spins = 0;
        while (ld_volatile(word) < target) {
            if (++spins >= kPhaseSpinLimit) {
                report(st, MTX_ERR_TIMEOUT, kSiteBatched, phase, target);
                ok = 0;
                break;
            }
            backoff(spins);
        }
        __threadfence();
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0;
}

// Every thread fences its writes, then one thread bumps the counter.
__device__ __forceinline__ void cta_signal(uint32_t *word, uint32_t v) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(word, v);
}

__device__ __forceinline__ uint32_t warp_ticket(uint32_t *word, uint32_t n) {
    uint32_t t = 0;
    if ((threadIdx.x & 31) == 0) t = atomicAdd(word, n);
    return __shfl_sync(0xffffffffu, t, 0);
}

// ------------------------------------------------------------ filter
// Tile words: [31:30] flag (1 aggregate, 2 inclusive, 3 aborted), [29:0] count.
__device__ __forceinline__ bool lookback_sum30(const uint32_t *status, uint32_t t, uint32_t &prefix,
                                               DevStatus *st) {
    const uint32_t lane = threadIdx.x & 31;
    prefix = 0;
    int64_t j = (int64_t)t - 1;
    uint32_t spins = 0;
    while (true) {
        const int64_t k = j - (int64_t)lane;
        const uint32_t w = k >= 0 ? ld_volatile(&status[k]) : (2u << 30);
        const uint32_t flag = w >> 30;
        if (__any_sync(0xffffffffu, flag == 3u)) return false;
        const uint32_t inc = __ballot_sync(0xffffffffu, flag == 2u);
        const uint32_t emp = __ballot_sync(0xffffffffu, flag == 0u);
        const uint32_t first = inc ? (uint32_t)(__ffs(inc) - 1) : 32u;
        const uint32_t window = first >= 31 ? 0xffffffffu : ((2u << first) - 1u);
        if (emp & window) {
            if (++spins >= kSpinLimit) {
                if (lane == 0) report(st, MTX_ERR_TIMEOUT, kSiteFilterLookback, t, (uint32_t)j);
                return false;
            }
            backoff(spins);
            continue;
        }
        uint32_t v = lane <= first ? (w & 0x3fffffffu) : 0u;
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        prefix += v;
        if (first < 32) return true;
        j -= 32;
    }
}

__device__ __forceinline__ void batch_filter_tile(const BatchArgs &a, uint32_t t, uint32_t *s_tmp, uint32_t *s_u) {
    const uint32_t tid = threadIdx.x;
    const uint32_t j = a.tile_job[t];
    const BJob job = a.jobs[j];
    const BVol &v = a.vols[job.vol];
    const uint64_t nb = v.p.nblocks;
    const uint32_t dtype = v.p.dtype;
    const uint64_t base = (uint64_t)(t - job.tile_begin) * kBTile + (uint64_t)tid * kBItems;
    const uint2 *leaf = a.leaf + v.leaf_off;
    uint32_t f[kBItems];
    if (base + kBItems <= nb) {
        const uint4 *q = reinterpret_cast<const uint4 *>(leaf + base);
        const uint4 x = __ldcg(q), y = __ldcg(q + 1);
        f[0] = block_active(dtype, x.x, x.y, job.iso);
        f[1] = block_active(dtype, x.z, x.w, job.iso);
        f[2] = block_active(dtype, y.x, y.y, job.iso);
        f[3] = block_active(dtype, y.z, y.w, job.iso);
    } else {
#pragma unroll
        for (uint32_t i = 0; i < kBItems; ++i) {
            f[i] = 0;
            if (base + i < nb) {
                const uint2 w = leaf[base + i];
                f[i] = block_active(dtype, w.x, w.y, job.iso);
            }
        }
    }
    uint32_t total;
    const uint32_t excl = cta_exclusive_scan<kBThreads>(f[0] + f[1] + f[2] + f[3], s_tmp, &total);
    if (tid < 32) {
        uint32_t prefix = 0;
        bool ok = true;
        if (t == 0) {
            if (tid == 0) st_volatile(&a.filter_status[0], (2u << 30) | total);
        } else {
            if (tid == 0) st_volatile(&a.filter_status[t], (1u << 30) | total);
            ok = lookback_sum30(a.filter_status, t, prefix, &a.ctrl->status);
            if (ok && prefix + total >= (1u << 30)) {
                if (tid == 0) report(&a.ctrl->status, MTX_ERR_CAPACITY, kSiteBatched, 1, prefix);
                ok = false;
            }
            if (tid == 0) st_volatile(&a.filter_status[t], ok ? ((2u << 30) | (prefix + total)) : (3u << 30));
        }
        if (tid == 0) {
            s_u[0] = prefix;
            s_u[1] = ok;
        }
    }
    __syncthreads();
    if (!s_u[1]) return;
    const uint32_t prefix = s_u[0];
    uint32_t r = prefix + excl;
    uint32_t rk[kBItems];
#pragma unroll
    for (uint32_t i = 0; i < kBItems; ++i) {
        rk[i] = kNoVertex;
        if (f[i]) {
            if (r < a.block_cap) {
                a.ids[r] = (uint32_t)(base + i);
                a.job_of[r] = j;
            }
            rk[i] = r++;
        }
    }
    uint32_t *rank_map = a.rank_pool + job.rank_off;
    if (base + kBItems <= nb) {
        *reinterpret_cast<uint4 *>(rank_map + base) = make_uint4(rk[0], rk[1], rk[2], rk[3]);
    } else {
#pragma unroll
        for (uint32_t i = 0; i < kBItems; ++i)
            if (base + i < nb) rank_map[base + i] = rk[i];
    }
    if (tid == 0) {
        if (t == job.tile_begin) a.res[j].meshletOffset = prefix;
        if (t == job.tile_begin + job.ntiles - 1) a.job_end[j] = prefix + total;
        if (t == a.n_ftiles - 1) a.ctrl->total_active = prefix + total;
    }
}

// ------------------------------------------------------------ segmented scan
// Tile words as in the single-volume scan ([63:62] flag, [61:31] triangles,
// [30:0] vertices).  A tile holding a job's first block publishes its
// inclusive word (the sum after its last job start) at once; it looks back
// only if its first block continues the job of the tile before.
__device__ __forceinline__ bool lookback_seg(uint64_t *status, uint32_t t, bool has_head, uint64_t tail,
                                             bool need_carry, uint64_t &cv, uint64_t &ct, DevStatus *st) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t tv = (uint32_t)tail, tt = tail >> 32;
    cv = ct = 0;
    bool ok = true;
    if (has_head) {
        ok = tv <= kCnt31 && tt <= kCnt31 && 3ull * tt <= 0xffffffffull;
        if (lane == 0) st_volatile(&status[t], ok ? ((2ull << 62) | (tt << 31) | tv) : (3ull << 62));
        if (!ok && lane == 0) report(st, MTX_ERR_CAPACITY, kSiteCountOverflow, (uint32_t)tv, (uint32_t)tt);
    } else if (lane == 0) {
        st_volatile(&status[t], (1ull << 62) | (tt << 31) | tv);
    }
    if (need_carry && ok) ok = lookback_sum31(status, t, cv, ct, st);
    if (!has_head) {
        const uint64_t iv = cv + tv, it = ct + tt;
        if (ok && (iv > kCnt31 || it > kCnt31 || 3ull * it > 0xffffffffull)) {
            if (lane == 0) report(st, MTX_ERR_CAPACITY, kSiteCountOverflow, (uint32_t)(iv >> 32), (uint32_t)it);
            ok = false;
        }
        if (lane == 0) st_volatile(&status[t], ok ? ((2ull << 62) | (it << 31) | iv) : (3ull << 62));
    }
    return ok;
}

// x (later) absorbs y (earlier) unless x already holds a job start.
__device__ __forceinline__ void seg_add(uint64_t &x, uint32_t &fx, uint64_t y, uint32_t fy) {
    if (!fx) x += y;
    fx |= fy;
}

__device__ __forceinline__ void batch_scan_tile(const BatchArgs &a, uint32_t t, uint32_t n, uint64_t *s_v,
                                                uint32_t *s_f, uint64_t *s_carry, uint32_t *s_u) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t base = t * kBTile + tid * kBItems;
    uint64_t val[kBItems];
    uint32_t jb[kBItems], head = 0;
    uint32_t prev = base > 0 && base - 1 < n ? __ldcg(a.job_of + base - 1) : kNoVertex;
#pragma unroll
    for (uint32_t i = 0; i < kBItems; ++i) {
        const uint32_t r = base + i;
        val[i] = 0;
        jb[i] = kNoVertex;
        if (r < n) {
            const uint2 c = __ldcg(reinterpret_cast<const uint2 *>(&a.desc[r].vertexCount));
            val[i] = ((uint64_t)c.y << 32) | c.x;
            jb[i] = __ldcg(a.job_of + r);
            if (r == 0 || jb[i] != prev) head |= 1u << i;
            prev = jb[i];
        }
    }
    // thread aggregate: the sum after the thread's last job start
    uint64_t x = 0;
#pragma unroll
    for (uint32_t i = 0; i < kBItems; ++i) x = ((head >> i) & 1u) ? val[i] : x + val[i];
    uint32_t fx = head != 0;
    // inclusive segmented scan of the warp, then of the warps
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        const uint32_t fy = __shfl_up_sync(0xffffffffu, fx, o);
        if (lane >= (uint32_t)o) seg_add(x, fx, y, fy);
    }
    if (lane == 31) {
        s_v[warp] = x;
        s_f[warp] = fx;
    }
    __syncthreads();
    if (warp == 0) {
        uint64_t w = lane < kBWarps ? s_v[lane] : 0ull;
        uint32_t fw = lane < kBWarps ? s_f[lane] : 0u;
#pragma unroll
        for (int o = 1; o < (int)kBWarps; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
            const uint32_t fy = __shfl_up_sync(0xffffffffu, fw, o);
            if (lane >= (uint32_t)o) seg_add(w, fw, y, fy);
        }
        if (lane < kBWarps) {
            s_v[lane] = w;
            s_f[lane] = fw;
        }
    }
    __syncthreads();
    // exclusive value of the thread within the tile
    uint64_t ex = __shfl_up_sync(0xffffffffu, x, 1);
    uint32_t fex = __shfl_up_sync(0xffffffffu, fx, 1);
    if (lane == 0) {
        ex = 0;
        fex = 0;
    }
    if (warp > 0) seg_add(ex, fex, s_v[warp - 1], s_f[warp - 1]);  // (warps before) then (lanes before)
    if (warp == 0) {
        const uint64_t tail = s_v[kBWarps - 1];
        const bool has_head = s_f[kBWarps - 1] != 0;
        const bool need_carry = __shfl_sync(0xffffffffu, head & 1u, 0) == 0u;
        uint64_t cv, ct;
        const bool ok = lookback_seg(a.scan_status, t, has_head, tail, need_carry, cv, ct, &a.ctrl->status);
        if (lane == 0) {
            s_carry[0] = (ct << 32) | cv;
            s_u[0] = ok;
        }
    }
    __syncthreads();
    if (!s_u[0]) return;
    uint64_t cur = fex ? ex : ex + s_carry[0];
#pragma unroll
    for (uint32_t i = 0; i < kBItems; ++i) {
        const uint32_t r = base + i;
        if (r >= n) break;
        if ((head >> i) & 1u) cur = 0;
        *reinterpret_cast<uint2 *>(&a.desc[r].vertexOffset) =
            make_uint2((uint32_t)cur, 3u * (uint32_t)(cur >> 32));
        cur += val[i];
        const uint32_t next = i + 1 < kBItems ? jb[i + 1] : (r + 1 < n ? __ldcg(a.job_of + r + 1) : kNoVertex);
        if (r + 1 == n || next != jb[i]) {  // the job's last block: its totals
            a.res[jb[i]].vertexCount = (uint32_t)cur;
            a.res[jb[i]].indexCount = 3u * (uint32_t)(cur >> 32);
        }
    }
}

// ------------------------------------------------------------ bases
__device__ __forceinline__ void batch_bases(const BatchArgs &a, uint32_t n, uint32_t total_active,
                                            uint64_t *s_tmp) {
    const uint32_t tid = threadIdx.x;
    uint64_t vb = 0, ib = 0;
    for (uint32_t j0 = 0; j0 < a.njobs; j0 += kBThreads) {
        const uint32_t j = j0 + tid;
        uint32_t vc = 0, ic = 0;
        if (j < a.njobs) {
            vc = __ldcg(&a.res[j].vertexCount);
            ic = __ldcg(&a.res[j].indexCount);
        }
        uint64_t tv, ti;
        const uint64_t ev = cta_exclusive_scan64<kBThreads>(vc, s_tmp, &tv);
        const uint64_t ei = cta_exclusive_scan64<kBThreads>(ic, s_tmp, &ti);
        if (j < a.njobs) {
            a.res[j].vertexOffset = vb + ev;
            a.res[j].indexOffset = ib + ei;
            a.res[j].meshletCount = __ldcg(a.job_end + j) - __ldcg(&a.res[j].meshletOffset);
        }
        vb += tv;
        ib += ti;
    }
    if (tid == 0) {
        BCtrl *c = a.ctrl;
        c->total_vertices = vb;
        c->total_triangles = ib / 3;
        const bool fits = n == total_active && vb <= a.vcap && ib / 3 <= a.tcap;
        if (!fits) report(&c->status, MTX_ERR_CAPACITY, kSiteBatched, 5, total_active);
        c->emit_ok = fits && !failed(&c->status);
        __threadfence();
        st_volatile(&c->bases_ready, 1u);
    }
}

// ------------------------------------------------------------ per block
// The tile of every block is staged as float whatever the volume's dtype
// (exact for uint8 and uint16: the same compares and interpolation bits as
// the single-volume kernels), so one copy of each block body serves all
// dtypes and the kernel's instruction footprint stays small.  The bodies are
// the balanced ones (pmb_balanced.cuh): batches of many volumes and
// isovalues tend to have dense blocks.
__device__ __forceinline__ void batch_count_block(const BatchArgs &a, const Problem &p, const WPlan &pl,
                                                  const GridDiv &dv, unsigned char *ws, const uint8_t *ntab,
                                                  uint32_t id, uint32_t r) {
    const Geo g = block_geo(id, p, false, 4, dv);
    tile_load_rows(p, pl, ws, g);
    count_block_balanced(p, pl, ws, g, ntab, a.desc + r, a.faces + (uint64_t)r * a.face_stride);
}

template <int CPL, bool GENERIC, bool EO>
__device__ __forceinline__ void batch_emit_block(const BatchArgs &a, const Problem &p, const WPlan &pl,
                                                 const GridDiv &dv, unsigned char *ws, const uint64_t *tab,
                                                 const uint8_t *ntab, const uint8_t *owner, uint32_t id, uint32_t r,
                                                 uint64_t rank_off, const mtx_batch_job_result &jr) {
    const Geo g = block_geo(id, p, false, 4, dv);
    const uint4 q = __ldcg(reinterpret_cast<const uint4 *>(a.desc + r));
    const mtx_meshlet_descriptor d{q.x, q.y, q.z, q.w};
    const uint32_t nb_rk = neighbour_rank<false>(p, g, id, a.rank_pool + rank_off);
    const uint32_t nb_vb = nb_rk != kNoVertex ? __ldcg(&a.desc[nb_rk].vertexOffset) : kNoVertex;
    tile_load_rows(p, pl, ws, g);
    void *verts = a.vertices ? (void *)((char *)a.vertices + jr.vertexOffset * a.vsz) : nullptr;
    if (!emit_vertices_balanced<GENERIC>(p, pl, ws, g, d, ntab, jr.indexCount / 3u, verts, jr.vertexCount, a.vfmt,
                                         a.frame, a.normals, &a.ctrl->status, r))
        return;
    // the tile is dead: the vertex table takes its place, its context layer
    // gathered from the neighbours' face records
    uint32_t rec[CPL];
    gather_issue<CPL, false>(p, pl, g, nb_rk, a.faces, a.face_stride, rec);
    fill_context_vertices<CPL>(pl, ws, nb_vb, rec);
    emit_triangles_balanced<EO>(p, pl, ws, g, d, tab, ntab, owner, a.indices + jr.indexOffset, &a.ctrl->status, r);
}

// ------------------------------------------------------------ the kernel
// BC: every volume's block edge at compile time (0: each volume's own, at run
// time).  When all volumes of a batch have edge 8 the plan and every division
// by the edge fold to constants, and the kernel's code gets smaller.  Its
// register use is held to four CTAs per SM (62 registers, no spills), the
// occupancy of the run-time-edge variants.
template <int CPL, bool GENERIC, int BC>
__global__ void __launch_bounds__(kBThreads, BC ? 4 : 1) batch_extract_kernel(const __grid_constant__ BatchArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint32_t s_u[4];
    __shared__ uint32_t s_tmp[kBWarps + 1];
    __shared__ uint64_t s_tmp64[kBWarps + 1];
    __shared__ uint32_t s_f[kBWarps];
    __shared__ uint64_t s_carry[1];
    uint64_t *tab = reinterpret_cast<uint64_t *>(smem);
    uint8_t *ntab = smem + 2048;
    uint8_t *owner = smem + 2048 + 256;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned char *ws = smem + kTableBytes + min(warp, a.block_warps - 1) * a.ws_bytes;
    for (uint32_t i = tid; i < 256; i += kBThreads) {
        tab[i] = c_mc_cases[i];
        ntab[i] = (uint8_t)(c_mc_cases[i] & 0xFu);
    }
    if (tid < 12) owner[tid] = c_mc_owner[tid];
    if (BC) edge_offsets(reinterpret_cast<uint16_t *>(owner + 16), BC + 1);  // the edge is known: table_vertex<true>
    __syncthreads();
    BCtrl *ctrl = a.ctrl;
    DevStatus *st = &ctrl->status;

    // filter + ordered compaction
    for (;;) {
        if (tid == 0) s_u[2] = atomicAdd(&ctrl->filter_ticket, 1u);
        __syncthreads();
        const uint32_t t = s_u[2];
        __syncthreads();
        if (t >= a.n_ftiles) break;
        batch_filter_tile(a, t, s_tmp, s_u);
        cta_signal(&ctrl->filter_done, 1u);
    }
    if (!cta_wait_geq(&ctrl->filter_done, a.n_ftiles, st, 1, &s_u[3])) return;
    const uint32_t total_active = __ldcg(&ctrl->total_active);
    const uint32_t n = total_active <= a.block_cap ? total_active : 0u;

    // per-block counts
    uint32_t done = 0;
    for (;;) {
        if (warp >= a.block_warps) break;
        const uint32_t c0 = warp_ticket(&ctrl->count_ticket, kBChunk);
        if (c0 >= n) break;
        const uint32_t c1 = min(c0 + kBChunk, n);
        for (uint32_t r = c0; r < c1; ++r) {
            const uint32_t j = __ldcg(a.job_of + r), id = __ldcg(a.ids + r);
            const BJob &job = a.jobs[j];
            const BVol &v = a.vols[job.vol];
            Problem p = v.p;
            p.iso = job.iso;
            if (BC) p.B = BC;
            const WPlan pl = BC ? make_wplan_balanced(BC) : v.pl;
            batch_count_block(a, p, pl, v.dv, ws, ntab, id, r);
            ++done;
        }
    }
    __threadfence();
    __syncwarp();
    if (lane == 0 && done) atomicAdd(&ctrl->count_done, done);
    if (!cta_wait_geq(&ctrl->count_done, n, st, 2, &s_u[3])) return;

    // segmented offset scan
    const uint32_t nst = (n + kBTile - 1) / kBTile;
    for (;;) {
        if (tid == 0) s_u[2] = atomicAdd(&ctrl->scan_ticket, 1u);
        __syncthreads();
        const uint32_t t = s_u[2];
        __syncthreads();
        if (t >= nst) break;
        batch_scan_tile(a, t, n, s_tmp64, s_f, s_carry, s_u);
        cta_signal(&ctrl->scan_done, 1u);
    }

    // job bases: the CTA with the first ticket
    if (tid == 0) s_u[2] = atomicAdd(&ctrl->bases_ticket, 1u);
    __syncthreads();
    if (s_u[2] == 0) {
        if (cta_wait_geq(&ctrl->scan_done, nst, st, 3, &s_u[3])) batch_bases(a, n, total_active, s_tmp64);
    }
    if (!cta_wait_geq(&ctrl->bases_ready, 1u, st, 4, &s_u[3])) return;
    if (!__ldcg(&ctrl->emit_ok)) return;

    // vertices and triangles
    for (;;) {
        if (warp >= a.block_warps) break;
        const uint32_t c0 = warp_ticket(&ctrl->emit_ticket, kBChunk);
        if (c0 >= n) break;
        const uint32_t c1 = min(c0 + kBChunk, n);
        for (uint32_t r = c0; r < c1; ++r) {
            const uint32_t j = __ldcg(a.job_of + r), id = __ldcg(a.ids + r);
            const BJob &job = a.jobs[j];
            const BVol &v = a.vols[job.vol];
            Problem p = v.p;
            p.iso = job.iso;
            if (BC) p.B = BC;
            const WPlan pl = BC ? make_wplan_balanced(BC) : v.pl;
            mtx_batch_job_result jr;
            jr.vertexOffset = __ldcg(&a.res[j].vertexOffset);
            jr.indexOffset = __ldcg(&a.res[j].indexOffset);
            jr.vertexCount = __ldcg(&a.res[j].vertexCount);
            jr.indexCount = __ldcg(&a.res[j].indexCount);
            batch_emit_block<CPL, GENERIC, BC != 0>(a, p, pl, v.dv, ws, tab, ntab, owner, id, r, job.rank_off, jr);
        }
    }
}

MTX_BC_READER(bc_take_batched)

}  // namespace mtx

// ------------------------------------------------------------------ host
using namespace mtx;

struct mtx_batch {
    mtx_context *ctx = nullptr;
    uint32_t nvol = 0, njobs = 0, n_ftiles = 0;
    uint64_t mm_warps = 0;
    uint32_t grid = 0, smem = 0, vsz = 12;
    uint64_t block_cap = 0, vcap = 0, tcap = 0;
    int variant = 0;  // CPL 8/32 x GENERIC (0-3), edge 8 at compile time x GENERIC (4-5)
    std::vector<void *> allocs;
    BVol *vols = nullptr;
    uint2 *leaf = nullptr;
    void *ctrl_region = nullptr;
    size_t ctrl_bytes = 0;
    BatchArgs args{};
    bool use_graph = false;
    cudaStream_t capture_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

using KernelFn = void (*)(BatchArgs);
KernelFn batch_kernel(int variant) {
    switch (variant) {
    case 0: return batch_extract_kernel<8, false, 0>;
    case 1: return batch_extract_kernel<8, true, 0>;
    case 2: return batch_extract_kernel<32, false, 0>;
    case 3: return batch_extract_kernel<32, true, 0>;
    case 4: return batch_extract_kernel<8, false, 8>;
    default: return batch_extract_kernel<8, true, 8>;
    }
}

WPlan plan_in_layout(uint32_t B, const WPlan &L) {
    WPlan p = make_wplan_balanced(B);
    p.off_tile[0] = p.off_tile[1] = L.off_tile[0];
    p.off_vtab = L.off_vtab;
    p.off_bar = L.off_bar;
    p.off_rows = L.off_rows;
    p.off_cross = L.off_cross;
    p.off_vp = L.off_vp;
    p.off_list = L.off_list;
    p.off_vmsk = L.off_vmsk;
    p.off_jobs = L.off_jobs;
    p.bytes = L.bytes;
    return p;
}

uint64_t align4(uint64_t x) { return (x + 3) & ~3ull; }
size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

mtx_status batch_alloc(mtx_batch *b, void **p, size_t bytes) {
    mtx_status s = dev_alloc(b->ctx, p, std::max<size_t>(bytes, 16));
    if (s == MTX_OK) b->allocs.push_back(*p);
    return s;
}

void batch_release(mtx_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    for (void *p : b->allocs) dev_free(b->ctx, p);
    delete b;
}

mtx_status batch_enqueue(mtx_batch *b, cudaStream_t s) {
    mtx_context *c = b->ctx;
    MTX_CUDA(c, cudaMemsetAsync(b->ctrl_region, 0, b->ctrl_bytes, s));
    if (b->mm_warps) {
        const uint64_t blocks = (b->mm_warps + 3) / 4;
        batch_minmax_kernel<2><<<(unsigned)blocks, 128, 0, s>>>(b->vols, b->nvol, b->mm_warps, b->leaf);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(c, e, "batch min/max launch");
    }
    batch_kernel(b->variant)<<<b->grid, kBThreads, b->smem, s>>>(b->args);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "batch extract launch");
    return MTX_OK;
}

}  // namespace

extern "C" {

mtx_status mtx_batch_create(mtx_context_t c, const mtx_batch_desc *d, mtx_batch_t *out) {
    if (!c || !d || !out) return MTX_ERR_INVALID_ARG;
    *out = nullptr;
    DeviceGuard dg(c->device);
    join_extract(c);
    if (d->volumeCount == 0 || d->jobCount == 0 || !d->volumes || !d->blockEdges || !d->jobs)
        return fail(c, MTX_ERR_INVALID_ARG, "batch: empty volume or job list");
    if (d->vertexFormat > MTX_VERTEX_DATA || d->frame > MTX_FRAME_NDC)
        return fail(c, MTX_ERR_INVALID_ARG, "batch: bad vertex format or frame");
    mtx_status rs = load_case_tables(c);
    if (rs != MTX_OK) return rs;

    mtx_batch *b = new mtx_batch();
    b->ctx = c;
    b->nvol = d->volumeCount;
    b->njobs = d->jobCount;
    b->vsz = d->vertexFormat == MTX_VERTEX_DATA ? 32u : 12u;

    // volume table, warp layout, min/max warps
    uint32_t Bmax = 2;
    for (uint32_t v = 0; v < b->nvol; ++v) {
        rs = check_volume(c, &d->volumes[v]);
        if (rs != MTX_OK) { batch_release(b); return rs; }
        const uint32_t B = d->blockEdges[v];
        if (B < 2 || B > 16) { batch_release(b); return fail(c, MTX_ERR_INVALID_ARG, "batch: block edge outside 2..16"); }
        Bmax = std::max(Bmax, B);
    }
    const WPlan L = make_wplan_balanced(Bmax);  // float tile, vertex table in its place
    std::vector<BVol> vols(b->nvol);
    uint64_t leaf_total = 0, want = (uint64_t)c->sm_count * 48;
    for (uint32_t v = 0; v < b->nvol; ++v) {
        const mtx_volume &mv = d->volumes[v];
        const uint32_t B = d->blockEdges[v], esz = dtype_size(mv.dtype);
        BVol &bv = vols[v];
        memset(&bv, 0, sizeof(bv));
        Problem &p = bv.p;
        p.vol = mv.data.ptr;
        p.X = mv.dims[0];
        p.Y = mv.dims[1];
        p.Z = mv.dims[2];
        p.dtype = mv.dtype;
        p.B = B;
        p.GX = ceil_div(p.X, B);
        p.GY = ceil_div(p.Y, B);
        p.GZ = ceil_div(p.Z, B);
        p.nblocks = (uint64_t)p.GX * p.GY * p.GZ;
        bv.pl = plan_in_layout(B, L);
        bv.dv = grid_div(p);
        bv.vec = ((uintptr_t)p.vol % 16 == 0) && (((uint64_t)p.X * esz) % 16 == 0) && (B == 4 || B == 8 || B == 16);
        bv.leaf_off = leaf_total;
        leaf_total += align4(p.nblocks);
        bv.mm_begin = b->mm_warps;
        if (bv.vec) {
            bv.nXS = ceil_div(p.X, 32 * (16 / esz));
            const uint64_t cols = (uint64_t)bv.nXS * p.GY;
            const uint64_t share = std::max<uint64_t>(1, want / b->nvol);
            const uint32_t nzc = (uint32_t)std::min<uint64_t>(p.GZ, std::max<uint64_t>(1, (share + cols - 1) / cols));
            bv.zchunk = ceil_div(p.GZ, nzc);
            b->mm_warps += cols * ceil_div(p.GZ, bv.zchunk);
        } else {
            b->mm_warps += (p.nblocks + 31) / 32;
        }
    }

    // job table and filter tiles
    std::vector<BJob> jobs(b->njobs);
    std::vector<uint32_t> tile_job;
    uint64_t rank_total = 0, blocks_total = 0;
    for (uint32_t j = 0; j < b->njobs; ++j) {
        const mtx_batch_job &bj = d->jobs[j];
        if (bj.volume >= b->nvol) { batch_release(b); return fail(c, MTX_ERR_INVALID_ARG, "batch: job names no volume"); }
        const uint64_t nb = vols[bj.volume].p.nblocks;
        jobs[j].vol = bj.volume;
        jobs[j].iso = bj.isovalue;
        jobs[j].tile_begin = (uint32_t)tile_job.size();
        jobs[j].ntiles = (uint32_t)((nb + kBTile - 1) / kBTile);
        jobs[j].rank_off = rank_total;
        rank_total += align4(nb);
        blocks_total += nb;
        tile_job.insert(tile_job.end(), jobs[j].ntiles, j);
    }
    if (blocks_total >= (1ull << 30)) { batch_release(b); return fail(c, MTX_ERR_UNSUPPORTED, "batch: 2^30 blocks or more"); }
    b->n_ftiles = (uint32_t)tile_job.size();
    b->block_cap = d->maxActiveBlocks ? std::min<uint64_t>(d->maxActiveBlocks, blocks_total) : blocks_total;
    b->vcap = d->vertexCapacity ? d->vertexCapacity : b->block_cap * 4ull * Bmax * Bmax;
    b->tcap = d->triangleCapacity ? d->triangleCapacity : b->block_cap * 8ull * Bmax * Bmax;
    const uint32_t face_stride = 3 * Bmax * Bmax;
    const uint64_t n_stiles = (b->block_cap + kBTile - 1) / kBTile;

    // device memory
    void *p_vols, *p_jobs, *p_tiles, *p_leaf, *p_rank, *p_ids, *p_jobof, *p_desc, *p_faces, *p_verts, *p_idx;
    b->ctrl_bytes = align256(sizeof(BCtrl));
    const size_t off_fst = b->ctrl_bytes;
    const size_t off_sst = align256(off_fst + 4ull * b->n_ftiles);
    const size_t off_res = align256(off_sst + 8ull * n_stiles);
    const size_t off_end = align256(off_res + sizeof(mtx_batch_job_result) * b->njobs);
    b->ctrl_bytes = align256(off_end + 4ull * b->njobs);
    if ((rs = batch_alloc(b, &p_vols, sizeof(BVol) * b->nvol)) != MTX_OK ||
        (rs = batch_alloc(b, &p_jobs, sizeof(BJob) * b->njobs)) != MTX_OK ||
        (rs = batch_alloc(b, &p_tiles, 4ull * b->n_ftiles)) != MTX_OK ||
        (rs = batch_alloc(b, &p_leaf, 8ull * leaf_total)) != MTX_OK ||
        (rs = batch_alloc(b, &p_rank, 4ull * rank_total)) != MTX_OK ||
        (rs = batch_alloc(b, &p_ids, 4ull * b->block_cap)) != MTX_OK ||
        (rs = batch_alloc(b, &p_jobof, 4ull * b->block_cap)) != MTX_OK ||
        (rs = batch_alloc(b, &p_desc, sizeof(mtx_meshlet_descriptor) * b->block_cap)) != MTX_OK ||
        (rs = batch_alloc(b, &p_faces, 4ull * face_stride * b->block_cap)) != MTX_OK ||
        (rs = batch_alloc(b, &p_verts, (size_t)b->vsz * b->vcap)) != MTX_OK ||
        (rs = batch_alloc(b, &p_idx, 12ull * b->tcap)) != MTX_OK ||
        (rs = batch_alloc(b, &b->ctrl_region, b->ctrl_bytes)) != MTX_OK) {
        batch_release(b);
        return rs;
    }
    b->vols = (BVol *)p_vols;
    b->leaf = (uint2 *)p_leaf;
    cudaError_t e = cudaMemcpy(p_vols, vols.data(), sizeof(BVol) * b->nvol, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p_jobs, jobs.data(), sizeof(BJob) * b->njobs, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p_tiles, tile_job.data(), 4ull * b->n_ftiles, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        batch_release(b);
        return cuda_fail(c, e, "batch tables");
    }

    BatchArgs &a = b->args;
    char *cr = (char *)b->ctrl_region;
    a.vols = (const BVol *)p_vols;
    a.jobs = (const BJob *)p_jobs;
    a.tile_job = (const uint32_t *)p_tiles;
    a.leaf = (const uint2 *)p_leaf;
    a.njobs = b->njobs;
    a.n_ftiles = b->n_ftiles;
    a.ws_bytes = L.bytes;
    a.face_stride = face_stride;
    a.rank_pool = (uint32_t *)p_rank;
    a.ids = (uint32_t *)p_ids;
    a.job_of = (uint32_t *)p_jobof;
    a.block_cap = b->block_cap;
    a.desc = (mtx_meshlet_descriptor *)p_desc;
    a.faces = (uint32_t *)p_faces;
    a.filter_status = (uint32_t *)(cr + off_fst);
    a.scan_status = (uint64_t *)(cr + off_sst);
    a.res = (mtx_batch_job_result *)(cr + off_res);
    a.job_end = (uint32_t *)(cr + off_end);
    a.vertices = p_verts;
    a.vcap = b->vcap;
    a.indices = (uint32_t *)p_idx;
    a.tcap = b->tcap;
    a.vfmt = d->vertexFormat;
    a.frame = d->frame;
    a.normals = d->vertexFormat == MTX_VERTEX_DATA ? d->normals : 0u;
    a.vsz = b->vsz;
    a.ctrl = (BCtrl *)b->ctrl_region;

    // persistent grid: every CTA that fits at once
    const bool generic = d->vertexFormat != MTX_VERTEX_XYZ || d->frame != MTX_FRAME_VOXEL;
    bool all8 = true;
    for (uint32_t v = 0; v < b->nvol; ++v) all8 = all8 && d->blockEdges[v] == 8;
    b->variant = all8 ? 4 + (generic ? 1 : 0) : (Bmax > 8 ? 2 : 0) + (generic ? 1 : 0);
    // as many block warps per CTA as the shared memory holds (8 unless the
    // largest plan is a 16^3 float32 tile)
    const int static_smem = 1024;
    const int room = (c->max_smem_optin > 0 ? c->max_smem_optin : 227 * 1024) - (int)kTableBytes - static_smem;
    a.block_warps = (uint32_t)std::min<int>(kBWarps, std::max(0, room / (int)L.bytes));
    if (d->blockWarps > kBWarps) {
        batch_release(b);
        return fail(c, MTX_ERR_INVALID_ARG, "batch: blockWarps outside 0..8");
    }
    if (d->blockWarps) a.block_warps = std::min<uint32_t>(a.block_warps, d->blockWarps);
    if (a.block_warps == 0) {
        batch_release(b);
        return fail(c, MTX_ERR_UNSUPPORTED, "batch: warp layout does not fit shared memory");
    }
    b->smem = kTableBytes + a.block_warps * L.bytes;
    KernelFn fn = batch_kernel(b->variant);
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem);
    // all of the unified L1 as shared memory: more resident warps hide the
    // block bodies' shared-memory latencies
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    int occ = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kBThreads, b->smem);
    if (e != cudaSuccess) {
        batch_release(b);
        return cuda_fail(c, e, "batch kernel occupancy");
    }
    if (occ < 1) {
        batch_release(b);
        return fail(c, MTX_ERR_UNSUPPORTED, "batch: warp layout does not fit shared memory");
    }
    b->grid = (uint32_t)occ * (uint32_t)c->sm_count;
    b->use_graph = d->useGraph != 0;
    *out = b;
    return MTX_OK;
}

mtx_status mtx_batch_run(mtx_batch_t b) {
    if (!b) return MTX_ERR_INVALID_ARG;
    mtx_context *c = b->ctx;
    DeviceGuard dg(c->device);
    join_extract(c);
    if (!b->use_graph) return batch_enqueue(b, c->stream);
    if (!b->exec) {
        if (!b->capture_stream) MTX_CUDA(c, cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking));
        MTX_CUDA(c, cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
        mtx_status rs = batch_enqueue(b, b->capture_stream);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->capture_stream, &g);
        if (rs != MTX_OK) {
            if (g) cudaGraphDestroy(g);
            return rs;
        }
        if (e != cudaSuccess) return cuda_fail(c, e, "batch graph capture");
        b->graph = g;
        MTX_CUDA(c, cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    MTX_CUDA(c, cudaGraphLaunch(b->exec, c->stream));
    return MTX_OK;
}

mtx_status mtx_batch_get_outputs(mtx_batch_t b, mtx_batch_outputs *o) {
    if (!b || !o) return MTX_ERR_INVALID_ARG;
    memset(o, 0, sizeof(*o));
    o->vertexBuffer = {b->args.vertices, (uint64_t)b->vsz * b->vcap};
    o->indexBuffer = {b->args.indices, 12ull * b->tcap};
    o->meshletDescriptorBuffer = {b->args.desc, sizeof(mtx_meshlet_descriptor) * b->block_cap};
    o->jobResultBuffer = {b->args.res, sizeof(mtx_batch_job_result) * b->njobs};
    o->vertexStride = b->vsz;
    return MTX_OK;
}

mtx_status mtx_batch_read_results(mtx_batch_t b, mtx_batch_job_result *results, mtx_batch_totals *totals) {
    if (!b) return MTX_ERR_INVALID_ARG;
    mtx_context *c = b->ctx;
    DeviceGuard dg(c->device);
    join_extract(c);
    MTX_CUDA(c, cudaStreamSynchronize(c->stream));
    if (results)
        MTX_CUDA(c, cudaMemcpy(results, b->args.res, sizeof(mtx_batch_job_result) * b->njobs, cudaMemcpyDeviceToHost));
    BCtrl h;
    MTX_CUDA(c, cudaMemcpy(&h, b->ctrl_region, sizeof(BCtrl), cudaMemcpyDeviceToHost));
    if (totals) {
        totals->status = (int32_t)h.status.code;
        totals->activeBlocks = h.total_active;
        totals->vertexCount = h.total_vertices;
        totals->triangleCount = h.total_triangles;
    }
    if (h.status.code != 0)
        return fail(c, (mtx_status)h.status.code,
                    "batch run: device error at site " + std::to_string(h.status.where) + " (" +
                        std::to_string(h.status.info0) + ", " + std::to_string(h.status.info1) + ")");
    return MTX_OK;
}

mtx_status mtx_batch_destroy(mtx_batch_t b) {
    if (!b) return MTX_ERR_INVALID_ARG;
    DeviceGuard dg(b->ctx->device);
    join_extract(b->ctx);
    batch_release(b);
    return MTX_OK;
}

}  // extern "C"
