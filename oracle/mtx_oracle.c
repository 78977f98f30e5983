/*
 * meshtrex CPU oracle -- TEST INFRASTRUCTURE ONLY (see mtx_oracle.h).
 *
 * Compiled with -ffp-contract=off so that every float operation below rounds
 * once, in the order written: the CUDA kernels use the same formulas with
 * __fadd_rn/__fsub_rn/__fmul_rn/__fdiv_rn/__fsqrt_rn and must agree bit for bit.
 */
#include "mtx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../meshtrex_b200/csrc/mc_case_table.h"

/* ------------------------------------------------------------------ values */

uint32_t orc_key_of_f32(float f) {
    uint32_t b;
    memcpy(&b, &f, 4);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

float orc_f32_of_key(uint32_t k) {
    uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    memcpy(&f, &b, 4);
    return f;
}

static inline size_t vidx(const orc_volume *v, uint32_t x, uint32_t y, uint32_t z) {
    return ((size_t)z * v->dims[1] + y) * v->dims[0] + x;
}

/* Voxel value as the float the extraction compares and interpolates with
 * (marching_cubes_pmb.mesh.glsl:123-124,150: float(imageLoad(...))). */
static inline float valf(const orc_volume *v, size_t i) {
    switch (v->dtype) {
    case ORC_U8: return (float)((const uint8_t *)v->data)[i];
    case ORC_U16: return (float)((const uint16_t *)v->data)[i];
    case ORC_F32: return ((const float *)v->data)[i];
    default: return (float)((const double *)v->data)[i];
    }
}

static inline double vald(const orc_volume *v, size_t i) {
    if (v->dtype == ORC_F64) return ((const double *)v->data)[i];
    return (double)valf(v, i);
}

static inline uint32_t keyv(const orc_volume *v, size_t i) {
    switch (v->dtype) {
    case ORC_U8: return ((const uint8_t *)v->data)[i];
    case ORC_U16: return ((const uint16_t *)v->data)[i];
    default: return orc_key_of_f32(valf(v, i));
    }
}

/* Inside test of one corner: bit i of the case is set iff value <= iso
 * (marching_cubes_pmb.mesh.glsl:150-153).  Exact in double for every dtype. */
static inline int inside(const orc_volume *v, size_t i, double iso) { return vald(v, i) <= iso; }

void orc_block_grid(const uint32_t dims[3], const uint32_t blk[3], uint32_t grid[3]) {
    /* blockGridDim = ceil(volumeDim / blockDim) (src/meshtrex.cpp:79-83) */
    for (int a = 0; a < 3; ++a) grid[a] = (dims[a] + blk[a] - 1) / blk[a];
}

static int nthreads_or_1(int n) { return n > 0 ? n : 1; }

/* ---------------------------------------------------------------- min/max */

static void minmax_range(const orc_volume *v, const uint32_t lo[3], const uint32_t hi[3],
                         uint32_t *mn, uint32_t *mx, int *any) {
    uint32_t a = 0xFFFFFFFFu, b = 0u;
    int seen = 0;
    for (uint32_t z = lo[2]; z <= hi[2]; ++z)
        for (uint32_t y = lo[1]; y <= hi[1]; ++y)
            for (uint32_t x = lo[0]; x <= hi[0]; ++x) {
                uint32_t k = keyv(v, vidx(v, x, y, z));
                if (k < a) a = k;
                if (k > b) b = k;
                seen = 1;
            }
    *mn = a;
    *mx = b;
    *any = seen;
}

void orc_minmax_halo(const orc_volume *v, const uint32_t blk[3], uint32_t *out, int nthreads) {
    uint32_t g[3];
    orc_block_grid(v->dims, blk, g);
    int64_t rows = (int64_t)g[1] * g[2];
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads_or_1(nthreads))
    for (int64_t r = 0; r < rows; ++r) {
        uint32_t by = (uint32_t)(r % g[1]), bz = (uint32_t)(r / g[1]);
        for (uint32_t bx = 0; bx < g[0]; ++bx) {
            uint32_t b[3] = {bx, by, bz}, lo[3], hi[3];
            for (int a = 0; a < 3; ++a) {
                /* (blockDim + 1) voxels from blockID * blockDim, bounds-checked
                 * (minMaxLeaf.comp.glsl:39,46-47,73) */
                lo[a] = b[a] * blk[a];
                hi[a] = lo[a] + blk[a];
                if (hi[a] > v->dims[a] - 1) hi[a] = v->dims[a] - 1;
            }
            uint32_t mn, mx;
            int any;
            minmax_range(v, lo, hi, &mn, &mx, &any);
            size_t i = ((size_t)bz * g[1] + by) * g[0] + bx;
            out[2 * i] = mn;
            out[2 * i + 1] = mx;
        }
    }
}

void orc_minmax_core(const orc_volume *v, const uint32_t blk[3], uint32_t *out) {
    uint32_t g[3];
    orc_block_grid(v->dims, blk, g);
    for (uint32_t bz = 0; bz < g[2]; ++bz)
        for (uint32_t by = 0; by < g[1]; ++by)
            for (uint32_t bx = 0; bx < g[0]; ++bx) {
                uint32_t b[3] = {bx, by, bz}, lo[3], hi[3];
                for (int a = 0; a < 3; ++a) {
                    lo[a] = b[a] * blk[a];
                    hi[a] = lo[a] + blk[a] - 1; /* B voxels (testMinMax.h:88-96) */
                    if (hi[a] > v->dims[a] - 1) hi[a] = v->dims[a] - 1;
                }
                uint32_t mn, mx;
                int any;
                minmax_range(v, lo, hi, &mn, &mx, &any);
                size_t i = ((size_t)bz * g[1] + by) * g[0] + bx;
                /* empty block -> {0,0} (testMinMax.h:119-127) */
                out[2 * i] = any ? mn : 0u;
                out[2 * i + 1] = any ? mx : 0u;
            }
}

/* --------------------------------------------------------------- pyramid */

int orc_mip_levels(const uint32_t grid[3]) {
    uint32_t m = grid[0];
    if (grid[1] > m) m = grid[1];
    if (grid[2] > m) m = grid[2];
    int l = 1;
    while (m > 1) { /* 1 + floor(log2(m)) */
        m >>= 1;
        ++l;
    }
    return l;
}

void orc_mip_extent(const uint32_t grid[3], int level, uint32_t ext[3]) {
    for (int a = 0; a < 3; ++a) {
        uint32_t e = grid[a];
        for (int l = 0; l < level; ++l) e = (e + 1) / 2; /* ceil: minMaxManager.cpp:147-151 */
        ext[a] = e;
    }
}

uint64_t orc_mip_offset(const uint32_t grid[3], int level) {
    uint64_t off = 0;
    for (int l = 0; l < level; ++l) {
        uint32_t e[3];
        orc_mip_extent(grid, l, e);
        off += (uint64_t)e[0] * e[1] * e[2];
    }
    return off;
}

void orc_pyramid(const uint32_t *leaf, const uint32_t grid[3], uint32_t *all) {
    int L = orc_mip_levels(grid);
    uint64_t n0 = (uint64_t)grid[0] * grid[1] * grid[2];
    memcpy(all, leaf, n0 * 2 * sizeof(uint32_t));
    for (int l = 1; l < L; ++l) {
        uint32_t es[3], ed[3];
        orc_mip_extent(grid, l - 1, es);
        orc_mip_extent(grid, l, ed);
        const uint32_t *src = all + 2 * orc_mip_offset(grid, l - 1);
        uint32_t *dst = all + 2 * orc_mip_offset(grid, l);
        for (uint32_t z = 0; z < ed[2]; ++z)
            for (uint32_t y = 0; y < ed[1]; ++y)
                for (uint32_t x = 0; x < ed[0]; ++x) {
                    uint32_t mn = 0xFFFFFFFFu, mx = 0u;
                    for (int c = 0; c < 8; ++c) {
                        uint32_t sx = 2 * x + (c & 1), sy = 2 * y + ((c >> 1) & 1),
                                 sz = 2 * z + ((c >> 2) & 1);
                        /* invalid children are skipped (minMaxOctreeReduce.comp.glsl:37-47) */
                        if (sx >= es[0] || sy >= es[1] || sz >= es[2]) continue;
                        size_t si = ((size_t)sz * es[1] + sy) * es[0] + sx;
                        if (src[2 * si] < mn) mn = src[2 * si];
                        if (src[2 * si + 1] > mx) mx = src[2 * si + 1];
                    }
                    size_t di = ((size_t)z * ed[1] + y) * ed[0] + x;
                    dst[2 * di] = mn;
                    dst[2 * di + 1] = mx;
                }
    }
}

/* ------------------------------------------------------------- filtering */

int orc_block_active(int dtype, uint32_t kmin, uint32_t kmax, float iso) {
    if (dtype == ORC_F32) {
        float a = orc_f32_of_key(kmin), b = orc_f32_of_key(kmax);
        return (a != b) && iso >= a && iso <= b;
    }
    /* isovalue_uint = round(isovalue); active iff min != max and
     * isovalue_uint in [min, max] (blockFilteringTestUtils.h:456-469).  The
     * comparison is done on the rounded float, which equals the reference
     * for every isovalue its cast defines and rejects negative ones. */
    float r = roundf(iso);
    return (kmin != kmax) && r >= (float)kmin && r <= (float)kmax;
}

uint32_t orc_compact(const uint32_t *mm, uint64_t nblocks, int dtype, float iso, uint32_t *ids) {
    uint32_t n = 0;
    for (uint64_t b = 0; b < nblocks; ++b) /* ascending 1D order (:462-474) */
        if (orc_block_active(dtype, mm[2 * b], mm[2 * b + 1], iso)) {
            if (ids) ids[n] = (uint32_t)b;
            ++n;
        }
    return n;
}

/* ------------------------------------------------------- marching cubes */

typedef struct {
    const orc_volume *v;
    uint32_t blk[3], grid[3];
    double iso;
    float isof;
} mc_ctx;

static void block_origin(const mc_ctx *m, uint32_t id, uint32_t o[3]) {
    /* unpack_block_id (marching_cubes_pmb.task.glsl:75-79) */
    o[0] = (id % m->grid[0]) * m->blk[0];
    o[1] = ((id / m->grid[0]) % m->grid[1]) * m->blk[1];
    o[2] = (id / (m->grid[0] * m->grid[1])) * m->blk[2];
}

/* 3-bit mask of the crossed +x/+y/+z edges owned by voxel u (PMB ownership,
 * marching_cubes_pmb.mesh.glsl:31-35,224-226); edges leaving the volume do not exist. */
static unsigned owned_mask(const mc_ctx *m, const uint32_t u[3]) {
    const orc_volume *v = m->v;
    if (u[0] >= v->dims[0] || u[1] >= v->dims[1] || u[2] >= v->dims[2]) return 0;
    int s = inside(v, vidx(v, u[0], u[1], u[2]), m->iso);
    unsigned mask = 0;
    for (int a = 0; a < 3; ++a) {
        uint32_t w[3] = {u[0], u[1], u[2]};
        w[a] += 1;
        if (w[a] >= v->dims[a]) continue;
        if (inside(v, vidx(v, w[0], w[1], w[2]), m->iso) != s) mask |= 1u << a;
    }
    return mask;
}

/* Case index of the cell at c (calculate_configuration, pmb.mesh.glsl:144-156);
 * -1 if the cell leaves the volume (pmb.task.glsl:121). */
static int cell_case(const mc_ctx *m, const uint32_t c[3]) {
    const orc_volume *v = m->v;
    for (int a = 0; a < 3; ++a)
        if (c[a] + 1 >= v->dims[a]) return -1;
    unsigned cfg = 0;
    for (int i = 0; i < 8; ++i) {
        uint32_t x = c[0] + MTX_MC_CORNER[i][0], y = c[1] + MTX_MC_CORNER[i][1],
                 z = c[2] + MTX_MC_CORNER[i][2];
        if (inside(v, vidx(v, x, y, z), m->iso)) cfg |= 1u << i;
    }
    return (int)cfg;
}

static void count_block(const mc_ctx *m, uint32_t id, uint32_t *nv, uint32_t *nt) {
    uint32_t o[3];
    block_origin(m, id, o);
    uint32_t a = 0, b = 0;
    for (uint32_t lz = 0; lz < m->blk[2]; ++lz)
        for (uint32_t ly = 0; ly < m->blk[1]; ++ly)
            for (uint32_t lx = 0; lx < m->blk[0]; ++lx) {
                uint32_t u[3] = {o[0] + lx, o[1] + ly, o[2] + lz};
                unsigned mask = owned_mask(m, u);
                a += (mask & 1) + ((mask >> 1) & 1) + ((mask >> 2) & 1);
                int cfg = cell_case(m, u);
                if (cfg >= 0) b += (uint32_t)mtx_mc_tri_count((unsigned)cfg);
            }
    *nv = a;
    *nt = b;
}

void orc_cell_cases(const orc_volume *v, const uint32_t blk[3], float iso, const uint32_t *ids,
                    uint32_t n_active, uint8_t *out) {
    mc_ctx m = {v, {blk[0], blk[1], blk[2]}, {0, 0, 0}, (double)iso, iso};
    orc_block_grid(v->dims, blk, m.grid);
    size_t cells = (size_t)blk[0] * blk[1] * blk[2];
    for (uint32_t r = 0; r < n_active; ++r) {
        uint32_t o[3];
        block_origin(&m, ids[r], o);
        size_t k = 0;
        for (uint32_t lz = 0; lz < blk[2]; ++lz)
            for (uint32_t ly = 0; ly < blk[1]; ++ly)
                for (uint32_t lx = 0; lx < blk[0]; ++lx, ++k) {
                    uint32_t c[3] = {o[0] + lx, o[1] + ly, o[2] + lz};
                    int cfg = cell_case(&m, c);
                    out[r * cells + k] = (uint8_t)(cfg < 0 ? 0 : cfg);
                }
    }
}

/* FP32 edge parameter (interpolate_vertex, marching_cubes_pmb.mesh.glsl:129-134;
 * extractionTestUtils.cpp:34-36): t = (iso - a) / (b - a) when |b - a| > 1e-5,
 * else 0.5; clamped to [0,1]. */
static float edge_t(float fa, float fb, float iso) {
    float den = fb - fa;
    float t = 0.5f;
    if (fabsf(den) > 1e-5f) t = (iso - fa) / den;
    if (t < 0.0f) t = 0.0f;
    if (t > 1.0f) t = 1.0f;
    return t;
}

static double edge_t64(double fa, double fb, double iso) {
    double den = fb - fa;
    double t = 0.5;
    if (fabs((float)fb - (float)fa) > 1e-5f) t = (iso - fa) / den;
    if (t < 0.0) t = 0.0;
    if (t > 1.0) t = 1.0;
    return t;
}

static void normalize3(float n[3]) {
    float d = n[0] * n[0] + n[1] * n[1];
    d = d + n[2] * n[2];
    if (d == 0.0f) {
        n[0] = n[1] = n[2] = 0.0f;
        return;
    }
    float l = sqrtf(d);
    n[0] = n[0] / l;
    n[1] = n[1] / l;
    n[2] = n[2] / l;
}

/* Clamped central difference, normalised (calculate_normal, pmb.mesh.glsl:111-120). */
static void voxel_normal(const orc_volume *v, const uint32_t p[3], float n[3]) {
    for (int a = 0; a < 3; ++a) {
        uint32_t lo[3] = {p[0], p[1], p[2]}, hi[3] = {p[0], p[1], p[2]};
        lo[a] = p[a] > 0 ? p[a] - 1 : 0;
        hi[a] = p[a] + 1 < v->dims[a] ? p[a] + 1 : v->dims[a] - 1;
        n[a] = valf(v, vidx(v, lo[0], lo[1], lo[2])) - valf(v, vidx(v, hi[0], hi[1], hi[2]));
    }
    normalize3(n);
}

int orc_mc_extract(const orc_volume *v, const uint32_t blk[3], float iso, const uint32_t *ids,
                   uint32_t n_active, int frame, int nthreads, orc_mesh_counts *counts,
                   uint32_t *nvpb, uint32_t *ntpb, float *xyz, double *xyz64, float *normals,
                   uint32_t *indices) {
    mc_ctx m = {v, {blk[0], blk[1], blk[2]}, {0, 0, 0}, (double)iso, iso};
    orc_block_grid(v->dims, blk, m.grid);
    uint64_t nblocks = (uint64_t)m.grid[0] * m.grid[1] * m.grid[2];
    uint32_t *nv = (uint32_t *)calloc(n_active ? n_active : 1, 4);
    uint32_t *nt = (uint32_t *)calloc(n_active ? n_active : 1, 4);
    if (!nv || !nt) return -1;
    (void)nthreads;

#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads_or_1(nthreads))
    for (int64_t r = 0; r < (int64_t)n_active; ++r) count_block(&m, ids[r], &nv[r], &nt[r]);

    /* exclusive scans over the active blocks in rank order */
    uint64_t *vb = (uint64_t *)malloc(8 * (size_t)(n_active + 1));
    uint64_t *tb = (uint64_t *)malloc(8 * (size_t)(n_active + 1));
    if (!vb || !tb) return -1;
    vb[0] = tb[0] = 0;
    for (uint32_t r = 0; r < n_active; ++r) {
        vb[r + 1] = vb[r] + nv[r];
        tb[r + 1] = tb[r] + nt[r];
    }
    if (counts) {
        counts->n_vertices = vb[n_active];
        counts->n_triangles = tb[n_active];
    }
    if (nvpb) memcpy(nvpb, nv, 4 * (size_t)n_active);
    if (ntpb) memcpy(ntpb, nt, 4 * (size_t)n_active);

    int want = xyz || xyz64 || normals || indices;
    if (!want) {
        free(nv); free(nt); free(vb); free(tb);
        return 0;
    }

    /* rank map and the first vertex id (relative to the block) of every voxel */
    uint32_t *rank = (uint32_t *)malloc(4 * (size_t)nblocks);
    size_t cells = (size_t)blk[0] * blk[1] * blk[2];
    uint32_t *first = (uint32_t *)malloc(4 * cells * (size_t)(n_active ? n_active : 1));
    if (!rank || !first) return -1;
    for (uint64_t b = 0; b < nblocks; ++b) rank[b] = 0xFFFFFFFFu;
    for (uint32_t r = 0; r < n_active; ++r) rank[ids[r]] = r;

    int err = 0;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads_or_1(nthreads))
    for (int64_t r = 0; r < (int64_t)n_active; ++r) {
        uint32_t o[3];
        block_origin(&m, ids[r], o);
        uint32_t run = 0;
        size_t k = 0;
        for (uint32_t lz = 0; lz < blk[2]; ++lz)
            for (uint32_t ly = 0; ly < blk[1]; ++ly)
                for (uint32_t lx = 0; lx < blk[0]; ++lx, ++k) {
                    uint32_t u[3] = {o[0] + lx, o[1] + ly, o[2] + lz};
                    unsigned mask = owned_mask(&m, u);
                    first[(size_t)r * cells + k] = run;
                    for (int a = 0; a < 3; ++a) {
                        if (!(mask & (1u << a))) continue;
                        uint64_t id = vb[r] + run++;
                        uint32_t w[3] = {u[0], u[1], u[2]};
                        w[a] += 1;
                        size_t ia = vidx(v, u[0], u[1], u[2]), ib = vidx(v, w[0], w[1], w[2]);
                        if (xyz) {
                            float t = edge_t(valf(v, ia), valf(v, ib), iso);
                            float p[3] = {(float)u[0], (float)u[1], (float)u[2]};
                            p[a] = p[a] + t;
                            for (int c = 0; c < 3; ++c) {
                                float q = p[c];
                                if (frame == ORC_FRAME_NDC) {
                                    /* (pos / volumeDim) * 2 - 1 (pmb.mesh.glsl:138) */
                                    q = q / (float)v->dims[c];
                                    q = q * 2.0f;
                                    q = q - 1.0f;
                                }
                                xyz[3 * id + c] = q;
                            }
                        }
                        if (xyz64) {
                            double t = edge_t64(vald(v, ia), vald(v, ib), (double)iso);
                            double p[3] = {(double)u[0], (double)u[1], (double)u[2]};
                            p[a] += t;
                            for (int c = 0; c < 3; ++c)
                                xyz64[3 * id + c] =
                                    frame == ORC_FRAME_NDC ? p[c] / v->dims[c] * 2.0 - 1.0 : p[c];
                        }
                        if (normals) {
                            float t = edge_t(valf(v, ia), valf(v, ib), iso);
                            float n1[3], n2[3], n[3];
                            voxel_normal(v, u, n1);
                            voxel_normal(v, w, n2);
                            float omt = 1.0f - t;
                            for (int c = 0; c < 3; ++c) {
                                float x1 = n1[c] * omt, x2 = n2[c] * t;
                                n[c] = x1 + x2; /* mix(n1, n2, t) */
                            }
                            normalize3(n);
                            for (int c = 0; c < 3; ++c) normals[3 * id + c] = n[c];
                        }
                    }
                }
    }

    if (indices) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads_or_1(nthreads))
        for (int64_t r = 0; r < (int64_t)n_active; ++r) {
            uint32_t o[3];
            block_origin(&m, ids[r], o);
            uint64_t tri = tb[r];
            for (uint32_t lz = 0; lz < blk[2]; ++lz)
                for (uint32_t ly = 0; ly < blk[1]; ++ly)
                    for (uint32_t lx = 0; lx < blk[0]; ++lx) {
                        uint32_t c[3] = {o[0] + lx, o[1] + ly, o[2] + lz};
                        int cfg = cell_case(&m, c);
                        if (cfg < 0) continue;
                        int ntri = mtx_mc_tri_count((unsigned)cfg);
                        for (int t = 0; t < ntri; ++t, ++tri)
                            for (int k = 0; k < 3; ++k) {
                                int e = mtx_mc_tri_edge((unsigned)cfg, 3 * t + k);
                                unsigned own = MTX_MC_EDGE_OWNER[e];
                                uint32_t u[3] = {c[0] + (own & 1), c[1] + ((own >> 1) & 1),
                                                 c[2] + ((own >> 2) & 1)};
                                unsigned axis = own >> 3;
                                uint32_t b[3] = {u[0] / blk[0], u[1] / blk[1], u[2] / blk[2]};
                                uint64_t bid = ((uint64_t)b[2] * m.grid[1] + b[1]) * m.grid[0] + b[0];
                                uint32_t ru = rank[bid];
                                unsigned mask = owned_mask(&m, u);
                                if (ru == 0xFFFFFFFFu || !(mask & (1u << axis))) {
                                    err = 1; /* impossible for a consistent mesh */
                                    continue;
                                }
                                size_t loc = ((size_t)(u[2] - b[2] * blk[2]) * blk[1] +
                                              (u[1] - b[1] * blk[1])) * blk[0] + (u[0] - b[0] * blk[0]);
                                unsigned below = mask & ((1u << axis) - 1u);
                                uint64_t id = vb[ru] + first[(size_t)ru * cells + loc] +
                                              (below & 1) + ((below >> 1) & 1);
                                indices[3 * tri + k] = (uint32_t)id;
                            }
                    }
        }
    }
    free(rank); free(first); free(nv); free(nt); free(vb); free(tb);
    return err ? -2 : 0;
}

int orc_mc_adjoint(const orc_volume *v, const uint32_t blk[3], float iso, const uint32_t *ids,
                   uint32_t n_active, const float *g, double *dfield, double *diso) {
    mc_ctx m = {v, {blk[0], blk[1], blk[2]}, {0, 0, 0}, (double)iso, iso};
    orc_block_grid(v->dims, blk, m.grid);
    size_t nvox = (size_t)v->dims[0] * v->dims[1] * v->dims[2];
    memset(dfield, 0, nvox * sizeof(double));
    double acc_iso = 0.0;
    uint64_t id = 0;
    double isod = (double)iso;
    for (uint32_t r = 0; r < n_active; ++r) {
        uint32_t o[3];
        block_origin(&m, ids[r], o);
        for (uint32_t lz = 0; lz < blk[2]; ++lz)
            for (uint32_t ly = 0; ly < blk[1]; ++ly)
                for (uint32_t lx = 0; lx < blk[0]; ++lx) {
                    uint32_t u[3] = {o[0] + lx, o[1] + ly, o[2] + lz};
                    unsigned mask = owned_mask(&m, u);
                    for (int a = 0; a < 3; ++a) {
                        if (!(mask & (1u << a))) continue;
                        uint32_t w[3] = {u[0], u[1], u[2]};
                        w[a] += 1;
                        size_t ia = vidx(v, u[0], u[1], u[2]), ib = vidx(v, w[0], w[1], w[2]);
                        double fa = vald(v, ia), fb = vald(v, ib), ga = (double)g[3 * id + a];
                        ++id;
                        /* pos[a] = u[a] + t, t = (iso - fa) / (fb - fa); the
                         * constant branch (|den| <= 1e-5) has no gradient. */
                        if (!(fabs((float)fb - (float)fa) > 1e-5f)) continue;
                        double den = fb - fa, t = (isod - fa) / den;
                        if (t < 0.0 || t > 1.0) continue;
                        dfield[ia] += ga * (isod - fb) / (den * den);
                        dfield[ib] += ga * (fa - isod) / (den * den);
                        acc_iso += ga / den;
                    }
                }
    }
    *diso = acc_iso;
    return 0;
}

int orc_pipeline(const orc_volume *v, const uint32_t blk[3], float iso, int nthreads,
                 orc_mesh_counts *counts, uint32_t *n_active_out, float *xyz, uint32_t *indices) {
    uint32_t g[3];
    orc_block_grid(v->dims, blk, g);
    uint64_t nb = (uint64_t)g[0] * g[1] * g[2];
    uint32_t *mm = (uint32_t *)malloc(8 * (size_t)nb);
    uint32_t *ids = (uint32_t *)malloc(4 * (size_t)nb);
    if (!mm || !ids) return -1;
    orc_minmax_halo(v, blk, mm, nthreads);
    uint32_t na = orc_compact(mm, nb, v->dtype, iso, ids);
    if (n_active_out) *n_active_out = na;
    int rc = orc_mc_extract(v, blk, iso, ids, na, ORC_FRAME_VOXEL, nthreads, counts, NULL, NULL,
                            xyz, NULL, NULL, indices);
    free(mm);
    free(ids);
    return rc;
}

/* Meshlet split (see the header): a straight restatement with a linear
 * search of the current meshlet's vertex list. */
uint64_t orc_meshlets(const uint32_t *ntri_per_block, uint32_t n_blocks, const uint32_t *indices, uint32_t max_v,
                      uint32_t max_p, uint32_t *desc, uint32_t *mverts, uint32_t *midx, uint64_t *n_mverts) {
    uint64_t m = 0, mv = 0, t = 0;
    uint32_t list[1024];
    for (uint32_t b = 0; b < n_blocks; ++b) {
        const uint64_t t1 = t + ntri_per_block[b];
        uint32_t cur_v = 0, cur_p = 0;
        uint64_t first_t = t, vstart = mv;
        for (; t < t1; ++t) {
            uint32_t loc[3], fresh = 0;
            for (int k = 0; k < 3; ++k) {
                loc[k] = UINT32_MAX;
                for (uint32_t i = 0; i < cur_v; ++i)
                    if (list[i] == indices[3 * t + k]) loc[k] = i;
                int dup = 0;
                for (int j = 0; j < k; ++j) dup |= indices[3 * t + j] == indices[3 * t + k];
                if (loc[k] == UINT32_MAX && !dup) ++fresh;
            }
            if (cur_p > 0 && (cur_v + fresh > max_v || cur_p >= max_p)) {
                if (desc) {
                    desc[4 * m + 0] = (uint32_t)vstart;
                    desc[4 * m + 1] = (uint32_t)(3 * first_t);
                    desc[4 * m + 2] = cur_v;
                    desc[4 * m + 3] = cur_p;
                }
                ++m;
                vstart = mv;
                cur_v = cur_p = 0;
                first_t = t;
                loc[0] = loc[1] = loc[2] = UINT32_MAX;
            }
            for (int k = 0; k < 3; ++k) {
                const uint32_t id = indices[3 * t + k];
                if (loc[k] == UINT32_MAX) {
                    for (uint32_t i = 0; i < cur_v; ++i)
                        if (list[i] == id) loc[k] = i;
                }
                if (loc[k] == UINT32_MAX) {
                    loc[k] = cur_v;
                    list[cur_v++] = id;
                    if (mverts) mverts[mv] = id;
                    ++mv;
                }
                if (midx) midx[3 * t + k] = (uint32_t)(vstart + loc[k]);
            }
            ++cur_p;
        }
        if (cur_p > 0) {
            if (desc) {
                desc[4 * m + 0] = (uint32_t)vstart;
                desc[4 * m + 1] = (uint32_t)(3 * first_t);
                desc[4 * m + 2] = cur_v;
                desc[4 * m + 3] = cur_p;
            }
            ++m;
        }
    }
    if (n_mverts) *n_mverts = mv;
    return m;
}
