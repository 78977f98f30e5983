/*
 * meshtrex CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of meshtrex's isosurface-extraction path (block
 * min/max -> active-block filtering and compaction -> PMB marching cubes),
 * used by the tests, by smoke() and by bench.py's CPU baseline as the checker.
 * Nothing in the product library links, loads or calls it; the product fails
 * loudly when its CUDA library is missing instead of falling back to this.
 *
 * Parity pins (what this restatement is checked against):
 *  - block min/max in "core" mode (B voxels per axis, no overlap) against
 *    meshtrex's own computeMinMaxFromFile (src/testMinMax.h:28-135), compiled
 *    from the reference sources by oracle/build_ref.sh into oracle/_ref;
 *  - active-block counts against computeActiveBlockCountCPU
 *    (src/testMinMax.h:220-242) for integral isovalues;
 *  - the case table against MarchingCubes::triTable / edgeTable
 *    (src/mc_tables.h:17-308);
 *  - those outputs are also frozen as fixtures under tests/golden/.
 * The extraction geometry itself has no golden vectors in meshtrex (its only
 * extraction checks are structural, src/extractionTestUtils.cpp:371-464):
 * vertex positions and index buffers are parity-unpinned and are checked here
 * against an FP64 recomputation instead.
 */
#ifndef MTX_ORACLE_H
#define MTX_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_U8 = 0, ORC_U16 = 1, ORC_F32 = 2, ORC_F64 = 3 };
enum { ORC_FRAME_VOXEL = 0, ORC_FRAME_NDC = 1 };

typedef struct {
    const void *data;   /* x fastest, then y, then z (src/volume.h:8-12) */
    uint32_t dims[3];
    int dtype;
} orc_volume;

/* Order-preserving 32-bit key of a voxel value (identity for u8/u16, sign-flip for f32). */
uint32_t orc_key_of_f32(float f);
float orc_f32_of_key(uint32_t k);

void orc_block_grid(const uint32_t dims[3], const uint32_t blk[3], uint32_t grid[3]);

/* Per-block min/max keys over (B+1)^3 voxels starting at block*B, clipped to
 * the volume (src/shaders/minMaxLeaf.comp.glsl:39-79).  out[2i]=min, out[2i+1]=max. */
void orc_minmax_halo(const orc_volume *v, const uint32_t blk[3], uint32_t *out, int nthreads);

/* Per-block min/max over exactly B voxels per axis (src/testMinMax.h:79-130);
 * a block without voxels gets {0,0}. */
void orc_minmax_core(const orc_volume *v, const uint32_t blk[3], uint32_t *out);

/* Min/max octree: 1 + floor(log2(max grid extent)) levels
 * (src/minMaxManager.cpp:86-92), every level ceil(previous/2) per axis; a
 * texel reduces its (up to 8) children (src/shaders/minMaxOctreeReduce.comp.glsl:23-59). */
int orc_mip_levels(const uint32_t grid[3]);
void orc_mip_extent(const uint32_t grid[3], int level, uint32_t ext[3]);
uint64_t orc_mip_offset(const uint32_t grid[3], int level); /* texel offset of a level */
void orc_pyramid(const uint32_t *leaf, const uint32_t grid[3], uint32_t *all_levels);

/* Activity rule (src/blockFilteringTestUtils.h:456-474): min != max and the
 * isovalue inside [min, max]; integer volumes compare round(iso). */
int orc_block_active(int dtype, uint32_t kmin, uint32_t kmax, float iso);

/* Ordered compaction (src/blockFilteringTestUtils.h:438-478): ascending IDs. */
uint32_t orc_compact(const uint32_t *leaf_minmax, uint64_t nblocks, int dtype, float iso,
                     uint32_t *ids /* may be NULL */);

/* Per-cell case index of every cell of each active block (B^3 bytes per
 * block, x fastest; cells outside the volume are 0). */
void orc_cell_cases(const orc_volume *v, const uint32_t blk[3], float iso, const uint32_t *ids,
                    uint32_t n_active, uint8_t *out);

/* PMB marching cubes over the active blocks, canonical order:
 *  vertices: (owner block rank, owner voxel x-fastest in its block, axis x<y<z);
 *  triangles: (block rank, cell x-fastest in its block, triangle # in the case);
 *  indices are global vertex ids.
 * Pass NULL outputs to count only.  Returns 0 on success. */
typedef struct {
    uint64_t n_vertices;
    uint64_t n_triangles;
} orc_mesh_counts;

int orc_mc_extract(const orc_volume *v, const uint32_t blk[3], float iso, const uint32_t *ids,
                   uint32_t n_active, int frame, int nthreads, orc_mesh_counts *counts,
                   uint32_t *nvert_per_block, uint32_t *ntri_per_block, /* optional */
                   float *xyz,          /* 3 floats per vertex, optional */
                   double *xyz64,       /* FP64 recomputation, optional */
                   float *normals,      /* 3 floats per vertex, optional */
                   uint32_t *indices);  /* 3 per triangle, optional */

/* Adjoint of the vertex positions (voxel frame) with the topology held fixed:
 * dL/dfield (FP64, one per voxel, zero-filled here) and dL/diso. */
int orc_mc_adjoint(const orc_volume *v, const uint32_t blk[3], float iso, const uint32_t *ids,
                   uint32_t n_active, const float *dl_dxyz, double *dl_dfield, double *dl_diso);

/* Meshlet split of a canonical mesh (the rule of mtx_build_meshlets; no
 * meshtrex counterpart restated here, its limits are those of
 * marching_cubes_pmb.task.glsl:24-25): each block's triangles in order; a
 * triangle starts a new meshlet when its vertices not yet in the current
 * meshlet would take it past max_v, or the meshlet already has max_p
 * triangles.  A meshlet's vertices are listed in the order its triangles
 * first use them.  Writes per meshlet {vertexOffset, indexOffset, vertexCount,
 * primitiveCount} (desc, 4 words), the mesh vertex id of every meshlet vertex
 * (mverts) and the indices into the meshlet vertex stream (midx, 3 per
 * triangle); NULL outputs count only.  Returns the number of meshlets and
 * sets *n_mverts. */
uint64_t orc_meshlets(const uint32_t *ntri_per_block, uint32_t n_blocks, const uint32_t *indices, uint32_t max_v,
                      uint32_t max_p, uint32_t *desc, uint32_t *mverts, uint32_t *midx, uint64_t *n_mverts);

/* Whole plain pipeline (min/max -> compaction -> extraction) in one call, for
 * the CPU baseline: counts only when the output pointers are NULL. */
int orc_pipeline(const orc_volume *v, const uint32_t blk[3], float iso, int nthreads,
                 orc_mesh_counts *counts, uint32_t *n_active, float *xyz, uint32_t *indices);

#ifdef __cplusplus
}
#endif
#endif
