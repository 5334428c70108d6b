/*
 * oracle.h — CPU oracle for the RKIField SDF ray-march path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, as the checker / timed CPU baseline.
 *
 * It restates crates/rkf-render/shaders/ray_march.wgsl (the brute, BVH and
 * tiled marches, their samplers, bisection, normals, material and blend
 * lookups),
 * shade_common_shading.wgsl:9-47 (soft shadow), the voxelizer of
 * crates/rkf-core/src/voxelize_object.rs:53-182, the analytic SDFs of
 * crates/rkf-core/src/sdf.rs:12-51, the binary16 conversion of the `half`
 * crate (IEEE-754 round-to-nearest-even) and the CPU CSG edit of
 * crates/rkf-edit/src/cpu_apply.rs:28-262.
 *
 * Two arithmetic modes: FP32 with the reference operation order and no
 * contraction (the parity target of the GPU kernels), and FP64 with the same
 * control flow plus a root refinement of the trilinear surface (the error
 * reference).
 *
 * Parity status: no reference test pins ray_march.wgsl's output and the WGSL
 * pass cannot run here (no graphics stack), so the march restatement is
 * "parity unpinned" against the shader itself.  The pieces the reference's
 * own unit tests pin (VoxelSample packing, brick indexing, brick maps, the
 * analytic SDFs, smin, falloff, CSG edits) are pinned by tests/ against the
 * values those tests assert.
 */
#ifndef RKF_ORACLE_H
#define RKF_ORACLE_H

#include <stdint.h>
#include "../include/rkf_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

void orc_march_params_default(rkf_march_params* p);

/* The tiled strategy's coarse field over these objects' AABBs (0.32 m cells
 * over the union grown by 1 m, at most 128 per axis; binary16 texels of the
 * distance to the nearest AABB, x + y*dx + z*dx*dy).  Writes origin and
 * dims, and the texels when cap holds them; returns the texel count. */
uint64_t orc_coarse_field(const rkf_gpu_object* objects, uint32_t n, float origin[3], uint32_t dims[3],
                          uint16_t* tex, uint64_t cap);

/* ---- binary16 ---------------------------------------------------------- */
uint16_t orc_f16_from_f32(float f);
float orc_f16_to_f32(uint16_t h);

/* ---- analytic SDFs and the synthetic scene ------------------------------ */
float orc_prim_sdf(const rkf_prim* p, const float pos[3]);
float orc_smin(float a, float b, float k);
/* Scene distance with material/blend (the voxelizer's sdf_fn). */
float orc_scene_eval(const rkf_prim* prims, uint32_t n, float k, float cut,
                     const float pos[3], uint32_t* material, uint32_t* secondary,
                     uint32_t* blend);

/* ---- voxelizer -------------------------------------------------------- */
typedef struct orc_voxelized orc_voxelized;
/* Voxelize into a fresh pool (slots 0..n-1) + a flat brick map. */
orc_voxelized* orc_voxelize(const rkf_prim* prims, uint32_t n_prims,
                            const rkf_voxelize_params* vp, int threads);
// Voxelization into a two-level index and SoA planes (no flat map): the
// same slots and words as orc_voxelize, for grids too large for a flat map.
struct orc_sparse;
orc_sparse* orc_voxelize_sparse(const rkf_prim* prims, uint32_t n_prims, const rkf_voxelize_params* vp,
                                int threads);
void orc_sparse_info(const orc_sparse* v, uint32_t dims[3], uint32_t tdim[3], uint32_t* n_bricks,
                     uint32_t* n_interior, uint32_t* n_leaves);
void orc_sparse_copy(const orc_sparse* v, uint32_t* top, uint32_t* leaves, uint16_t* dist_f16, uint16_t* mat,
                     uint8_t* blend, uint32_t* bxyz);
void orc_sparse_free(orc_sparse* v);

void orc_voxelized_info(const orc_voxelized* v, uint32_t dims[3], uint32_t* n_bricks,
                        uint32_t* n_interior);
/* words: 1024 u32 per brick (VoxelSample AoS). map: dims.x*dims.y*dims.z. */
void orc_voxelized_copy(const orc_voxelized* v, uint32_t* words, uint32_t* map);
/* f32 distances before f16 rounding: 512 floats per brick. */
void orc_voxelized_copy_f32(const orc_voxelized* v, float* dist);
void orc_voxelized_free(orc_voxelized* v);
/* Classify selected bricks only (for huge grids): class[i] = slot-agnostic
 * result (0 = allocated, 1 = EMPTY, 2 = INTERIOR) and, when allocated, the
 * 1024 VoxelSample words of the brick into words[i*1024...]. */
void orc_voxelize_bricks(const rkf_prim* prims, uint32_t n_prims,
                         const rkf_voxelize_params* vp, const uint32_t* bxyz,
                         uint32_t n, uint32_t* cls, uint32_t* words, int threads);

/* ---- scene view consumed by the march --------------------------------- */
/* Pool: either reference AoS words (2 u32 per voxel) or SoA planes. */
typedef struct orc_scene {
    const uint32_t* pool_words;    /* AoS VoxelSample, may be NULL          */
    const uint16_t* dist_f16;      /* SoA distance plane, f16               */
    const float* dist_f32;         /* SoA distance plane, f32               */
    const int8_t* dist_u8;         /* SoA distance plane, signed code       */
    const float* brick_scale;      /* per-brick step for dist_u8            */
    const uint16_t* mat_plane;     /* SoA: mat | sec<<6 (u16 per voxel)     */
    const uint8_t* blend_plane;    /* SoA: blend weight                     */
    uint32_t precision;            /* rkf_precision of the SoA plane used   */
    /* index: flat reference brick maps, or two-level */
    const uint32_t* brick_maps;    /* flat packed buffer, may be NULL       */
    const uint32_t* top;           /* two-level: top grid per object       */
    const uint32_t* leaves;        /* two-level: 512 u32 per leaf block     */
    const uint32_t* obj_top_info;  /* per object: top_offset, bdx, bdy, bdz */
    const rkf_gpu_object* objects;
    uint32_t num_objects;
    const double* dist_f64;        /* analytic distances (precision 3)      */
    /* BVH strategy (ray_march_bvh): nodes root first, a tree whose children
     * follow their parent (rkf_bvh_import's rule) */
    const rkf_bvh_node* bvh;
    uint32_t bvh_nodes;
} orc_scene;

/* Distance-plane code for orc_scene.dist_f64. */
#define ORC_PRECISION_F64 3u

/* The scene SDF evaluated in FP64 at the voxel centres of the allocated
 * bricks of a flat brick map (dist[slot*512 + x+8y+64z]): the analytic
 * values a perfect storage format would hold. */
void orc_voxel_values_f64(const rkf_prim* prims, uint32_t n_prims, const rkf_voxelize_params* vp,
                          const uint32_t* map, uint32_t n_slots, double* dist, int threads);
// orc_voxel_values_f64 for n bricks given by their coordinates (bxyz, 3 per
// brick) and pool slots.
void orc_voxel_values_f64_bricks(const rkf_prim* prims, uint32_t n_prims, const rkf_voxelize_params* vp,
                                 const uint32_t* bxyz, const uint32_t* slots, uint64_t n, double* dist,
                                 int threads);

typedef struct orc_stats {
    uint64_t sectors;        /* distinct 32-B sectors, summed over rays     */
    uint64_t index_sectors;
    uint64_t dist_sectors;
    uint64_t mat_sectors;
    uint64_t steps;          /* march iterations, summed                    */
    uint64_t evals;          /* evaluate_object calls, summed               */
} orc_stats;

/* Primary-ray march of a w x h view (ray_march.wgsl:1036-1112).
 * fp64 = 0: FP32-faithful; 1: FP64 same control flow.  Outputs as in
 * rkf_gbuffer (host arrays; optional planes may be NULL).  margin (optional,
 * per ray) receives the smallest distance of any FP decision to its
 * threshold (for grazing flags); t_root (optional, fp64 only) the refined
 * trilinear surface crossing.  When row1 > row0 only rows [row0,row1) are
 * marched and the output arrays hold just those rows. */
void orc_march(const orc_scene* s, const rkf_camera* cam, const rkf_march_params* p,
               uint32_t w, uint32_t h, int fp64, int threads, uint32_t row0, uint32_t row1,
               float* t, float* normal, uint32_t* slot, uint16_t* material, uint16_t* flags,
               float* position, uint32_t* packed, float* motion,
               double* t64, double* normal64, double* margin, double* t_root,
               int count_sectors, orc_stats* stats);

/* Generic ray casts (mode = rkf_trace_mode). */
void orc_trace_rays(const orc_scene* s, const float* origins, const float* dirs,
                    const float* tmax, uint32_t n, uint32_t mode,
                    const rkf_march_params* p, int fp64, int threads,
                    float* t, float* normal, uint32_t* slot, uint16_t* material,
                    uint16_t* flags, double* t64, double* margin);

/* Point queries (SdfQueryable::evaluate/gradient over the brick pool). */
void orc_query_points(const orc_scene* s, const float* points, uint32_t n,
                      float* dist, float* grad, uint16_t* material, int threads);

/* sdf_ao (shade_common_shading.wgsl:37-47) at pos along normal -> ao[n]. */
void orc_sdf_ao(const orc_scene* s, const float* pos, const float* normal, uint32_t n, float* ao,
                int threads);

/* soft_shadow and sdf_ao through the shading pass's own sample_sdf
 * (shade_common.wgsl:521-572: the coarse field beyond 0.5 m, seen from the
 * camera at cam), for bounding how far the library's exact-distance forms
 * move from it. */
void orc_shadow_shader(const orc_scene* s, const float* origins, const float* dirs, const float* tmax, uint32_t n,
                       const float cam[3], int threads, float* shadow);
void orc_sdf_ao_shader(const orc_scene* s, const float* pos, const float* normal, uint32_t n, const float cam[3],
                       int threads, float* ao);

/* CPU CSG edit on one brick (cpu_apply.rs:28-200): rewrites the 1024 words
 * of the brick in place; brick_local_min as find_affected_bricks computes
 * it.  Returns 1 when the brick counts as modified. */
int orc_apply_edit_brick(uint32_t* words, const float brick_local_min[3], float vs,
                         const rkf_edit_op* op);
// The edit on a brick of planes with f32 distances (f32 and u8 pools).
int orc_apply_edit_planes(float* dist, uint16_t* mat, uint8_t* blend, const float bmin[3], float vs,
                          const rkf_edit_op* op);
// Band-normalised u8 code of one brick (the u8 pool's encoding).
void orc_encode_u8(const float* dist, float band, int nearest, int8_t* code, float* step);
/* fill_brick_with_brush_sdf (cpu_apply.rs:204-229). */
void orc_fill_brick_with_brush(uint32_t* words, const float brick_local_min[3], float vs,
                               const rkf_edit_op* op);
float orc_evaluate_falloff(uint32_t curve, float distance, float radius);
float orc_evaluate_shape(uint32_t shape, const float dims[3], const float pos[3]);

/* Reference unit-test helpers (crates/rkf-core/src/sampling.rs:23-66):
 * single-brick trilinear sample of 512 f16 distances at a brick-local pos. */
float orc_sample_brick_trilinear(const uint32_t* words, const float local[3], float vs);

#ifdef __cplusplus
}
#endif
#endif
