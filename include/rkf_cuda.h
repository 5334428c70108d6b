/*
 * rkf_cuda.h — C ABI of the B200 (sm_100a) SDF ray-march engine.
 *
 * This header is the drop-in boundary for the RKIField march path.  Every
 * entry point names the reference interface it replaces (paths are relative
 * to the RKIField workspace root).  The ABI is plain C: POD structs, raw
 * pointers and sizes, status codes; no exceptions or aborts cross it.
 *
 * Ownership: the caller owns every host buffer it passes; a context owns all
 * device memory it allocates.  Output buffers may be host or device pointers
 * (see rkf_mem_kind).  A context is externally synchronised for import, edit
 * and direct march calls; rkf_submit / rkf_poll are thread-safe.
 */
#ifndef RKF_CUDA_H
#define RKF_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RKF_ABI_VERSION 1u

#if defined(__GNUC__)
#define RKF_API __attribute__((visibility("default")))
#else
#define RKF_API
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                             */
/* ------------------------------------------------------------------------ */
typedef enum rkf_status {
    RKF_OK = 0,
    RKF_INVALID_ARG = 1,   /* bad pointer, size, enum or layout            */
    RKF_OOM = 2,           /* device allocation failed / budget exceeded   */
    RKF_CUDA_ERROR = 3,    /* a CUDA runtime call failed                    */
    RKF_TIMEOUT = 4,       /* rkf_poll timed out / bounded device wait hit  */
    RKF_BUSY = 5,          /* admission refused: no slot or memory budget  */
    RKF_EPOCH_STALE = 6,   /* request pinned an epoch that was retired     */
    RKF_NOT_READY = 7,     /* result not complete yet (non-blocking poll)  */
    RKF_UNSUPPORTED = 8,   /* feature not available on this device/build   */
    RKF_CANCELLED = 9      /* request was cancelled before completion      */
} rkf_status;

/* ------------------------------------------------------------------------ */
/* Reference-layout sentinels and constants                                 */
/* crates/rkf-core/src/brick_map.rs:31-37 and ray_march.wgsl:25-48          */
/* ------------------------------------------------------------------------ */
#define RKF_EMPTY_SLOT    0xFFFFFFFFu
#define RKF_INTERIOR_SLOT 0xFFFFFFFEu
#define RKF_BRICK_DIM     8u
#define RKF_BRICK_VOXELS  512u

/* sdf_type / primitive_type / blend_mode of rkf_gpu_object
 * (crates/rkf-render/src/gpu_object.rs:97-125). */
#define RKF_SDF_NONE        0u
#define RKF_SDF_ANALYTICAL  1u
#define RKF_SDF_VOXELIZED   2u
#define RKF_PRIM_SPHERE   0u
#define RKF_PRIM_BOX      1u
#define RKF_PRIM_CAPSULE  2u
#define RKF_PRIM_TORUS    3u
#define RKF_PRIM_CYLINDER 4u
#define RKF_PRIM_PLANE    5u

/* ------------------------------------------------------------------------ */
/* Reference structs, byte-for-byte                                         */
/* ------------------------------------------------------------------------ */

/* CameraUniforms, 144 B (crates/rkf-render/src/camera.rs:196-213).
 * right/up are pre-scaled by tan(fov/2)*aspect and tan(fov/2)
 * (camera.rs:161-184).  prev_vp is column-major. */
typedef struct rkf_camera {
    float position[4];
    float forward[4];
    float right[4];
    float up[4];
    float resolution[2];
    float jitter[2];
    float prev_vp[16];
} rkf_camera;

/* SceneUniforms, 16 B (crates/rkf-render/src/gpu_scene.rs:23-43). */
typedef struct rkf_scene_uniforms {
    uint32_t num_objects;
    uint32_t max_steps;
    float max_distance;
    float hit_threshold;
} rkf_scene_uniforms;

/* GpuObject, 256 B (crates/rkf-render/src/gpu_object.rs:41-95). */
typedef struct rkf_gpu_object {
    float inverse_world[16]; /* column-major mat4 */
    float aabb_min[4];
    float aabb_max[4];
    uint32_t brick_map_offset;
    uint32_t brick_map_dims[3];
    float voxel_size;
    uint32_t material_id;
    uint32_t sdf_type;
    uint32_t blend_mode;
    float blend_radius;
    float sdf_params[4];
    float accumulated_scale[3];
    uint32_t lod_level;
    uint32_t object_id;
    uint32_t primitive_type;
    float geometry_aabb_min[3];
    float geometry_aabb_max[3];
    float _padding[15];
} rkf_gpu_object;

/* ------------------------------------------------------------------------ */
/* March parameters: SceneUniforms plus the shader's compile-time constants */
/* as explicit fields (ray_march.wgsl:28-41).                               */
/* ------------------------------------------------------------------------ */
typedef enum rkf_strategy {
    RKF_STRATEGY_BRUTE = 0,  /* ray_march_brute (:776-858): every object each */
                             /* step, in index order                          */
    RKF_STRATEGY_TILED = 1,  /* ray_march_tiled (:874-985): coarse-field skips */
                             /* and per-16x16-tile object lists; views only;  */
                             /* at most 256 objects (RKF_UNSUPPORTED beyond;  */
                             /* brute and BVH take any count)                 */
    RKF_STRATEGY_BVH = 2     /* ray_march_bvh (:641-773): each step walks the  */
                             /* imported BVH (rkf_bvh_import), skipping nodes */
                             /* farther than the best distance so far; views  */
                             /* and closest/any ray batches                   */
} rkf_strategy;

typedef struct rkf_march_params {
    rkf_scene_uniforms scene;        /* num_objects is filled by the ctx   */
    uint32_t hard_max_steps;         /* HARD_MAX_STEPS = 1024              */
    uint32_t bisect_steps;           /* BISECT_STEPS = 8                   */
    float min_step;                  /* MIN_STEP = 0.0005                  */
    float near_surface_threshold;    /* NEAR_SURFACE_THRESHOLD = 0.02      */
    uint32_t strategy;               /* rkf_strategy (tiled: views only;   */
                                     /* shadow rays march every object)    */
    uint32_t reserved;
} rkf_march_params;

/* Fill p with the reference defaults (gpu_scene.rs:34-43, ray_march.wgsl:28-41). */
RKF_API void rkf_march_params_default(rkf_march_params* p);

/* ------------------------------------------------------------------------ */
/* Context                                                                  */
/* ------------------------------------------------------------------------ */
typedef struct rkf_ctx rkf_ctx;

/* Distance-plane storage precision of the device pool. */
typedef enum rkf_precision {
    RKF_PRECISION_F16 = 0,  /* reference VoxelSample distance (default)     */
    RKF_PRECISION_F32 = 1,  /* full float distances                          */
    RKF_PRECISION_U8 = 2    /* band-normalised u8 with a per-brick scale     */
} rkf_precision;

typedef enum rkf_mem_kind {
    RKF_MEM_HOST = 0,       /* pointers are host memory (pageable or pinned) */
    RKF_MEM_DEVICE = 1      /* pointers are device memory of ctx's device    */
} rkf_mem_kind;

typedef struct rkf_config {
    int device;                     /* CUDA ordinal                          */
    uint32_t pool_capacity_bricks;  /* slots reserved for the brick pool     */
    uint32_t precision;             /* rkf_precision                         */
    uint32_t keep_reference_pool;   /* also keep the AoS VoxelSample pool    */
                                    /* (needed by rkf_march_plain)           */
    uint64_t mem_budget_bytes;      /* serving admission budget, 0 = auto    */
    uint32_t max_inflight;          /* serving slots, 0 = default (64)       */
    float u8_band;                  /* u8 precision: half-width (metres) of  */
                                    /* the distance band the codes cover;    */
                                    /* 0 = 3 voxels for voxelized objects,   */
                                    /* each brick's largest |d| for imports  */
    uint32_t u8_round;              /* u8 precision: 0 = codes round toward  */
                                    /* zero (a decoded |d| never exceeds the */
                                    /* true one), 1 = to nearest (unbiased)  */
    uint32_t reserved[5];
} rkf_config;

RKF_API void rkf_config_default(rkf_config* cfg);

/* Replaces RenderContext + GpuScene construction
 * (crates/rkf-render/src/context.rs:29, gpu_scene.rs:52). */
RKF_API rkf_status rkf_create(const rkf_config* cfg, rkf_ctx** out);
RKF_API rkf_status rkf_destroy(rkf_ctx* ctx);
/* Human-readable message for the last failed call on this thread. */
RKF_API const char* rkf_last_error(void);

/* ------------------------------------------------------------------------ */
/* Scene import (the reference's upload path)                               */
/* ------------------------------------------------------------------------ */

/* Upload reference VoxelSample bricks (2 u32 per voxel, x+8y+64z within a
 * brick) into slots [first_slot, first_slot+n_bricks).
 * Replaces the whole-pool write_buffer of render.rs:106-126 and
 * GpuScene::set_brick_pool (gpu_scene.rs:231). */
RKF_API rkf_status rkf_pool_import_voxelsample(rkf_ctx* ctx, const uint32_t* words,
                                       uint32_t first_slot, uint32_t n_bricks);

/* Upload bricks given as structure-of-arrays planes, 512 voxels per brick in
 * x+8y+64z order: dist_f16 (binary16 bits), mat (material | secondary << 6,
 * 6 bits each) and blend, into slots [first_slot, first_slot+n_bricks).
 * The same content as rkf_pool_import_voxelsample without the 8-byte word
 * packing (VoxelSample::new_blended, voxel.rs:43-54, is how the words hold it). */
RKF_API rkf_status rkf_pool_import_soa(rkf_ctx* ctx, const uint16_t* dist_f16, const uint16_t* mat,
                                       const uint8_t* blend, uint32_t first_slot, uint32_t n_bricks);

/* Upload the packed BrickMapAllocator buffer (brick_map.rs:246 as_slice).
 * Replaces GpuScene::upload_brick_maps (gpu_scene.rs:170). */
RKF_API rkf_status rkf_brickmap_import(rkf_ctx* ctx, const uint32_t* packed, uint64_t n);

/* Upload GpuObject records.  Replaces GpuScene::upload_objects
 * (gpu_scene.rs:141).  Builds the device two-level brick index for every
 * voxelized object from the imported brick maps. */
RKF_API rkf_status rkf_objects_import(rkf_ctx* ctx, const rkf_gpu_object* objects, uint32_t n);

/* Replace the object records and keep the brick index: the per-frame
 * GpuScene::upload_objects of the runtime (render.rs:135-137), where
 * transforms, materials and the set of analytic objects change but the
 * voxelized objects' brick maps do not.  For a voxelized record i,
 * index_source[i] names the current object whose index it uses (same
 * brick_map_dims and voxel_size; NULL: object i's own); other records need
 * no index.  Works on objects made by rkf_voxelize_prims, which have no
 * flat brick map to re-import.  On a refused record nothing changes. */
RKF_API rkf_status rkf_objects_update(rkf_ctx* ctx, const rkf_gpu_object* objects, uint32_t n,
                                      const int32_t* index_source);

/* ------------------------------------------------------------------------ */
/* Object records from a node tree: transform flattening                    */
/* (crates/rkf-core/src/transform_flatten.rs:23-110 and                     */
/* crates/rkf-render/src/gpu_object.rs:135-266).  Host only.                */
/* ------------------------------------------------------------------------ */
#define RKF_NO_PARENT 0xFFFFFFFFu
/* blend_mode of rkf_gpu_object and rkf_scene_node (gpu_object.rs:123-133) */
#define RKF_BLEND_SMOOTH_UNION 0u
#define RKF_BLEND_UNION        1u
#define RKF_BLEND_SUBTRACT     2u
#define RKF_BLEND_INTERSECT    3u

/* One node of an object's tree (SceneNode, scene_node.rs): its local
 * transform (Transform::to_matrix = scale, then rotation, then translation),
 * whether it is visible (NodeMetadata::visible, scene_node.rs:178), how it blends with its
 * siblings and its SDF source.  A tree is passed in depth-first pre-order --
 * a node, then the subtree of each child in order -- each node naming its
 * parent's index (RKF_NO_PARENT for the root, which comes first). */
typedef struct rkf_scene_node {
    float position[3];
    float rotation[4];         /* quaternion x, y, z, w, used as given        */
    float scale[3];
    uint32_t parent;
    uint32_t visible;          /* 0: the node and its subtree are left out   */
                               /* (the root is always kept)                   */
    uint32_t sdf_type;         /* RKF_SDF_NONE / ANALYTICAL / VOXELIZED       */
    uint32_t primitive_type;   /* analytical: RKF_PRIM_*                      */
    float params[4];           /* analytical: primitive_params order          */
    uint32_t material_id;      /* analytical                                  */
    uint32_t brick_map_offset; /* voxelized: BrickMapHandle                   */
    uint32_t brick_map_dims[3];
    float voxel_size;          /* voxelized                                   */
    uint32_t blend_mode;       /* RKF_BLEND_*                                 */
    float blend_radius;        /* smooth union only                           */
} rkf_scene_node;

/* FlatNode (transform_flatten.rs:23-38) with the index of its source node. */
typedef struct rkf_flat_node {
    float inverse_world[16];   /* column-major                                */
    float accumulated_scale[3];
    uint32_t depth;            /* 0 for the root                              */
    uint32_t parent_index;     /* in the flat array; RKF_NO_PARENT: root      */
    uint32_t node;             /* the rkf_scene_node it came from             */
} rkf_flat_node;

/* flatten_object (transform_flatten.rs:56-110): walks the tree depth-first with
 * world = parent world * local, starting from the object's own transform
 * (object_scale, object_rotation, then world_position: the object's baked
 * world-space, or camera-relative, position), and writes one flat node per
 * visible node in pre-order, with the inverse of its world matrix and the
 * product of the scales from the object down to it.  The products and the
 * inverse are computed in double precision and rounded to float once.
 * out holds n_nodes entries; *n_out receives the count written.
 * RKF_INVALID_ARG for a tree not in pre-order, a parent index out of range or
 * a singular world matrix. */
RKF_API rkf_status rkf_flatten_object(const rkf_scene_node* nodes, uint32_t n_nodes,
                                      const float object_rotation[4], const float object_scale[3],
                                      const float world_position[3], rkf_flat_node* out, uint32_t* n_out);

/* GpuObject::from_flat_node (gpu_object.rs:141-220, 233-266): the record of a flat
 * node whose source is `source`; analytic sources keep their primitive type,
 * parameters and material, voxelized ones their brick map handle and voxel
 * size, and a smooth union its radius (other modes get 0). */
RKF_API rkf_status rkf_gpu_object_from_flat_node(const rkf_flat_node* flat, const rkf_scene_node* source,
                                                 uint32_t object_id, const float aabb_min[4],
                                                 const float aabb_max[4], const float geometry_aabb_min[3],
                                                 const float geometry_aabb_max[3], rkf_gpu_object* out);

/* One BVH node as the shader reads it (GpuBvhNode, gpu_bvh.rs:24-41;
 * BvhNode, ray_march.wgsl:99-108): 32 bytes. */
#define RKF_BVH_INVALID 0xFFFFFFFFu
typedef struct rkf_bvh_node {
    float aabb_min[3];
    uint32_t left;             /* left child, or RKF_BVH_INVALID for a leaf  */
    float aabb_max[3];
    uint32_t right_or_object;  /* right child (internal) or object index     */
} rkf_bvh_node;

/* Upload BVH nodes, root first.  Replaces GpuScene::upload_bvh
 * (gpu_scene.rs:186).  The nodes must form one tree: every internal node
 * names two children with larger indices than its own, and every node but
 * the root is named exactly once (Bvh::build, bvh.rs:66-260, lays nodes out
 * this way); anything else returns RKF_INVALID_ARG and keeps the previous
 * BVH.  Leaves may name any object index: the march skips indices at or
 * beyond the object count, as the shader does.  n = 0 removes the BVH.  At
 * most 65,536 nodes. */
RKF_API rkf_status rkf_bvh_import(rkf_ctx* ctx, const rkf_bvh_node* nodes, uint32_t n);

/* Object AABB for rkf_bvh_build: the (object_id, aabb) pairs of
 * Bvh::build (bvh.rs:66). */
typedef struct rkf_bvh_item {
    uint32_t object_index;
    float aabb_min[3];
    float aabb_max[3];
} rkf_bvh_item;

/* Host-side BVH build with the reference's surface-area heuristic
 * (Bvh::build, bvh.rs:66-260, converted by GpuBvhNode::from_cpu,
 * gpu_bvh.rs:45-60): one object per leaf, 2n-1 nodes for n >= 1 items,
 * 0 for n = 0.  Writes *n_out nodes to out (cap entries available; too few
 * returns RKF_INVALID_ARG).  Needs no context or device. */
RKF_API rkf_status rkf_bvh_build(const rkf_bvh_item* items, uint32_t n, rkf_bvh_node* out, uint32_t cap,
                                 uint32_t* n_out);

/* Counts of what the context holds. */
typedef struct rkf_scene_info {
    uint32_t num_objects;
    uint32_t pool_bricks_used;
    uint32_t pool_capacity;
    uint32_t leaf_blocks;
    uint64_t device_bytes;
    uint64_t epoch;
} rkf_scene_info;
RKF_API rkf_status rkf_scene_info_get(rkf_ctx* ctx, rkf_scene_info* out);

/* Download n_bricks of the device pool as reference VoxelSample words
 * (inverse of rkf_pool_import_voxelsample; used to cross-check). */
RKF_API rkf_status rkf_pool_export_voxelsample(rkf_ctx* ctx, uint32_t first_slot,
                                       uint32_t n_bricks, uint32_t* words);
/* Download n_bricks of the structure-of-arrays planes: distances at the
 * context precision (f16: u16 bits, f32: float, u8: int8 codes; 512 per
 * brick), the u8 per-brick step (u8 precision only, may be NULL), material
 * (mat | secondary<<6) and blend planes (may be NULL).  No reference
 * counterpart (the reference pool is AoS); used to cross-check. */
RKF_API rkf_status rkf_pool_export_planes(rkf_ctx* ctx, uint32_t first_slot, uint32_t n_bricks,
                                          void* dist, float* step, uint16_t* mat, uint8_t* blend);

/* Copy the device brick index out: the top grids (8^3-brick blocks: EMPTY,
 * INTERIOR or a leaf number), the 512-entry leaves, and per object
 * {top offset, top dims x, y, z}.  No reference counterpart (the reference
 * keeps only flat maps); used to cross-check the device index.  Pass NULL
 * arrays to query the sizes. */
RKF_API rkf_status rkf_index_export(rkf_ctx* ctx, uint32_t* top, uint64_t* top_n,
                                    uint32_t* leaves, uint64_t* leaf_entries,
                                    uint32_t* obj_top_info, uint32_t* n_objects);
/* Look up the slot (or sentinel) of brick (bx,by,bz) of object obj. */
RKF_API rkf_status rkf_brick_lookup(rkf_ctx* ctx, uint32_t obj, const uint32_t* bxyz,
                            uint32_t n, uint32_t* slots);

/* ------------------------------------------------------------------------ */
/* Seeded synthetic scenes built on the device                              */
/* ------------------------------------------------------------------------ */

/* One analytic primitive of a seeded synthetic scene (object-local metres).
 * type: RKF_PRIM_SPHERE / BOX / CAPSULE.  rot is row-major R with
 * local = R^T (p - centre).  params: sphere r; box hx,hy,hz; capsule r,h. */
typedef struct rkf_prim {
    uint32_t type;
    uint32_t material;
    float centre[3];
    float params[3];
    float rot[9];
    float bound_radius;
} rkf_prim;

/* Band rule used to decide which bricks are allocated. */
typedef enum rkf_band_rule {
    RKF_BAND_VOXELS = 0,   /* any voxel |d| <= band_voxels*vs; deep interior  */
                           /* bricks become INTERIOR_SLOT                     */
    RKF_BAND_REFERENCE = 1 /* voxelize_object.rs:86-109: |d(centre)| < 1.8 *  */
                           /* brick extent, everything else EMPTY_SLOT        */
} rkf_band_rule;

typedef struct rkf_voxelize_params {
    float voxel_size;       /* metres                                         */
    float smooth_k;         /* smooth-min radius (sdf.rs:48)                  */
    float band_voxels;      /* narrow band half-width in voxels (3)           */
    float cut_distance;     /* prims with |p-c|-bound >= cut are ignored      */
    float aabb_min[3];      /* local-space AABB to voxelize                   */
    float aabb_max[3];
    uint32_t band_rule;     /* rkf_band_rule                                  */
    uint32_t object_id;
} rkf_voxelize_params;

/* Voxelize the smooth union of prims into the device pool as one object
 * (voxelize_sdf, crates/rkf-core/src/voxelize_object.rs:53-182), appending a
 * GpuObject with identity transform.  Output slot order is the reference's
 * z,y,x brick loop order starting at the pool's first free slot. */
RKF_API rkf_status rkf_voxelize_prims(rkf_ctx* ctx, const rkf_prim* prims, uint32_t n_prims,
                              const rkf_voxelize_params* vp, uint32_t* out_object_index);

/* Fetch object record i as the device holds it. */
RKF_API rkf_status rkf_object_get(rkf_ctx* ctx, uint32_t i, rkf_gpu_object* out);

/* ------------------------------------------------------------------------ */
/* G-buffer march (replaces RayMarchPass::dispatch, ray_march.rs:96-118)     */
/* ------------------------------------------------------------------------ */

/* Per-ray flags written to rkf_gbuffer.flags */
#define RKF_FLAG_HIT       0x1u
#define RKF_FLAG_BISECTED  0x2u   /* hit found by the overstep bisection    */
#define RKF_FLAG_STEPS_OUT 0x4u   /* ended by the near-step or hard budget  */

/* SoA G-buffer.  Required planes: t, normal (3 floats per ray), slot,
 * material, flags.  Optional reference-format planes (may be NULL):
 * position = hit_pos.xyz + t (ray_march.wgsl:1091), packed_material
 * (:1087-1090), motion = motion.xy, 1, sdf_at_hit (:1095-1105). */
typedef struct rkf_gbuffer {
    float* t;
    float* normal;
    uint32_t* slot;
    uint16_t* material;
    uint16_t* flags;
    float* position;
    uint32_t* packed_material;
    float* motion;
    uint32_t mem;            /* rkf_mem_kind of every pointer above          */
    uint32_t _pad;
} rkf_gbuffer;

/* The B200 march: SoA distance plane at the context precision, two-level
 * brick index with empty-brick read skipping, warp-compacted persistent
 * kernel.  Bit-identical results to the reference algorithm in FP32.  With
 * host outputs, a view of 256K rays or more (brute and BVH strategies) in
 * page-locked host planes is marched in bands of rows whose copies to the
 * host overlap the next band's march; the call returns once every output is
 * written. */
RKF_API rkf_status rkf_march(rkf_ctx* ctx, const rkf_camera* cam, const rkf_march_params* p,
                     uint32_t width, uint32_t height, rkf_gbuffer* out);

/* The plain march: one launch, one thread per ray, reference AoS pool and
 * the reference loop order.  The baseline the batched path is measured
 * against. */
RKF_API rkf_status rkf_march_plain(rkf_ctx* ctx, const rkf_camera* cam, const rkf_march_params* p,
                           uint32_t width, uint32_t height, rkf_gbuffer* out);

/* Enqueue a march on a caller stream without waiting for it: the analogue
 * of recording RayMarchPass::dispatch into a wgpu command encoder
 * (ray_march.rs:96).  Device-pointer G-buffers only.  `stream` is a
 * cudaStream_t of the context's device (NULL = the context stream).  Calls
 * on one context share its launch scratch: issue them on one stream, or
 * synchronise between streams. */
RKF_API rkf_status rkf_march_async(rkf_ctx* ctx, const rkf_camera* cam, const rkf_march_params* p,
                                   uint32_t width, uint32_t height, const rkf_gbuffer* out,
                                   void* stream);
RKF_API rkf_status rkf_march_plain_async(rkf_ctx* ctx, const rkf_camera* cam,
                                         const rkf_march_params* p, uint32_t width,
                                         uint32_t height, const rkf_gbuffer* out, void* stream);

/* ------------------------------------------------------------------------ */
/* Generic ray casts (secondary rays; shade_common_shading.wgsl:9-47)        */
/* ------------------------------------------------------------------------ */
typedef enum rkf_trace_mode {
    RKF_TRACE_CLOSEST = 0,  /* full march: t, normal, material, slot          */
    RKF_TRACE_ANY = 1,      /* any-hit: stop at the first surface (no bisect) */
    RKF_TRACE_SHADOW = 2    /* soft_shadow (shade_common_shading.wgsl:9-33)   */
} rkf_trace_mode;

typedef struct rkf_hits {
    float* t;          /* closest/any: hit t or MAX_FLOAT; shadow: factor    */
    float* normal;     /* closest only (may be NULL)                         */
    uint32_t* slot;    /* closest only (may be NULL)                         */
    uint16_t* material;/* closest only (may be NULL)                         */
    uint16_t* flags;   /* may be NULL                                        */
    uint32_t mem;
    uint32_t _pad;
} rkf_hits;

/* Rays: origins[3n], dirs[3n], tmax[n] (per-ray max_distance), mem kind of
 * the inputs = in_mem. */
RKF_API rkf_status rkf_trace_rays(rkf_ctx* ctx, const float* origins, const float* dirs,
                          const float* tmax, uint32_t n, uint32_t mode,
                          const rkf_march_params* p, uint32_t in_mem, rkf_hits* out);

/* Shadow and ambient-occlusion rays for the hit pixels of a view, as the
 * reference's shading pass queries them (shade_common_shading.wgsl:9-47):
 * per pixel n_lights (<= 16) soft-shadow rays towards the point lights
 * (origin = hit + normal*0.08, tmax = distance to the light) and ao_per_hit
 * cosine-weighted hemisphere any-hit rays (origin = hit + normal*0.02,
 * tmax = ao_radius).  Pixel p owns ray slots [p*n, p*n+n); pixels that missed
 * get tmax = -1 (the ray ends on its first iteration).  gb: the view's device
 * G-buffer; lights: host, 3 floats each; outputs: device arrays sized for
 * w*h*n_lights / w*h*ao_per_hit rays.  *hit_pixels (host) receives the
 * number of hit pixels.  Waits for completion. */
RKF_API rkf_status rkf_secondary_rays(rkf_ctx* ctx, const rkf_camera* cam, uint32_t w, uint32_t h,
                                      const rkf_gbuffer* gb, const float* lights,
                                      uint32_t n_lights, uint32_t ao_per_hit, float ao_radius,
                                      uint32_t seed, float* shadow_o, float* shadow_d,
                                      float* shadow_tmax, float* ao_o, float* ao_d,
                                      float* ao_tmax, uint32_t* hit_pixels, void* stream);

/* ------------------------------------------------------------------------ */
/* Point queries: SdfQueryable::{evaluate, gradient}                         */
/* (crates/rkf-physics/src/sdf_collision.rs:38-56)                          */
/* ------------------------------------------------------------------------ */
/* points[3n] -> dist[n] (min over objects, evaluate_object), grad[3n] (unit
 * normal of the closest object, compute_normal_for_object; may be NULL),
 * material[n] (may be NULL).  mem applies to all pointers. */
RKF_API rkf_status rkf_query_points(rkf_ctx* ctx, const float* points, uint32_t n,
                            float* dist, float* grad, uint16_t* material, uint32_t mem);

/* Ambient occlusion: sdf_ao (shade_common_shading.wgsl:37-47) at pos[3n]
 * along normal[3n] (4 taps 0.12 m apart through sample_sdf, strength 0.7)
 * -> ao[n] in [0, 1].  The shading pass calls it at world_pos + normal *
 * SHADOW_BIAS (0.08, shade_main.wgsl:186).  mem applies to all pointers. */
RKF_API rkf_status rkf_sdf_ao(rkf_ctx* ctx, const float* pos, const float* normal, uint32_t n,
                              float* ao, uint32_t mem);

/* ------------------------------------------------------------------------ */
/* CSG edits (crates/rkf-edit/src/edit_op.rs:15, cpu_apply.rs:28-229)       */
/* ------------------------------------------------------------------------ */
typedef struct rkf_edit_op {
    uint32_t object_index;   /* index into the object table                  */
    uint32_t edit_type;      /* EditType: 0 union 1 subtract 2 intersect     */
                             /* 3 smooth union 4 smooth subtract 5 smooth    */
                             /* brush 6 flatten 7 paint (8 color paint:      */
                             /* RKF_UNSUPPORTED, no companion color pool)    */
    uint32_t shape_type;     /* ShapeType: 0 sphere 1 box 2 capsule          */
    uint32_t falloff;        /* FalloffCurve: 0 linear 1 smooth 2 sharp      */
    float position[3];       /* object-local                                 */
    float rotation[4];       /* quaternion x,y,z,w                           */
    float dimensions[3];
    float strength;
    float blend_k;
    uint32_t material_id;
    uint32_t _pad[2];
} rkf_edit_op;

/* Apply one edit on the device: touched allocated bricks are rewritten into
 * fresh slots (copy-on-write), EMPTY (union, smooth union) or INTERIOR
 * (subtract, intersect, smooth subtract) bricks the brush reaches are
 * allocated and filled, and a new index epoch is published.  The smooth
 * brush, flatten and paint act on allocated bricks only, as
 * find_affected_bricks (edit_op.rs:97-141) hands them to apply_edit_cpu.
 * Requests admitted before the call keep reading the previous epoch. */
RKF_API rkf_status rkf_edit_csg(rkf_ctx* ctx, const rkf_edit_op* op, uint64_t* new_epoch);

/* ------------------------------------------------------------------------ */
/* Batched march: many views and ray batches in one persistent launch       */
/* ------------------------------------------------------------------------ */
typedef struct rkf_view {
    rkf_camera camera;
    uint32_t width, height;
    rkf_gbuffer out;         /* device pointers only                         */
} rkf_view;

typedef struct rkf_ray_batch {
    const float* origins;    /* device pointers only                         */
    const float* dirs;
    const float* tmax;
    uint32_t n;
    uint32_t mode;           /* rkf_trace_mode                               */
    rkf_hits out;            /* device pointers only                         */
} rkf_ray_batch;

typedef struct rkf_batch_tuning {
    uint32_t tile_w, tile_h;     /* ray-tile shape of a work item            */
    uint32_t step_budget;        /* empty-space steps a lane runs before its */
                                 /* warp re-converges (0 = 32)               */
    uint32_t compact_interval;   /* march iterations between lane refills;   */
                                 /* a warp also refills once refill_idle of  */
                                 /* its lanes are done (0 = 64)              */
    uint32_t blocks_per_sm;
    uint32_t threads_per_block;
    uint32_t refill_idle;        /* a warp leaves the march loop to refill   */
                                 /* once this many of its lanes are idle     */
                                 /* (0 = 32: only when all are idle)         */
    uint32_t probe_in_run;       /* 1: a lane whose EMPTY cube ends probes   */
                                 /* the next one inside the run (0: at the   */
                                 /* run's end, with the warp's other lanes)  */
    uint32_t no_empty_path;      /* 1: march every step through the full     */
                                 /* sampler (0: EMPTY runs wherever the      */
                                 /* scene allows them).  rkf_march,          */
                                 /* rkf_march_batch and rkf_trace_rays only; */
                                 /* the outputs are the same either way      */
    uint32_t order_tiles;        /* 1: hand out each view's ray tiles        */
                                 /* heaviest first, by an estimate of their  */
                                 /* empty-space steps (0: row order); the    */
                                 /* outputs are the same either way          */
    uint32_t tail_share;         /* once a warp has no work left to fetch    */
                                 /* and at most this many of its lanes still */
                                 /* march (1..32), the warp's 32 lanes take  */
                                 /* those lanes' EMPTY runs together, one    */
                                 /* run at a time, up to 32 steps a round;   */
                                 /* 0: off.  Single-object empty-space path; */
                                 /* the outputs are the same either way      */
} rkf_batch_tuning;

/* Run every view and ray batch in one persistent work-stealing launch.
 * tuning may be NULL (autotuned defaults).  Blocks until complete. */
RKF_API rkf_status rkf_march_batch(rkf_ctx* ctx, const rkf_view* views, uint32_t n_views,
                           const rkf_ray_batch* batches, uint32_t n_batches,
                           const rkf_march_params* p, const rkf_batch_tuning* tuning);

/* rkf_march_batch enqueued on a caller stream (cudaStream_t, NULL = context
 * stream) without waiting.  Shares the context's launch scratch with the
 * other context launches: issue them on one stream or synchronise. */
RKF_API rkf_status rkf_march_batch_async(rkf_ctx* ctx, const rkf_view* views, uint32_t n_views,
                                         const rkf_ray_batch* batches, uint32_t n_batches,
                                         const rkf_march_params* p,
                                         const rkf_batch_tuning* tuning, void* stream);

/* Plain ray casts: one launch per request, one thread per ray, reference
 * AoS pool and flat maps, the reference loop (ray_march.wgsl:776-858,
 * shade_common_shading.wgsl:9-33).  The per-request baseline of the
 * batched path.  Device pointers; enqueued on `stream` without waiting. */
RKF_API rkf_status rkf_trace_rays_plain_async(rkf_ctx* ctx, const float* origins,
                                              const float* dirs, const float* tmax, uint32_t n,
                                              uint32_t mode, const rkf_march_params* p,
                                              const rkf_hits* out, void* stream);

/* rkf_march_batch for callers that cannot allocate device memory when they
 * call: callers on a fixed per-frame time budget (cudaMalloc synchronises
 * the device) and callers whose framework owns every device allocation.  No
 * counterpart in the reference (its march allocates nothing per dispatch).
 *
 * Same inputs, outputs and results as rkf_march_batch for the brute
 * strategy (device pointers only; the tiled and BVH strategies return
 * RKF_UNSUPPORTED), but it allocates nothing: the launch scratch (segment
 * table and work counter) is one fixed static device array of
 * RKF_NOALLOC_MAX_SEGMENTS segments (about 17 KB, held on every device that
 * loads the library until the process exits).  More views plus ray batches
 * than that in one call returns RKF_INVALID_ARG.  The first call on a device
 * resolves the array's device address; make that first call before any
 * stream capture.  The segment table travels as the parameter of a small
 * staging kernel, so the call enqueues two kernels on `stream` (a
 * cudaStream_t, NULL = the context stream) and returns without waiting on
 * it.  Refusals (sizes, strategy, tuning) come before anything is enqueued.
 * Every call shares the one array and the counter is cleared at the start
 * of each call, so calls that overlap on the GPU (other streams, other
 * contexts on the same device) race: order them on one stream or
 * synchronise between them. */
#define RKF_NOALLOC_MAX_SEGMENTS 64u
RKF_API rkf_status rkf_march_batch_noalloc(rkf_ctx* ctx, const rkf_view* views, uint32_t n_views,
                                           const rkf_ray_batch* batches, uint32_t n_batches,
                                           const rkf_march_params* p,
                                           const rkf_batch_tuning* tuning, void* stream);

/* Search tile shape x step budget x compaction interval (and the other
 * knobs of rkf_batch_tuning) on a sample of the given work and store the
 * winner in the context.  Writes it to *out. */
RKF_API rkf_status rkf_autotune(rkf_ctx* ctx, const rkf_view* views, uint32_t n_views,
                        const rkf_ray_batch* batches, uint32_t n_batches,
                        const rkf_march_params* p, rkf_batch_tuning* out);
/* The tuning the context's marches use when none is given (rkf_march,
 * rkf_march_async, rkf_trace_rays, the serving loop): set one found earlier
 * (a tuning never changes results), or read the current one. */
RKF_API rkf_status rkf_tuning_set(rkf_ctx* ctx, const rkf_batch_tuning* tuning);
RKF_API rkf_status rkf_tuning_get(rkf_ctx* ctx, rkf_batch_tuning* out);

/* ------------------------------------------------------------------------ */
/* A batched march captured as a CUDA graph (no counterpart in the          */
/* reference, which records its passes into a wgpu command encoder)         */
/* ------------------------------------------------------------------------ */
/* For work that repeats every frame with the same sizes and output buffers:
 * rkf_batch_graph_create captures one rkf_march_batch of these views and ray
 * batches (device outputs, brute strategy) into a CUDA graph -- the segment
 * table's copy from page-locked memory the graph owns, the work counter's
 * reset, the persistent march kernel -- and rkf_batch_graph_launch replays it
 * on a stream (NULL = the context stream).  rkf_batch_graph_set_cameras
 * gives the views new cameras for the next launch (one per view given at
 * creation, in order; it waits for the previous launch to finish).  The graph
 * holds the scene as it was when made: after an object import, a
 * voxelization or an edit, rkf_batch_graph_launch returns RKF_EPOCH_STALE and
 * the caller makes a new graph.  Destroy graphs before their context. */
typedef struct rkf_batch_graph rkf_batch_graph;
RKF_API rkf_status rkf_batch_graph_create(rkf_ctx* ctx, const rkf_view* views, uint32_t n_views,
                                          const rkf_ray_batch* batches, uint32_t n_batches,
                                          const rkf_march_params* p, const rkf_batch_tuning* tuning,
                                          rkf_batch_graph** out);
RKF_API rkf_status rkf_batch_graph_set_cameras(rkf_batch_graph* graph, const rkf_camera* cameras, uint32_t n);
RKF_API rkf_status rkf_batch_graph_launch(rkf_batch_graph* graph, void* stream);
RKF_API rkf_status rkf_batch_graph_destroy(rkf_batch_graph* graph);

/* ------------------------------------------------------------------------ */
/* Serving: resident request loop with continuous batching                  */
/* ------------------------------------------------------------------------ */
typedef enum rkf_request_kind {
    RKF_REQ_RENDER = 0,   /* camera render -> G-buffer                       */
    RKF_REQ_RAYS = 1,     /* ray batch -> hits                               */
    RKF_REQ_POINTS = 2,   /* point queries -> distance/gradient/material     */
    RKF_REQ_EDIT = 3      /* CSG edit (ordered w.r.t. later admissions)      */
} rkf_request_kind;

typedef struct rkf_request {
    uint32_t kind;
    uint32_t mode;             /* rays: rkf_trace_mode                        */
    uint32_t width, height;    /* render                                      */
    uint32_t n;                /* rays / points                               */
    uint32_t _pad;
    rkf_camera camera;         /* render                                      */
    const float* in0;          /* rays: origins | points: xyz  (host)         */
    const float* in1;          /* rays: dirs                    (host)        */
    const float* in2;          /* rays: tmax                    (host)        */
    rkf_edit_op edit;          /* edit                                        */
    /* host outputs (caller-owned, must stay valid until the result is polled) */
    float* out_t;              /* render/rays: t; points: dist                */
    float* out_normal;         /* render/rays/points: 3 floats per item       */
    uint32_t* out_slot;
    uint16_t* out_material;
    uint16_t* out_flags;
} rkf_request;

typedef uint64_t rkf_ticket;

typedef struct rkf_result {
    rkf_status status;
    uint32_t kind;
    uint64_t epoch;            /* index epoch the request read               */
    double submit_us;          /* host clock at admission                    */
    double start_us;           /* host clock when its work was issued        */
    double done_us;            /* host clock when its result was complete    */
    double device_ms;          /* device time of its share of the work       */
} rkf_result;

/* Start / stop the resident serving loop (a host thread + streams). */
RKF_API rkf_status rkf_serve_start(rkf_ctx* ctx, const rkf_march_params* p);
RKF_API rkf_status rkf_serve_stop(rkf_ctx* ctx);
/* Admit a request.  RKF_BUSY when no slot or memory budget is free. */
RKF_API rkf_status rkf_submit(rkf_ctx* ctx, const rkf_request* req, rkf_ticket* ticket);
/* Wait up to timeout_us for a ticket.  RKF_NOT_READY if still running. */
RKF_API rkf_status rkf_poll(rkf_ctx* ctx, rkf_ticket ticket, rkf_result* out, uint32_t timeout_us);
RKF_API rkf_status rkf_cancel(rkf_ctx* ctx, rkf_ticket ticket);

/* ------------------------------------------------------------------------ */
/* FP64 rebasing (crates/rkf-core/src/world_position.rs:107-120)            */
/* ------------------------------------------------------------------------ */
typedef struct rkf_world_pos {
    int32_t chunk[3];
    float local[3];
} rkf_world_pos;

/* out = (float)(pos - origin) computed in FP64 (relative_to_f64). */
RKF_API void rkf_world_relative(const rkf_world_pos* pos, const rkf_world_pos* origin,
                        double out_f64[3], float out_f32[3]);

/* The WorldPosition that the scene's f32 world-space coordinates (object
 * transforms and grids) are relative to; chunk (0,0,0) and local (0,0,0)
 * until set.  A world far from the origin (chunks beyond what f32 metres
 * resolve) is uploaded relative to a nearby origin, and cameras and ray
 * origins given as WorldPositions are rebased against it in FP64 on the host
 * (WorldPosition::relative_to_f64, world_position.rs:107-120; the render
 * path's camera-relative positions, transform_flatten.rs:8-12) and rounded
 * to f32 once, before the f32 march.  Not while serving. */
RKF_API rkf_status rkf_scene_origin_set(rkf_ctx* ctx, const rkf_world_pos* origin);
RKF_API rkf_status rkf_scene_origin_get(rkf_ctx* ctx, rkf_world_pos* out);

/* rkf_march with the camera at a WorldPosition: the march uses cam with
 * its position replaced by the f32 rounding of relative_to_f64(cam_pos,
 * scene origin). */
RKF_API rkf_status rkf_march_world(rkf_ctx* ctx, const rkf_world_pos* cam_pos, const rkf_camera* cam,
                                   const rkf_march_params* p, uint32_t width, uint32_t height,
                                   rkf_gbuffer* out);

/* rkf_trace_rays with ray origins as WorldPositions (host arrays: origins[n],
 * dirs[3n], tmax[n]), each rebased against the scene origin in FP64 and
 * rounded to f32 once. */
RKF_API rkf_status rkf_trace_rays_world(rkf_ctx* ctx, const rkf_world_pos* origins, const float* dirs,
                                        const float* tmax, uint32_t n, uint32_t mode,
                                        const rkf_march_params* p, rkf_hits* out);

#ifdef __cplusplus
}
#endif
#endif /* RKF_CUDA_H */
