/*
 * tpt.h — C ABI of libtpt_cuda.so, the B200 (sm_100a) implementation of the
 * per-sample rendering hot path of the toy-path-tracing renderer.
 *
 * Every entry point replaces one operation of the reference Rust crate
 * `crates/renderer` (paths below are relative to that crate's src/ directory):
 * the C ABI is what a feature-gated `gpu` module of that crate binds with
 * `extern "C"`.
 *
 * Conventions
 *  - Every function returns a tpt_status; TPT_OK is 0.  No exception, abort or
 *    Rust panic crosses the boundary.  tpt_last_error() gives a message.
 *  - Host buffers passed in are owned by the caller and only read (or written)
 *    during the call.  Device allocations belong to a tpt_context / tpt_scene
 *    handle and are freed by the matching *_destroy / *_release call.
 *  - `*_device` variants take device pointers and a cudaStream_t (as void*,
 *    NULL = the context's stream); they are asynchronous on that stream.
 *  - Calls on one context must be serialised by the caller; contexts are
 *    independent.  There is no CPU fallback: without a usable CUDA device
 *    tpt_context_create fails with TPT_ERR_CUDA.
 *  - Vectors are float triples; matrices are column-major 4x4 (glam::Mat4
 *    layout) or 3x3 (glam::Mat3).
 */
#ifndef TPT_H_
#define TPT_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tpt_status {
  TPT_OK = 0,
  TPT_ERR_INVALID_ARG = 1,
  TPT_ERR_OUT_OF_MEMORY = 2,
  TPT_ERR_CUDA = 3,
  TPT_ERR_CAPACITY = 4,     /* a fixed-size device structure would overflow */
  TPT_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up */
  TPT_ERR_DEVICE_CHECK = 6, /* a device-side bounds/consistency check fired */
  TPT_ERR_NOT_BUILT = 7     /* acceleration structure missing (ClosestHitError::QbvhNotBuilt) */
} tpt_status;

typedef struct tpt_context tpt_context;
typedef struct tpt_scene tpt_scene;
typedef struct tpt_qbvh tpt_qbvh;

/* ------------------------------------------------------------------------ */
/* Context                                                                   */

/* Binds a context to CUDA device `device` and creates its stream. */
tpt_status tpt_context_create(int device, tpt_context** out);
tpt_status tpt_context_destroy(tpt_context* ctx);
/* Message of the last failed call on `ctx` (or of the last failed context-less
 * call when ctx is NULL).  Valid until the next call on the same context. */
const char* tpt_last_error(const tpt_context* ctx);
/* Library version string. */
const char* tpt_version(void);

/* ------------------------------------------------------------------------ */
/* QBVH (qbvh.rs)                                                             */

/* One 4-wide node, 128 bytes: lanes of min_x, min_y, min_z, max_x, max_y,
 * max_z, then the four child words (qbvh.rs:15-51 encoding: bit 31 = leaf,
 * bits 24..30 = primitive count, bits 0..23 = primitive offset; interior
 * children are node indices; 0x80000000 = empty) and the valid-lane mask.
 * Mirrors `QbvhNode` (qbvh.rs:53-63). */
typedef struct tpt_qbvh_node {
  float bounds[6][4];
  uint32_t children[4];
  uint32_t valid_mask;
  uint32_t reserved[3];
} tpt_qbvh_node;

/* A built QBVH: `Qbvh { nodes, primitive_indices }` (qbvh.rs:131-135).
 * num_nodes == 0 with num_primitives > 0 means the root is a single leaf. */
typedef struct tpt_qbvh_view {
  const tpt_qbvh_node* nodes;
  uint64_t num_nodes;
  const uint32_t* primitive_indices;
  uint64_t num_primitives;
} tpt_qbvh_view;

/* Host-side binned-SAH builder; replaces `build_qbvh` (qbvh.rs:144-172).
 * bounds: n x 6 floats (min xyz, max xyz).  threads <= 0 uses all cores.
 * Fails with TPT_ERR_INVALID_ARG for n == 0 (the reference returns None). */
tpt_status tpt_qbvh_build(const float* bounds, uint64_t n, int threads, tpt_qbvh** out);
tpt_status tpt_qbvh_view_of(const tpt_qbvh* q, tpt_qbvh_view* view);
tpt_status tpt_qbvh_free(tpt_qbvh* q);

/* ------------------------------------------------------------------------ */
/* Scene upload (scene/mod.rs `Scene`)                                       */

typedef struct tpt_mesh_desc {
  const float* positions; /* num_vertices x 3 */
  const float* normals;   /* num_vertices x 3, may be NULL (zero normals) */
  const float* uvs;       /* num_vertices x 2, may be NULL (zero uvs) */
  uint64_t num_vertices;
  const uint32_t* indices; /* num_indices, a multiple of 3 */
  uint64_t num_indices;
  /* Pre-built BLAS (`Mesh::qbvh`, mesh.rs:114-119).  Leave nodes and
   * primitive_indices NULL to have tpt_scene_upload build it on the host. */
  tpt_qbvh_view qbvh;
} tpt_mesh_desc;

typedef struct tpt_instance_desc {
  uint32_t mesh_index;
  uint32_t material_index;
  float local_to_world[16];
  float world_to_local[16];
  float normal_to_world[9];
} tpt_instance_desc;

typedef struct tpt_scene_desc {
  const tpt_mesh_desc* meshes;
  uint32_t num_meshes;
  const tpt_instance_desc* instances;
  uint32_t num_instances;
  /* Pre-built TLAS over instance world bounds (`Scene::qbvh`, scene/mod.rs:305-317);
   * NULL arrays = build on upload. */
  tpt_qbvh_view tlas;
} tpt_scene_desc;

/* Copies the scene into device memory in the B200 layout (128-byte nodes,
 * leaf-ordered triangle records).  Replaces `Scene::build_qbvh` +
 * residency of `Scene` for `Scene::closest_hit`. */
tpt_status tpt_scene_upload(tpt_context* ctx, const tpt_scene_desc* desc, tpt_scene** out);
tpt_status tpt_scene_release(tpt_scene* scene);
/* Device bytes held by the scene. */
tpt_status tpt_scene_device_bytes(const tpt_scene* scene, uint64_t* bytes);

/* ------------------------------------------------------------------------ */
/* Ray queries (`Scene::closest_hit`, scene/mod.rs:340-395)                   */

typedef enum tpt_query_mode {
  TPT_CLOSEST_HIT = 0, /* Scene::closest_hit: nearest hit, reference visit order and tie rule */
  TPT_ANY_HIT = 1      /* first hit found below tmax (occlusion query) */
} tpt_query_mode;

/* rays: 7 planes of n floats: ox, oy, oz, dx, dy, dz, tmax (structure of
 * arrays).  TPT_CLOSEST_HIT starts every ray at t_max = +inf exactly like
 * Scene::closest_hit (the tmax plane is not read); TPT_ANY_HIT stops at the
 * first hit accepted below the ray's tmax.  Outputs (n each): triangle index
 * within its mesh (-1 = miss), hit distance (+inf on a miss).  instance and
 * bary (3 planes of barycentrics) may be NULL.
 * Host-pointer variant: the batch is split into chunks pipelined over two
 * streams (copy in, query, copy out overlap); page-locked caller buffers are
 * copied directly, pageable ones through pinned staging. */
tpt_status tpt_traverse(tpt_context* ctx, const tpt_scene* scene, const float* rays, uint64_t n, int mode,
                        int32_t* prim, float* t, int32_t* instance, float* bary);
tpt_status tpt_traverse_device(tpt_context* ctx, const tpt_scene* scene, const float* rays, uint64_t n, int mode,
                               int32_t* prim, float* t, int32_t* instance, float* bary, void* stream);
/* Same query, also writing per-ray counts of 4-wide node tests and triangle
 * tests (device pointers, n each); used for the algorithmic-bytes account. */
tpt_status tpt_traverse_stats_device(tpt_context* ctx, const tpt_scene* scene, const float* rays, uint64_t n,
                                     int mode, int32_t* prim, float* t, uint32_t* node_tests,
                                     uint32_t* tri_tests, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TPT_H_ */
