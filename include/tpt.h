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
 *    NULL = the context's stream); they are asynchronous on that stream.  Their
 *    return value covers argument checks and launches only: the device-side
 *    checks of the work they queue (traversal stack depth, queue capacity,
 *    bounded waits, index checks) set a per-context error word that
 *    tpt_context_check reads once that work has run.  Host-buffer variants read
 *    it themselves before returning.
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
/* Waits for `stream` (NULL = the context's stream) and reads, then clears, the
 * device-side error word that kernels queued by `*_device` calls set when one
 * of their checks fires (the reference's `ClosestHitError` and debug_assert!s,
 * scene/mod.rs:100-113, qbvh.rs:666): TPT_ERR_DEVICE_CHECK (traversal stack
 * deeper than 128 entries, an index check), TPT_ERR_CAPACITY (a device queue
 * overflowed) or TPT_ERR_TIMEOUT (a bounded wait gave up); the message names
 * the entry points whose work was queued since the word was last read.  Call
 * it after a `*_device` call's work (or a captured graph's replay) has been
 * ordered on `stream`; it cannot be called inside a stream capture. */
tpt_status tpt_context_check(tpt_context* ctx, void* stream);
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
/* The same build on the GPU (no counterpart in the reference): `d_bounds` is a
 * device array of n x 6 floats (stream: NULL = the context's).  The result is
 * the host builder's tree, node for node and in the same primitive order (a box
 * face at zero may hold +0.0 where the host builder keeps -0.0: both builders
 * keep the first zero they meet, and the GPU reduces in no fixed order).
 * Large ranges split level by level with all ranges of a level processed
 * element-parallel (the reference's swap partition reproduced from prefix
 * counts); ranges below 512 primitives are built by one thread each. */
tpt_status tpt_qbvh_build_device(tpt_context* ctx, const float* d_bounds, uint64_t n, void* stream, tpt_qbvh** out);
/* Whether tpt_scene_upload builds the QBVHs the description leaves empty on
 * the GPU (meshes and instance sets of at least 4096 primitives); default 0.
 * A GPU build that fails falls back to the host builder. */
tpt_status tpt_context_set_gpu_build(tpt_context* ctx, int enable);
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

/* Materials in scope (material/mod.rs:99-115 subset). */
typedef enum tpt_material_kind {
  TPT_MATERIAL_NORMALIZED_LAMBERT = 0, /* NormalizedLambertMaterial::new(rho) */
  TPT_MATERIAL_EMISSIVE = 1,           /* EmissiveMaterial::new(color, strength): two-sided pure emitter */
  TPT_MATERIAL_OPENPBR = 2             /* OpenPbrMaterial (untextured), parameters in `openpbr` */
} tpt_material_kind;

/* OpenPbrMaterial's untextured parameters (material/open_pbr.rs:23-78), same
 * names and meaning; tpt_openpbr_defaults() fills the values of
 * OpenPbrMaterial::new (material/open_pbr.rs:84-145) with base_color 0.8.
 * Lowered on upload into a flat device table (make_bsdf, material/open_pbr.rs:
 * 393-487) plus directional-albedo and energy-compensation tables built on the
 * GPU (bsdf/directional_albedo.rs).  The device path covers the base (EON
 * diffuse), metal, specular reflection, coat and fuzz lobes with anisotropy and
 * smooth (delta) lobes, specular transmission (rough and smooth GGX BTDF with
 * its multiple-scattering term), thin-walled slabs, thin-film interference on
 * the Fresnel terms, and emission (OpenPbrMaterial::le, open_pbr.rs:351-391:
 * emission_color * emission_luminance from the front face, both faces when
 * thin-walled, tinted by the coat and fuzz above it; such a surface is a light
 * of the light tree and of BDPT's area-light table).  Upload rejects with
 * TPT_ERR_INVALID_ARG no untextured parameter: geometry_opacity < 1 is the
 * alpha test of tpt_material_desc.opacity.  subsurface_weight is ignored, as the reference forces it to 0
 * (validate_and_warn).  Dispersion (transmission_dispersion_scale > 0,
 * bsdf/dispersion.rs) makes the transmission IOR a Cauchy function of
 * wavelength: an unlocked path evaluates the rough BTDF integrated over the
 * camera's spectral basis, and a sampled dispersive refraction locks the path
 * to one wavelength (the path state every integrator carries). */
typedef struct tpt_openpbr_desc {
  float base_weight;
  float base_color[3];
  float base_diffuse_roughness;
  float base_metalness;
  float specular_weight;
  float specular_color[3];
  float specular_roughness;
  float specular_ior;
  float specular_roughness_anisotropy;
  float transmission_weight;
  float transmission_color[3];
  float subsurface_weight;
  float subsurface_color[3];
  float fuzz_weight;
  float fuzz_color[3];
  float fuzz_roughness;
  float coat_weight;
  float coat_color[3];
  float coat_roughness;
  float coat_roughness_anisotropy;
  float coat_ior;
  float coat_darkening;
  float thin_film_weight;
  float thin_film_thickness;
  float thin_film_ior;
  float emission_luminance;
  float emission_color[3];
  float geometry_opacity;
  uint32_t geometry_thin_walled;
  float transmission_dispersion_scale;       /* 0 = no dispersion */
  float transmission_dispersion_abbe_number; /* Abbe number at scale 1 (abbe / scale is used) */
} tpt_openpbr_desc;

void tpt_openpbr_defaults(tpt_openpbr_desc* desc);

typedef struct tpt_material_desc {
  uint32_t kind;
  float rho[3];     /* NormalizedLambert albedo */
  float color[3];   /* Emissive colour */
  float strength;   /* Emissive strength */
  const struct tpt_openpbr_desc* openpbr;
  /* NormalizedLambert / Emissive opacity (their `opacity` field): used when
   * has_opacity != 0, else the material is opaque (1), so that a zeroed
   * record is opaque.  OpenPBR materials take geometry_opacity instead.  An
   * opacity below 1 gives the material an alpha test: Scene::closest_hit keeps
   * a hit on it iff an AuxRng draw is below the (clamped) opacity
   * (scene/mod.rs:360-377, 686-723). */
  uint32_t has_opacity;
  float opacity;
} tpt_material_desc;

/* Lights other than emissive triangles (light/{point,spot,directional}.rs),
 * with the reference's authoring conventions.  PointLight::new: `intensity` is
 * the emitted power in W.  SpotLight::new: the same power with a cone mask,
 * angles in radians (total_width clamped to [0, pi], falloff_start to
 * [0, total_width]; smoothstep falloff between them), direction normalised on
 * upload.  DirectionalLight::new: `direction` is the direction of travel
 * (normalised on upload), `intensity` the perpendicular irradiance in W/m^2.
 * Point and spot lights are leaves of the SG light tree; each directional
 * light is its own category of the light sampler (light/mod.rs:1-21). */
typedef struct tpt_point_light_desc {
  float position[3];
  float color[3];
  float intensity;
} tpt_point_light_desc;

typedef struct tpt_spot_light_desc {
  float position[3];
  float direction[3];
  float color[3];
  float intensity;
  float total_width;
  float falloff_start;
} tpt_spot_light_desc;

typedef struct tpt_directional_light_desc {
  float direction[3];
  float color[3];
  float intensity;
} tpt_directional_light_desc;

/* EnvironmentLight::from_pixels (light/environment.rs:46-82): an
 * equirectangular map of width x height RGB radiance values, row-major, row 0
 * at the +y pole; u = phi / 2pi with phi = atan2(x, z), v = theta / pi with
 * theta measured from +y.  `scale` multiplies the radiance, `rotate_y` rotates
 * the map about +y (radians).  Sampled through the reference's two mip-pyramid
 * distributions (luminance x sin(theta), and its MIS-compensated variant for
 * NEE); the map is one category of the light sampler, weighted by its total
 * power. */
typedef struct tpt_environment_desc {
  uint32_t width;
  uint32_t height;
  const float* pixels; /* width * height * 3 */
  float scale;
  float rotate_y;
} tpt_environment_desc;

/* One node of the SG light tree (light_tree/mod.rs:65-86), 64 bytes:
 * interior nodes have leaf_instance == leaf_triangle == 0xFFFFFFFF; leaves name
 * the emissive triangle and carry its area, or a point light
 * (leaf_instance == TPT_LIGHT_LEAF_POINT, leaf_triangle = its index) or a spot
 * light (TPT_LIGHT_LEAF_SPOT).  Children/parent are node indices
 * (0xFFFFFFFF = none). */
#define TPT_LIGHT_LEAF_POINT 0xFFFFFFFEu
#define TPT_LIGHT_LEAF_SPOT 0xFFFFFFFDu
typedef struct tpt_light_node {
  float flux;
  float mu[3];
  float sigma_s2;
  float nu[3];
  float lambda;
  float radius;
  uint32_t left, right, parent;
  uint32_t leaf_instance, leaf_triangle;
  float area;
} tpt_light_node;

typedef struct tpt_light_tree_view {
  const tpt_light_node* nodes;
  uint64_t num_nodes;
  uint32_t root;
} tpt_light_tree_view;

typedef struct tpt_scene_desc {
  const tpt_mesh_desc* meshes;
  uint32_t num_meshes;
  const tpt_instance_desc* instances;
  uint32_t num_instances;
  /* Pre-built TLAS over instance world bounds (`Scene::qbvh`, scene/mod.rs:305-317);
   * NULL arrays = build on upload. */
  tpt_qbvh_view tlas;
  const tpt_material_desc* materials;
  uint32_t num_materials;
  /* Pre-built light tree (`Scene::light_tree`); NULL nodes = build on upload
   * with the binned-SAOH builder (light_tree/builder.rs) over the emissive
   * triangles, in the order Scene::add_instance registers them, then the
   * point lights, then the spot lights. */
  tpt_light_tree_view light_tree;
  /* Scene::point_lights / spot_lights / directional_lights (may be NULL when
   * the count is 0).  In BDPT, as in the reference, light subpaths start on
   * emissive triangles only; these lights (and the environment) reach BDPT
   * through one light sample per camera vertex (bdpt.rs:207-221, 396-464). */
  const tpt_point_light_desc* point_lights;
  uint32_t num_point_lights;
  const tpt_spot_light_desc* spot_lights;
  uint32_t num_spot_lights;
  const tpt_directional_light_desc* directional_lights;
  uint32_t num_directional_lights;
  /* Scene::set_environment_light; NULL = none (rays that escape carry no
   * radiance). */
  const tpt_environment_desc* environment;
} tpt_scene_desc;

/* Copies the scene into device memory in the B200 layout (128-byte nodes,
 * leaf-ordered triangle records).  Replaces `Scene::build_qbvh` +
 * residency of `Scene` for `Scene::closest_hit`. */
tpt_status tpt_scene_upload(tpt_context* ctx, const tpt_scene_desc* desc, tpt_scene** out);
tpt_status tpt_scene_release(tpt_scene* scene);
/* Device bytes held by the scene. */
tpt_status tpt_scene_device_bytes(const tpt_scene* scene, uint64_t* bytes);
/* Host copy of the light tree the scene uses (valid while the scene lives);
 * num_nodes == 0 when the scene has no emitter. */
tpt_status tpt_scene_light_tree(const tpt_scene* scene, tpt_light_tree_view* view);

/* Host-side light-tree builder without a device (`Scene::build_light_tree`,
 * scene/mod.rs:300-303 -> light_tree/builder.rs:58-99): binned SAOH over the
 * scene's emissive triangles.  `desc` needs meshes, instances and materials;
 * fails with TPT_ERR_INVALID_ARG when nothing emits. */
typedef struct tpt_light_tree tpt_light_tree;
tpt_status tpt_light_tree_build(const tpt_scene_desc* desc, tpt_light_tree** out);
/* The same with at most `threads` host threads (<= 0: all hardware threads;
 * no counterpart in the reference, which builds on one): subtrees of 1,024 or
 * more emitters are built in parallel, and the tree is the same for every
 * thread count.  tpt_scene_upload builds with all hardware threads. */
tpt_status tpt_light_tree_build_threads(const tpt_scene_desc* desc, int threads, tpt_light_tree** out);
tpt_status tpt_light_tree_view_of(const tpt_light_tree* tree, tpt_light_tree_view* view);
tpt_status tpt_light_tree_free(tpt_light_tree* tree);

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
 * copied directly, pageable ones through pinned staging.  For TPT_CLOSEST_HIT
 * the tmax plane is not copied. */
tpt_status tpt_traverse(tpt_context* ctx, const tpt_scene* scene, const float* rays, uint64_t n, int mode,
                        int32_t* prim, float* t, int32_t* instance, float* bary);
tpt_status tpt_traverse_device(tpt_context* ctx, const tpt_scene* scene, const float* rays, uint64_t n, int mode,
                               int32_t* prim, float* t, int32_t* instance, float* bary, void* stream);
/* Scene::closest_hit with the alpha tests of its materials (scene/mod.rs:
 * 340-395, 686-723): aux (device, n uint32) holds each ray's AuxRng state
 * (aux_rng.rs: the state after from_seed); a candidate hit on an instance whose
 * material has opacity < 1 draws next_f32 from it and is kept iff the draw is
 * below the opacity.  aux is advanced in place by the draws, as the
 * reference's &mut AuxRng.  Without alpha-tested materials this is the
 * closest-hit query.  tpt_traverse / tpt_traverse_device ignore opacity. */
tpt_status tpt_traverse_alpha_device(tpt_context* ctx, const tpt_scene* scene, const float* rays, uint64_t n,
                                     uint32_t* aux, int32_t* prim, float* t, int32_t* instance, float* bary,
                                     void* stream);
/* Same query, also writing per-ray counts of 4-wide node tests and triangle
 * tests (device pointers, n each); used for the algorithmic-bytes account. */
tpt_status tpt_traverse_stats_device(tpt_context* ctx, const tpt_scene* scene, const float* rays, uint64_t n,
                                     int mode, int32_t* prim, float* t, uint32_t* node_tests,
                                     uint32_t* tri_tests, void* stream);

/* ------------------------------------------------------------------------ */
/* Rendering (`IntegratorKind::trace_radiance` per sample, main.rs:99-126 loop) */

typedef enum tpt_integrator {
  TPT_INTEGRATOR_MIS = 0, /* integrator/mis.rs: BSDF sampling + light sampling, balance heuristic */
  /* integrator/bdpt.rs: camera and light subpaths, every connection between
   * them, balance-heuristic MIS over the strategies (area lights picked by
   * power; other lights through one light sample per camera vertex).  The
   * wavefront (subpath steps, connection queue) unless `execution` is
   * TPT_EXEC_MEGAKERNEL (one thread per sample); max_depth is limited to 16
   * (TPT_ERR_CAPACITY above). */
  TPT_INTEGRATOR_BDPT = 1,
  /* integrator/nee.rs: light sampling without MIS (emitters and the
   * environment count only from the camera and after delta samples). */
  TPT_INTEGRATOR_NEE = 2,
  /* integrator/pt.rs: BSDF sampling only; every emitter hit and escape counts. */
  TPT_INTEGRATOR_PT = 3
} tpt_integrator;

/* PinholeCamera::new(eye, look_at, up, fov_y, exposure) (scene/camera.rs:21-39). */
typedef struct tpt_camera_desc {
  float eye[3];
  float look_at[3];
  float up[3];
  float fov_y; /* radians */
  float exposure;
} tpt_camera_desc;

typedef enum tpt_execution {
  TPT_EXEC_WAVEFRONT = 0,  /* stage kernels over compacted ray queues (default) */
  TPT_EXEC_MEGAKERNEL = 1, /* one persistent kernel: each thread carries one path at a time */
  TPT_EXEC_AUTO = 2        /* the execution tpt_autotune last picked on this context (wavefront before) */
} tpt_execution;

typedef struct tpt_render_job {
  const tpt_scene* scene;
  tpt_camera_desc camera;
  uint32_t width, height;
  uint32_t spp;       /* samples per pixel */
  uint32_t max_depth; /* --depth */
  uint32_t integrator;
  uint32_t execution; /* tpt_execution; both give the same image bit for bit */
  /* Scramble seed of the per-pixel sample streams (no counterpart in the
   * reference, whose PathSampler scrambles with the constant 0,
   * path_sampler.rs:77): 0 gives the reference's streams and images; any other
   * value gives statistically independent streams of the same sampler (for
   * independent replicas, and for an adjoint whose paths are not the forward
   * image's). */
  uint32_t seed;
} tpt_render_job;

/* Path slots of the wavefront pipeline's queues: a render is processed in
 * chunks of at most this many paths (0 = the default 2^24; otherwise
 * [1024, 2^26]).  Larger chunks fill the GPU better, smaller ones hold less
 * device memory (about 250 bytes per slot).  tpt_autotune picks it per
 * workload.  Setting it also makes tpt_render_batch_device batch again after
 * tpt_autotune chose job-by-job rendering.  Results do not depend on it. */
tpt_status tpt_context_set_wavefront_capacity(tpt_context* ctx, uint32_t slots);
uint32_t tpt_context_wavefront_capacity(const tpt_context* ctx);
/* Wavefront bounces are replayed from captured CUDA graphs (one per bounce
 * shape, cached per scene, camera and arena; default on).  enable = 0 launches
 * every stage directly.  Inside a caller's own stream capture the stages are
 * always launched directly (they join the caller's graph).  Results do not
 * depend on it. */
tpt_status tpt_context_set_graphs(tpt_context* ctx, int enable);
/* Measurement aid (no counterpart in the reference): while `d_counters` (device,
 * 8 uint64, zeroed by the caller) is set, single-job wavefront renders
 * (MIS, NEE, PT, BDPT and the adjoint replay) launch their stages directly
 * instead of replaying graphs, and their traversals add, per launch,
 * d_counters[0..3] = rays, 4-wide node tests, triangle tests and hits of the
 * path (camera, bounce, subpath) rays, and d_counters[4..7] the same for the
 * shadow and visibility rays.  These give the algorithmic bytes of a render.
 * Megakernel and batched renders are not counted.  NULL turns it off.  Results
 * do not depend on it. */
tpt_status tpt_context_set_render_stats(tpt_context* ctx, uint64_t* d_counters);
/* Threads per block of the wavefront shade stage: 128 or 256 (default). */
tpt_status tpt_context_set_shade_block(tpt_context* ctx, uint32_t threads);

/* Renders each job into out_rgb[j] (host, width*height*3 floats, row-major,
 * pixel = y*width + x): per pixel the running mean of `spp` samples in sample
 * order, times exposure — the raw linear buffer main.rs writes before output.
 * Several MIS wavefront jobs go through one batched launch sequence
 * (tpt_render_batch_device); the images are the same either way. */
tpt_status tpt_render(tpt_context* ctx, const tpt_render_job* jobs, int n_jobs, float* const* out_rgb);
/* One job into a device buffer, asynchronous on `stream`. */
tpt_status tpt_render_device(tpt_context* ctx, const tpt_render_job* job, float* out_rgb, void* stream);
/* Pixels [first_pixel, first_pixel + num_pixels) of `job`'s image (pixel =
 * y * width + x) into out_rgb (device, num_pixels * 3 floats), each the same
 * bits as in tpt_render_device's image: the unit a multi-GPU caller gives each
 * rank (row bands), gathering the bands into one image. */
tpt_status tpt_render_pixels_device(tpt_context* ctx, const tpt_render_job* job, uint64_t first_pixel,
                                    uint64_t num_pixels, float* out_rgb, void* stream);
/* The per-sample radiance of paths [first, first+count) in (pixel, sample)
 * order, path = pixel * spp + sample, into a device buffer of count*3 floats
 * (parity testing and sample-level consumers). */
tpt_status tpt_render_samples_device(tpt_context* ctx, const tpt_render_job* job, uint64_t first, uint64_t count,
                                     float* out_samples, void* stream);

/* The device's per-pixel sample streams (`PathSampler`, sampler/path_sampler.rs:
 * 81-141, over the Z-Sobol IndexSampler of sampler/zsobol.rs:206-285 and the
 * PCG hash of sampler/pcg.rs:1-13), exposed for testing them value for value.
 * For an image of width x height pixels at spp samples per pixel and n queries
 * (device, n x 4 uint32, 16-byte aligned: px, py, sample_index, depth):
 * out (device, n x 16 floats) = camera_sample (2), then
 * path_vertex_randoms(depth): u_category, u_tree, u_light_aux, u_surface (2),
 * u_lobe, u_layer, u_dir (2), u_extra0, u_extra1, u_extra2, u_extra3, u_rr;
 * seeds (device, n x 2) = initial_aux_rng_seed, the vertex's aux_rng_seed.
 * These are the values every render kernel draws for that (pixel, sample). */
tpt_status tpt_sampler_values_device(tpt_context* ctx, uint32_t width, uint32_t height, uint32_t spp, uint64_t n,
                                     const uint32_t* queries, float* out, uint32_t* seeds, void* stream);

/* Autotuner (no counterpart in the reference): times the candidate settings
 * on pilots of `jobs` (each job's rows scaled down: every candidate on at most
 * 2^24 paths; the candidates within 5 % of the best, the default and the
 * megakernel again on at most 2^26) and applies the fastest to the context:
 * the execution used by jobs whose `execution` is TPT_EXEC_AUTO, and, when that
 * is the wavefront, its queue capacity (tpt_context_set_wavefront_capacity),
 * graph replay (tpt_context_set_graphs) and shade block size
 * (tpt_context_set_shade_block).  Candidates: the megakernel, and the
 * wavefront (batched when n_jobs > 1) at capacities 2^18 .. 2^23, with and
 * without graph replay, at the context's shade block size; on the last pilot
 * the best wavefront candidate also at the other block size.  Every time
 * reported is from that last pilot.  MIS, NEE and PT jobs.  Results do not
 * depend on the settings. */
typedef struct tpt_tune_result {
  uint32_t execution;          /* TPT_EXEC_WAVEFRONT or TPT_EXEC_MEGAKERNEL */
  uint32_t wavefront_capacity; /* path slots per chunk */
  uint32_t graphs;             /* 1: bounces replayed from captured graphs */
  uint32_t shade_block;        /* threads per block of the wavefront shade stage */
  float ms;                    /* last-pilot time of the chosen settings */
  float ms_megakernel;         /* last-pilot time of the megakernel */
  float ms_wavefront_default;  /* last-pilot time of the wavefront at 2^24 slots, graphs, the context's block */
  uint64_t pilot_paths;        /* paths of the last pilot (about) */
  uint32_t stage;              /* which pilot the times come from: 1 (at most 2^24 paths) or 2 (at most 2^26) */
  uint32_t candidates;         /* settings timed */
  uint32_t batched;            /* 1: tpt_render_batch_device runs the jobs through one launch
                                  sequence; 0: one job after another, each its own wavefront
                                  (chosen when that was faster on the pilot) */
} tpt_tune_result;
tpt_status tpt_autotune(tpt_context* ctx, const tpt_render_job* jobs, int n_jobs, tpt_tune_result* out);

/* Batched rendering: n_jobs MIS jobs (any mix of scenes, cameras,
 * resolutions, spp and depths; `execution` is not read) through one wavefront
 * launch sequence, job j into the device image out_rgb[j] (width*height*3
 * floats), asynchronous on `stream`.  Each image equals tpt_render_device's for
 * the same job bit for bit.  No counterpart in the reference, which renders one
 * image per run (main.rs:99-126). */
tpt_status tpt_render_batch_device(tpt_context* ctx, const tpt_render_job* jobs, int n_jobs, float* const* out_rgb,
                                   void* stream);

/* Allocation-free variant of tpt_render_device, for callers that cannot call
 * cudaMalloc while they render (work recorded in a CUDA stream capture, hosts
 * whose device memory belongs to another allocator with a fixed budget,
 * latency-critical loops).  It has no counterpart in the reference.
 * Runs the megakernel execution (the job's `execution` field is not read) with
 * its per-sample scratch in a fixed array inside the library: at most
 * width * height * spp = 2^20 paths per call (12 MiB, held on every device that
 * loads the library until exit); larger jobs fail with TPT_ERR_CAPACITY.
 * The first call on a device looks up the array's device address; make that
 * first call before any stream capture.  Calls share the array and the
 * kernel's work counter (a fixed word beside the array, not one of the
 * context's counters): two calls whose work overlaps on the GPU race.  Output
 * equals tpt_render_device's bit for bit.  Device-side checks surface through
 * tpt_context_check, as for every `*_device` call. */
tpt_status tpt_render_device_noalloc(tpt_context* ctx, const tpt_render_job* job, float* out_rgb, void* stream);

/* ---- OpenPBR tables and BSDF queries -------------------------------------
 * The context builds each table on the GPU the first time a scene needs it and
 * keeps it until destroyed (DirectionalAlbedoCache, directional_albedo.rs:
 * 38-118): one directional-albedo table per distinct eta, one of each
 * energy-compensation table.  These copy a table to host memory (building it
 * first when needed); layouts and sizes are the reference's:
 *   dielectric albedo  64 (sqrt cos) x 16 (phi) x 64 (roughness) x 16 (anisotropy)
 *   conductor E        64 (roughness) x 64 (sqrt cos), E_avg 64
 *   dielectric E       32 (eta) x 32 (roughness) x 32 (sqrt cos), E_avg 32 x 32 */
tpt_status tpt_lut_dielectric_albedo(tpt_context* ctx, float eta, float* out);
tpt_status tpt_lut_conductor_ec(tpt_context* ctx, float* e, float* e_avg);
tpt_status tpt_lut_dielectric_ec(tpt_context* ctx, float* e, float* e_avg);

/* OpenPbrBsdf::eval and ::pdf of material `material` of an uploaded scene, for
 * n direction pairs in the shading frame (device buffers: wo, wi n x 3;
 * front_face n; f n x 3; pdf n).  mode: 0 radiance, 1 importance transport
 * (TransportMode).  The material must be OpenPBR. */
tpt_status tpt_bsdf_eval_device(tpt_context* ctx, const tpt_scene* scene, uint32_t material, uint64_t n,
                                const float* wo, const float* wi, const uint32_t* front_face, uint32_t mode, float* f,
                                float* pdf, void* stream);
/* OpenPbrBsdf::sample for n (wo, u) pairs: u n x 3 = (u_lobe, u_dir.x, u_dir.y);
 * out n x 9 = weight (3), wi (3), pdf, pdf_rev, flags (as uint32 bits:
 * 1 reflection, 4 diffuse, 8 glossy, 16 delta; 0 = no sample). */
tpt_status tpt_bsdf_sample_device(tpt_context* ctx, const tpt_scene* scene, uint32_t material, uint64_t n,
                                  const float* wo, const float* u, const uint32_t* front_face, uint32_t mode,
                                  float* out, void* stream);
/* The same queries with the path state a shading vertex carries
 * (ShadingVertex::path_throughput and wavelength_lock, which dispersive
 * transmission reads): state n x 4 = throughput r, g, b and the lock in nm
 * (NaN = none).  Sampling takes u n x 7 = (u_lobe, u_dir.x, u_dir.y,
 * u_extra0..3 of MaterialSampleRandoms) and writes n x 10: the 9 values above
 * and the wavelength lock the sample sets (NaN = none). */
tpt_status tpt_bsdf_eval_path_device(tpt_context* ctx, const tpt_scene* scene, uint32_t material, uint64_t n,
                                     const float* wo, const float* wi, const uint32_t* front_face, const float* state,
                                     uint32_t mode, float* f, float* pdf, void* stream);
tpt_status tpt_bsdf_sample_path_device(tpt_context* ctx, const tpt_scene* scene, uint32_t material, uint64_t n,
                                       const float* wo, const float* u, const uint32_t* front_face, const float* state,
                                       uint32_t mode, float* out, void* stream);

/* ---- Material updates and the path-replay adjoint -------------------------
 * Neither has a counterpart in the reference: its materials are fixed once
 * added to a Scene, and its renderer is not differentiable.  They give the
 * renderer a forward/backward pair for inverse rendering of OpenPBR materials:
 * forward = tpt_render_device, backward = tpt_adjoint_device. */

/* Replaces the parameters of OpenPBR materials of an uploaded scene (count
 * entries: scene material index, new parameters).  The new records are lowered
 * on the host and copied on `stream` (NULL = the context's stream), ordered
 * after the work already queued there; renders on other streams that read the
 * scene must have finished.  Fails with TPT_ERR_INVALID_ARG for a material that
 * is not OpenPBR, for parameters upload would reject, and for a change of
 * emission_luminance or emission_color (the light tree was built from them). */
tpt_status tpt_scene_set_openpbr(tpt_context* ctx, tpt_scene* scene, uint32_t count, const uint32_t* material_ids,
                                 const tpt_openpbr_desc* descs, void* stream);

/* Gradient layout: per scene material, TPT_GRAD_PARAMS doubles in this order. */
enum {
  TPT_GRAD_BASE_COLOR_R = 0,
  TPT_GRAD_BASE_COLOR_G = 1,
  TPT_GRAD_BASE_COLOR_B = 2,
  TPT_GRAD_SPECULAR_ROUGHNESS = 3,
  TPT_GRAD_BASE_METALNESS = 4,
  TPT_GRAD_SPECULAR_IOR = 5,
  TPT_GRAD_COAT_WEIGHT = 6,
  TPT_GRAD_PARAMS = 7
};
/* Parameter groups (bits of tpt_adjoint_desc.param_mask). */
enum {
  TPT_GRAD_MASK_BASE_COLOR = 1,
  TPT_GRAD_MASK_ROUGHNESS = 2,
  TPT_GRAD_MASK_METALNESS = 4,
  TPT_GRAD_MASK_IOR = 8,
  TPT_GRAD_MASK_COAT = 16,
  TPT_GRAD_ALL = 31
};

typedef struct tpt_adjoint_desc {
  uint32_t param_mask; /* groups to differentiate; 0 = TPT_GRAD_ALL */
  float fd_step;       /* parameter step of the BSDF central differences; 0 = 1e-3 */
  /* Pixels [first_pixel, first_pixel + num_pixels) whose paths are replayed
   * (num_pixels 0 = the whole image); d_image then holds those pixels only
   * (num_pixels * 3 floats).  The gradients of disjoint pixel ranges sum to
   * the whole image's (a multi-GPU caller all-reduces them). */
  uint32_t first_pixel, num_pixels;
} tpt_adjoint_desc;

/* dLoss/d(material parameters) of the image tpt_render_device produces for
 * `job` (MIS integrator; `execution` is not read), given d_image = dLoss/dimage
 * (device, width*height*3 floats, or the pixel range's when adesc names one).
 * grad (device, num_materials x
 * TPT_GRAD_PARAMS doubles) is overwritten; non-OpenPBR materials get zeros.
 * Path replay with detached sampling: per chunk of paths the forward wavefront
 * is run again for the paths' radiance, then replayed from the same streams,
 * and every rough OpenPBR vertex adds dLoss/dL * R * (df/dtheta) / f, R being
 * the radiance the path collects after the vertex and df/dtheta a central
 * difference of the BSDF at the sampled direction between host-lowered
 * theta -/+ fd_step copies of the material (clipped to [0, 1], the IOR to
 * [1, 10]); an unoccluded light sample C at an OpenPBR vertex (directional
 * lights, environment) adds dLoss/dL * C * (df/dtheta) / f at the light direction.
 * Accumulation is FP64 atomics, so the sums' order (and last bits)
 * vary between runs.  adesc may be NULL (all groups, step 1e-3).  Emission is
 * replayed but not differentiated: with the coat group in the mask, a scene
 * holding an OpenPBR emitter under a coat (whose exit tint depends on
 * coat_weight) fails with TPT_ERR_INVALID_ARG. */
tpt_status tpt_adjoint_device(tpt_context* ctx, const tpt_render_job* job, const tpt_adjoint_desc* adesc,
                              const float* d_image, double* grad, void* stream);
/* Host-buffer variant (synchronous). */
tpt_status tpt_adjoint(tpt_context* ctx, const tpt_render_job* job, const tpt_adjoint_desc* adesc,
                       const float* d_image, double* grad);

#ifdef __cplusplus
}
#endif

#endif /* TPT_H_ */
