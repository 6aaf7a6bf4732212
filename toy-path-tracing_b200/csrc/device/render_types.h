// Render-side device records shared by host (upload) and device code.  Plain
// structs only, so both g++ and nvcc compile this header.
#pragma once
#include <cstdint>

namespace tpt {

struct DevLightNodeRec {
  float flux;
  float mu[3];
  float sigma_s2;
  float nu[3];
  float lambda;
  float radius;
  uint32_t left, right, parent;
  uint32_t leaf_instance, leaf_triangle;
  float area;
};
static_assert(sizeof(DevLightNodeRec) == 64, "light node layout");

enum DevMatKind : uint32_t { kDevLambert = 0, kDevEmissive = 1, kDevOpenPbr = 2 };

// Longest BDPT subpath the device keeps on chip (vertices per subpath).
constexpr uint32_t kBdptMaxDepthApi = 16;

struct alignas(16) DevMaterialRec {
  uint32_t kind;
  float rho[3];
  float color[3];    // Emissive colour; OpenPBR emission_color
  float strength;    // Emissive strength; OpenPBR emission_luminance
  uint32_t openpbr;  // index into the OpenPBR parameter table
  uint32_t emits;    // OpenPBR with emission_luminance > 0 (may_emit): le() at its hits
  uint32_t pad[6];
};
static_assert(sizeof(DevMaterialRec) == 64, "material record");

// OpenPBR material lowered on the host (OpenPbrMaterial::make_bsdf,
// material/open_pbr.rs:393-487, minus its per-vertex parts): the layer
// parameters plus every constant of bsdf/open_pbr.rs that depends only on the
// material (albedo-table axes, multiple-scattering terms, lobe weights, F82
// terms, the view-independent half of the coat darkening), so that the device
// evaluates the per-direction terms only.
struct DevLerpAxis {  // compute_lut_axis_lerp (directional_albedo.rs:388-408)
  uint32_t lo, hi;
  float t;
};
struct DevMsFace {  // dielectric multiple scattering of one lobe seen from one face
  float eta_o, one_minus_e_avg_o, ms_factor;
  float lobe_ss, lobe_ms, lobe_total;  // dielectric_reflection_lobe_weights
  DevLerpAxis r_axis, eta_axis;         // energy-compensation table axes at (roughness_eq, eta_o)
  // the transmission half of dielectric_ms_params (open_pbr.rs:612-636) and
  // dielectric_transmission_lobe_weights (638-646)
  float eta_rel, one_minus_e_avg_t, ratio_r;
  float trans_ss, trans_ms, trans_total;
  DevLerpAxis eta_rel_axis;  // table axis at eta_rel
};
struct DevFresnelFace {  // base_dielectric_fresnel's weighted_fresnel_ratio arguments
  float unc_ti, unc_tp, coat_ti, coat_tp;
};
enum : uint32_t {
  kOpbrCoatRough = 1u,    // coat > 0 and not effectively smooth
  kOpbrMetalRough = 2u,   // metalness > 0 and not smooth
  kOpbrSpecRough = 4u,    // specular > 0 and not smooth
  kOpbrDarkening = 8u,    // coat darkening active
  kOpbrSpecDaSmooth = 16u,
  kOpbrCoatDaSmooth = 32u,
  kOpbrTrans = 64u,         // transmission > 0
  kOpbrTransRough = 128u,   // transmission > 0 and not smooth (spec_btdf_is_smooth false)
  kOpbrThinWalled = 256u,   // geometry_thin_walled
  kOpbrFilm = 512u,         // thin film: weight > 0 and thickness > 0
  kOpbrDisp = 1024u,        // dispersive transmission (transmission_dispersion_abbe > 0)
};
// The dielectric energy-compensation table E (32 eta x 32 roughness x 32
// sqrt cos); its E_avg (32 eta x 32 roughness) follows it in the same buffer.
constexpr uint32_t kDecTableLen = 32u * 32u * 32u;
struct alignas(16) DevOpenPbr {
  float base_color[3], base;
  float specular, specular_color[3];
  float spec_ax, spec_ay, metalness, coat;
  float coat_color[3], coat_ax;
  float coat_ay, coat_eta, fuzz, fuzz_roughness;  // fuzz roughness clamped to [0.01, 1]
  float fuzz_color[3], eon_r;
  float eon_r_pow01;  // r^0.1 of the EON uniform-lobe probability
  uint32_t flags;
  float spec_da_eta, coat_da_eta;  // etas of the albedo tables
  const float* spec_da;            // directional albedo tables (64 x 16 x 64 x 16)
  const float* coat_da;
  DevLerpAxis spec_da_r, coat_da_r;  // roughness axis at the roughness proxies
  // metal (F82-tint Fresnel + conductor multiple scattering)
  float f0[3], f82_delta[3];  // F0 and Schlick(F0, cos82) - target(cos82)
  float f82_denom;
  float cond_ss, cond_ms, cond_total, cond_one_minus_e_avg;
  float cond_f_ms[3];
  DevLerpAxis cond_r;
  // dielectric multiple scattering: [0] specular, [1] coat; [face] 0 front, 1 back
  DevMsFace ms[2][2];
  DevFresnelFace fres[2];
  float coat_clamped;  // coat weight clamped to [0, 1] for the Fresnel blend
  // coat darkening (material/open_pbr.rs:823-858) without the view term
  float dk_kr, dk_rb, dk_wd, dk_eta;
  float dk_e_base[3];
  // specular transmission: weight, clamped transmission colour, the thin-wall
  // GGX alphas (thin_wall_transmission_alpha_xy), the transmission eta and
  // the relative eta per face (transmission_eta_rel: 1/eta front, eta back)
  float transmission;
  float trans_color[3], tw_ax;
  float tw_ay, trans_eta, teta_rel[2];
  // thin film (bsdf/thin_film.rs): weight, thickness in nm, film IOR, and the
  // metal base's complex IOR (artist_friendly_complex_ior)
  float film_w, film_thick, film_ior;
  float disp_abbe;  // transmission_dispersion_abbe (0: no dispersion)
  float metal_n[3], metal_k[3];
  uint32_t pad2[2];
};

struct alignas(16) DevShadeInstance {
  float l2w[12];  // local_to_world affine columns c0..c3 (xyz each)
  float n2w[9];   // normal_to_world, column-major
  uint32_t mesh;
  uint32_t material;
  uint32_t leaf_base;  // first emitter-map slot of this instance, or 0xFFFFFFFF
  uint32_t pad[8];
};
static_assert(sizeof(DevShadeInstance) == 128, "shade instance record");

// Scene::area_light_triangles entry (scene/mod.rs:48-54): emissive triangle,
// its area, selection weight (area * max_emission) and the running prefix.
struct alignas(16) DevAreaLight {
  uint32_t inst, tri;
  float area, weight, prefix_weight;
  uint32_t pad[3];
};
static_assert(sizeof(DevAreaLight) == 32, "area light record");

// PointLight / SpotLight / DirectionalLight (light/{point,spot,directional}.rs)
// as the constructors store them (spot and directional directions normalised,
// spot cone angles as cosines).
struct DevPointLight {
  float position[3], color[3], intensity, pad;
};
struct DevSpotLight {
  float position[3], direction[3], color[3], intensity, cos_total_width, cos_falloff_start;
};
struct DevDirLight {
  float direction[3], color[3], intensity, pad;
};
constexpr uint32_t kLeafPointDev = 0xFFFFFFFEu;  // light-tree leaf of a point light
constexpr uint32_t kLeafSpotDev = 0xFFFFFFFDu;   // light-tree leaf of a spot light
constexpr uint32_t kCatTree = 0u;                // light-sampler category: the light tree;
                                                 // 1 + i: directional light i
constexpr uint32_t kCatEnv = 0xFFFFFFFFu;        // light-sampler category: the environment

// One hierarchical distribution of EnvironmentLight (light/environment.rs:
// 22-35): all mip levels of the padded (power-of-two) weight map, coarsest
// (1 x 1) first; levels[3 l .. 3 l + 2] = width, height, offset of level l.
struct DevEnvDist {
  const float* weights;
  const uint32_t* levels;
  uint32_t num_levels;
  float total_weight;
};

// EnvironmentLight: RGB map (row-major), scale, rotation about +y as
// Mat3::from_rotation_y(+-rotate_y) columns, and its two distributions.
struct DevEnvironment {
  const float* pixels;
  uint32_t width, height;
  float scale;
  float cat_pmf;         // LightSampler pmf of the Environment category (0: not a category)
  float rot[9], inv_rot[9];  // column-major 3 x 3
  DevEnvDist dist;       // luminance x sin(theta)
  DevEnvDist mis;        // MIS-compensated: (luminance - mean) x sin(theta) where above epsilon
};

struct DevMeshInfo {
  uint32_t vtx_base, idx_base, num_tris, flags;  // flags bit 0: normals, bit 1: uvs
};

struct DevRenderData {
  const DevShadeInstance* inst;
  const DevMeshInfo* meshes;
  const float* pos;
  const float* nrm;
  const float* uv;
  const uint32_t* idx;
  const DevMaterialRec* mats;
  const DevLightNodeRec* ltree;
  const uint32_t* emitter_leaf;
  const DevOpenPbr* openpbr;  // OpenPBR parameter table
  const float* cec_e;         // conductor energy-compensation table (64 x 64)
  const float* dec_e;         // dielectric energy-compensation table (32 x 32 x 32)
  const DevAreaLight* area_lights;  // in registration (instance, triangle) order
  const uint32_t* area_light_of;    // emitter-map slot -> area light index (or 0xFFFFFFFF)
  uint32_t num_area_lights;
  float area_light_weight_sum;
  uint32_t ltree_root;
  uint32_t has_tree;
  float tree_cat_pmf;  // LightSampler pmf of the Tree category
  uint32_t num_materials;
  // lights that are not emissive triangles, and the light sampler's category
  // CDF (LightSampler::build_from_scene, light/mod.rs:134-188)
  const DevPointLight* points;
  const DevSpotLight* spots;
  const DevDirLight* dirs;
  const float* cat_cdf;      // num_cat + 1 entries, normalised
  const float* cat_pmf;      // num_cat
  const uint32_t* cat_kind;  // kCatTree, kCatEnv or 1 + directional index
  uint32_t num_cat;
  uint32_t num_extra_lights; // point + spot + directional lights + the environment
  uint32_t has_env;
  DevEnvironment env;
};

// Camera constants computed on the host (scene/camera.rs:21-39).
struct DevCamera {
  float eye[3], forward[3], right[3], up[3];
  float tan_half_fov_y;
  float exposure;
};

struct RenderLaunch {
  DevCamera cam;
  uint32_t width, height, spp, max_depth;
  uint32_t log2_spp, n_base4_digits;
  uint32_t integrator;  // tpt_integrator: 0 MIS, 1 BDPT, 2 NEE, 3 PT
  uint32_t seed;        // the sample streams' scramble seed (tpt_render_job.seed)
};
constexpr uint32_t kIntegMis = 0, kIntegBdpt = 1, kIntegNee = 2, kIntegPt = 3;

// Path-replay adjoint (no counterpart in the reference): inputs of the adjoint
// instantiation of the wavefront stages.  Gradients are per scene material,
// kGradParams doubles each: base_color r, g, b, specular_roughness,
// base_metalness, specular_ior, coat_weight.  The BSDF partials are central
// differences between two host-lowered copies of each OpenPBR material, one
// pair per parameter group (base colour, roughness, metalness, ior, coat).
constexpr uint32_t kGradParams = 7;
constexpr uint32_t kGradGroups = 5;
struct DevAdjoint {
  const DevOpenPbr* pert;  // [OpenPBR table index][group][lo, hi]
  const float* span;       // [OpenPBR table index][group][3]: hi - lo per channel
  const float* d_image;    // dLoss/dimage of pixels [pixel_base, ...): 3 floats each
  double* grad;            // [material][kGradParams]
  float scale;             // exposure / spp: d image / d sample radiance
  uint32_t mask;           // parameter groups to differentiate (bit g = group g)
  uint32_t pixel_base;     // first pixel of the replayed range
  // light samples at OpenPBR vertices (directional lights), per shadow-queue
  // entry: the gradient change if the shadow ray is unoccluded (kGradParams
  // planes of the wavefront capacity) and its material (0xFFFFFFFF: none).
  // NULL when the scene has no such light samples.
  float* s_grad;
  uint32_t* s_gkey;
};

// BDPT wavefront state (kernels/bdpt_wavefront.cu) for up to sample_capacity
// samples of max_vertices vertices per subpath and pair_capacity connections.
struct BdVertex;
struct BdCamState;
struct BdLightState;
constexpr uint32_t kBdVertexBytes = 128;  // >= sizeof(BdVertex), for host-side sizing
constexpr uint32_t kBdStateBytes = 64;    // >= sizeof(BdCamState), sizeof(BdLightState)
struct BdWfBuffers {
  uint32_t sample_capacity, pair_capacity, max_vertices, pad;
  // subpath stage: per-sample loop states and two ray queues of 2 x sample_capacity
  BdCamState* cam_state;
  BdLightState* light_state;
  float* q_ray[2];       // 7 planes each
  uint32_t* q_tag[2];    // sample index, bit 31: light subpath
  int32_t* h_tri;
  int32_t* h_inst;
  float* h_t;
  float* h_bary;         // 3 planes
  BdVertex* verts;       // [sample][camera 0..max_vertices, light 0..max_vertices]
  uint32_t* nc;          // camera subpath length per sample
  uint32_t* nl;          // light subpath length per sample
  uint32_t* pair_base;   // first connection slot of each sample
  float* L0;             // camera-subpath emission per sample (3 planes interleaved)
  uint32_t* pair_sample; // sample of each connection slot
  float* c;              // connection contribution before MIS (x3)
  float* contrib;        // MIS-weighted contribution, zero if none (x3)
  float* dist;           // connection length
  float* s_ray;          // visibility rays: 7 planes of pair_capacity
  uint32_t* s_pair;      // connection slot of each visibility ray
  int32_t* s_tri;
  int32_t* s_inst;
  float* s_t;
  uint32_t* counts;      // [0] connections, [1] visibility rays, [2], [3] camera and [4], [5] light
                         // halves of the subpath ray queues
};

// Wavefront state: per path slot of a chunk (capacity slots), two ray queues,
// the hit records of the current queue and the shadow queue.  Planes of a
// structured array are `capacity` elements apart.
struct WfBuffers {
  uint32_t capacity;
  float* beta;        // 3 planes
  float* L;           // 3 planes
  float* prev;        // 7 planes: previous vertex p (3), ns (3), BSDF pdf
  uint32_t* prev_mat; // previous vertex material index, bit 31 = delta sample
  uint32_t* depth;    // vertices processed
  float* lock;        // the path's wavelength lock (< 0: none)
  // alpha tests (NULL in renders without them): the AuxRng state each path's
  // next bounce ray starts from (per slot), each shadow ray's, and whether a
  // shadow ray's final state carries on to its path's bounce ray (MIS)
  uint32_t* q_aux;
  uint32_t* s_aux;
  uint32_t* s_aux_cont;
  uint32_t* q_slot[2];
  float* q_ray[2];    // 7 planes each: o, d, tmax
  int32_t* h_tri;
  int32_t* h_inst;
  float* h_t;
  float* h_bary;      // 3 planes
  uint32_t* s_slot;
  float* s_ray;       // 7 planes
  float* s_contrib;   // 3 planes
  uint32_t* s_target; // 2 planes: instance, triangle (0xFFFFFFFF: a point, spot or directional light)
  float* s_dist;      // distance to a point or spot light (inf: directional)
  int32_t* s_tri;
  int32_t* s_inst;
  float* s_t;
  uint32_t* counts;   // [0], [1]: ray queue lengths, [2]: shadow queue length
  // batched renders only: the job of each slot, of each queued ray and of
  // each shadow ray (index into the batch's DevJob array)
  uint32_t* job;
  uint32_t* q_job[2];
  uint32_t* s_job;
};

}  // namespace tpt
