// Oracle: per-sample rendering (MIS integrator with SG light-tree NEE) for the
// NormalizedLambert and Emissive materials.  Restates
// crates/renderer/src/{integrator/{mod,mis}.rs, light/{mod,area}.rs,
// light_tree/{traversal,importance,lobe}.rs, math/{sg,mod,orthonormal_basis}.rs,
// material/{mod,normalized_lambert,emissive}.rs, bsdf/normalized_lambert.rs,
// scene/{mod,camera}.rs, main.rs:99-126}.
//
// The light tree is scene preparation, not the per-sample path: the oracle takes
// the flattened node array as input (the same one the device uses).
#pragma once
#include "camera.h"
#include "environment.h"
#include "geometry.h"
#include "openpbr.h"
#include "sampler.h"

namespace orc {

static constexpr float kPi = 3.14159274101257324f;
static constexpr float kTau = 6.28318548202514648f;

enum MatKind : uint32_t { kLambert = 0, kEmissive = 1, kOpenPbr = 2 };

struct Material {
  uint32_t kind = kLambert;
  Vec3 rho;        // NormalizedLambert
  Vec3 color;      // Emissive
  float strength = 0;
  float opacity = 1;  // NormalizedLambert / Emissive opacity (OpenPBR: geometry_opacity)
  OpenPbrDesc openpbr{};   // OpenPbr
  OpenPbrLuts luts{};      // the tables the scene installed for it (scene/mod.rs:164-185)
};

// Scene-level table cache (DirectionalAlbedoCache, directional_albedo.rs:38-118):
// one albedo table per distinct eta, one of each energy-compensation table.
OpenPbrLuts openpbr_luts_for(const OpenPbrDesc& m, int nthreads);

// light_tree/mod.rs:65-86 flattened (64 bytes; same layout as the C ABI's tpt_light_node)
struct LightNode {
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
static_assert(sizeof(LightNode) == 64, "light node");
static constexpr uint32_t kNoNode = 0xFFFFFFFFu;

struct Frame {
  Vec3 t, b, n;
  static Frame from_normal(Vec3 n);
  static Frame from_normal_and_tangent(Vec3 n, Vec3 hint);
  Vec3 to_world(Vec3 d) const { return normalize(d.x * t + d.y * b + d.z * n); }
  Vec3 to_local(Vec3 w) const { return Vec3(dot(w, t), dot(w, b), dot(w, n)); }
};

struct Vertex {
  Vec3 p, ng, ns, wo;
  Frame frame;
  int32_t inst, tri;
  bool front_face;
  // ShadingVertex::path_throughput / wavelength_lock: set by the integrators
  // before the vertex is shaded (read by dispersive transmission only)
  Vec3 path_throughput = Vec3(1, 1, 1);
  bool has_lock = false;
  float wavelength_lock = 0;
};

// scene/mod.rs:48-54: an emissive triangle with its selection weight
// (area * max_emission) and the running prefix of the weights.
struct AreaLight {
  int32_t inst, tri;
  float area, weight, prefix_weight;
};

// light/point.rs, light/spot.rs, light/directional.rs as their constructors
// store them (SpotLight::new clamps the angles and keeps their cosines; spot and
// directional directions are normalised).
struct PointLight {
  Vec3 position, color;
  float intensity;
};
struct SpotLight {
  Vec3 position, direction, color;
  float intensity, cos_total_width, cos_falloff_start;
};
struct DirLight {
  Vec3 direction, color;
  float intensity;
};
static constexpr uint32_t kLeafPoint = 0xFFFFFFFEu;  // light-tree leaf of a point light
static constexpr uint32_t kLeafSpot = 0xFFFFFFFDu;   // light-tree leaf of a spot light

struct RenderScene {
  Geometry geo;
  std::vector<Material> materials;
  std::vector<PointLight> points;
  std::vector<SpotLight> spots;
  std::vector<DirLight> dirs;
  bool has_env = false;  // Scene::environment_light
  Environment env;
  float env_cat_pmf = 0.0f;  // LightSampler::category_pmf(Environment)
  // LightSampler (light/mod.rs:117-188): categories (-1 = the tree, -3 = the
  // environment, i >= 0 = directional light i), their CDF and pmfs
  std::vector<int> cat_kind;
  std::vector<float> cat_cdf, cat_pmf;
  std::vector<AreaLight> area_lights;  // Scene::area_light_triangles, instance order
  float area_light_weight_sum = 0.0f;
  std::vector<LightNode> tree;
  uint32_t root = kNoNode;
  // (instance, triangle) -> leaf node, replacing the reference's HashMap
  std::vector<std::vector<uint32_t>> leaf_of;  // per instance (empty if not emissive)
  bool has_tree = false;
  float tree_cat_pmf = 0;

  void finalize();  // derived tables (after materials and tree are set)
  const Material& mat_of(int inst) const { return materials[geo.instances[inst].material_index]; }
  void triangle_world(int inst, int tri, Vec3* p) const;
  Vertex shading_vertex(int inst, int tri, Vec3 bary, Vec3 incident) const;
};

struct RenderJob {
  Camera cam;
  uint32_t width, height, spp, max_depth;
  uint32_t integrator = 0;  // 0 MIS, 1 BDPT, 2 NEE, 3 PT
  uint32_t seed = 0;        // the sample streams' scramble seed
};

// Material interface (material/mod.rs:251-502) for the kinds in scope, with
// the transport mode (material.rs modified_bsdf_eval / _sample_weight).
struct MatSampleOut {
  Vec3 weight, wi;
  float pdf = 0, pdf_rev = 0;
  bool delta = false;
  bool has_lock = false;  // MaterialSample::wavelength_lock
  float wavelength_lock = 0;
};
Vec3 material_eval(const Material& m, const Vertex& v, Vec3 wi, TransportMode mode);
float material_pdf(const Material& m, const Vertex& v, Vec3 wi);
bool material_sample(const Material& m, const Vertex& v, const MaterialRandoms& r, TransportMode mode,
                     MatSampleOut* s);
// Material::le at vertex v: EmissiveMaterial two-sided (emissive.rs:68-81),
// OpenPbrMaterial front face only unless thin-walled, times its exit tint
// (material/open_pbr.rs:351-375, 608-638); false for None.
bool material_le(const Material& m, const Vertex& v, Vec3* le);
// Material::may_emit / max_emission (material/mod.rs:395-420)
bool may_emit(const Material& m);
float max_emission(const Material& m);
inline bool is_pure_emitter(const Material& m) { return m.kind == kEmissive; }

// Light sampling at a scattering vertex.  kDirectMis:
// direct_light_mis_contribution (integrator/mis.rs:145-210); kDirectBdptNonArea:
// direct_non_area_light_contribution (integrator/bdpt.rs:396-464), zero when
// the sampled light is an area light; kDirectNee: direct_light_nee_contribution
// (integrator/nee.rs:104-150), no MIS weight and the plain environment
// distribution.  wi_out (optional): the light direction.
enum DirectMode : int { kDirectMis = 0, kDirectBdptNonArea = 1, kDirectNee = 2 };
// aux: the AuxRng the shadow ray's alpha tests draw from (NULL: no alpha tests).
Vec3 direct_light(const RenderScene& s, const Material& m, const Vertex& v, const VertexRandoms& rnd,
                  Vec3* wi_out = nullptr, int mode = kDirectMis, AuxRng* aux = nullptr);
// The environment's radiance along `dir` for a ray that left the scene after a
// BSDF sample of pdf `bsdf_pdf` (`delta`: count it in full), MIS-weighted
// against the environment's NEE pdf; zero without an environment.
Vec3 env_escape(const RenderScene& s, Vec3 dir, bool delta, float bsdf_pdf);
// Scene::environment_light, point, spot or directional lights (bdpt.rs:131-136)
inline bool scene_has_non_area_lights(const RenderScene& s) {
  return s.has_env || !s.points.empty() || !s.dirs.empty() || !s.spots.empty();
}

// pt::trace_radiance and nee::trace_radiance for one sample
Vec3 trace_pt(const RenderScene& s, const Ray& ray, const PathSampler& sampler, uint32_t max_depth);
Vec3 trace_nee(const RenderScene& s, const Ray& ray, const PathSampler& sampler, uint32_t max_depth);
// mis::trace_radiance for one sample
Vec3 trace_mis(const RenderScene& s, const Ray& ray, const PathSampler& sampler, uint32_t max_depth);
// bdpt::trace_radiance for one sample (integrator/bdpt.rs:70-131)
Vec3 trace_bdpt(const RenderScene& s, const Ray& ray, const PathSampler& sampler, uint32_t max_depth);

// Path-replay adjoint (no counterpart in the reference): replays the path of
// trace_mis with the same streams, given its radiance L, and calls `vertex` at
// every rough (non-delta) OpenPBR scattering vertex with the sampled direction
// and R = the part of L the path collects after that vertex (emission and NEE
// of later vertices).  OpenPBR vertices do no NEE, so R is exact there.
struct AdjointVertexSink {
  virtual ~AdjointVertexSink() = default;
  virtual void vertex(uint32_t material_index, const Vertex& v, Vec3 wi, Vec3 R) = 0;
};
void replay_mis(const RenderScene& s, const Ray& ray, const PathSampler& sampler, uint32_t max_depth, Vec3 L,
                AdjointVertexSink& sink);

// main.rs:99-126 for pixels [p0, p1): running mean over spp samples, times exposure.
void render_pixels(const RenderScene& s, const RenderJob& job, uint32_t p0, uint32_t p1, float* out_rgb, int nthreads);
// Per-sample radiance of paths [first, first + count), path = pixel * spp + sample.
void render_samples(const RenderScene& s, const RenderJob& job, uint64_t first, uint64_t count, float* out, int nthreads);

}  // namespace orc
