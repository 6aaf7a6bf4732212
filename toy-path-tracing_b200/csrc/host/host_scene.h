// Host-side scene description shared by the uploader and the light-tree builder.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

namespace tpt {

constexpr uint32_t kInvalidNode = 0xFFFFFFFFu;

enum MaterialKind : uint32_t {
  kMatLambert = 0,   // NormalizedLambertMaterial (material/normalized_lambert.rs)
  kMatEmissive = 1,  // EmissiveMaterial (material/emissive.rs)
  kMatOpenPbr = 2,   // OpenPbrMaterial (material/open_pbr.rs)
};

struct HostMaterial {
  uint32_t kind;
  float rho[3];       // Lambert
  float color[3];     // Emissive colour; OpenPBR emission_color
  float strength;     // Emissive strength; OpenPBR emission_luminance
  // Material::may_emit (material/mod.rs): the emissive material, and an
  // OpenPBR material with emission_luminance > 0 (material/open_pbr.rs:377-379)
  bool may_emit() const { return kind == kMatEmissive || (kind == kMatOpenPbr && strength > 0.0f); }
  float max_emission() const {
    if (kind == kMatEmissive) {
      // EmissiveMaterial::max_emission (emissive.rs:87-94): max channel of colour * strength, >= 0
      float a = color[0] * strength, b = color[1] * strength, c = color[2] * strength;
      float m = std::fmax(a, std::fmax(b, c));
      return std::fmax(m, 0.0f);
    }
    if (kind == kMatOpenPbr && strength > 0.0f) {
      // OpenPbrMaterial::max_emission (material/open_pbr.rs:381-391), untextured
      const float m = std::fmax(color[0], std::fmax(color[1], color[2]));
      return std::fmax(m * strength * 1.0f, 0.0f);
    }
    return 0.0f;
  }
};

struct HostMesh {
  const float* positions;
  const float* normals;  // may be null
  const float* uvs;      // may be null
  const uint32_t* indices;
  uint32_t num_vertices;
  uint32_t num_triangles;
};

struct HostInstance {
  uint32_t mesh, material;
  const float* local_to_world;  // 16, column-major
  const float* world_to_local;
  const float* normal_to_world;  // 9, column-major
};

// PointLight::new / SpotLight::new (light/point.rs, light/spot.rs) as stored:
// spot direction normalised, cone angles as cosines.
struct HostPointLight {
  float position[3], color[3], intensity;
};
struct HostSpotLight {
  float position[3], direction[3], color[3], intensity, cos_total_width, cos_falloff_start;
};

struct HostSceneView {
  const HostMesh* meshes;
  uint32_t num_meshes;
  const HostInstance* instances;
  uint32_t num_instances;
  const HostMaterial* materials;
  uint32_t num_materials;
  const HostPointLight* points = nullptr;
  uint32_t num_points = 0;
  const HostSpotLight* spots = nullptr;
  uint32_t num_spots = 0;
};

constexpr uint32_t kLeafPoint = 0xFFFFFFFEu;  // tree leaf of a point light (leaf_triangle = index)
constexpr uint32_t kLeafSpot = 0xFFFFFFFDu;   // tree leaf of a spot light

// Same bytes as `tpt_light_node` in include/tpt.h (64 bytes).
struct LightNodeHost {
  float flux;
  float mu[3];
  float sigma_s2;
  float nu[3];
  float lambda;
  float radius;
  uint32_t left, right, parent;
  uint32_t leaf_instance, leaf_triangle;  // kInvalidNode for interior nodes
  float area;                             // emitter triangle area (leaves)
};
static_assert(sizeof(LightNodeHost) == 64, "light node layout");

struct LightTreeHost {
  std::vector<LightNodeHost> nodes;
  uint32_t root = kInvalidNode;
};

// glam Mat4::transform_point3 (column-major m[16]) of p[3] into out[3].
inline void transform_point_glam(const float* m, const float* p, float* out) {
  float r[3];
  for (int i = 0; i < 3; ++i) r[i] = m[0 + i] * p[0];
  for (int i = 0; i < 3; ++i) r[i] = m[4 + i] * p[1] + r[i];
  for (int i = 0; i < 3; ++i) r[i] = m[8 + i] * p[2] + r[i];
  for (int i = 0; i < 3; ++i) r[i] = m[12 + i] + r[i];
  out[0] = r[0]; out[1] = r[1]; out[2] = r[2];
}

// threads <= 0: all hardware threads; the tree does not depend on it.
bool build_light_tree_host(const HostSceneView& s, LightTreeHost* out, int threads = 0);
// SpotLight::new (light/spot.rs:32-48) from the C ABI's description.
void make_spot_light(const float* position, const float* direction, const float* color, float intensity,
                     float total_width_rad, float falloff_start_rad, HostSpotLight* out);

struct HostAreaLight {
  uint32_t inst, tri;
  float area, weight, prefix_weight;
};
void register_area_lights(const HostSceneView& s, std::vector<HostAreaLight>* out, float* weight_sum);

}  // namespace tpt
