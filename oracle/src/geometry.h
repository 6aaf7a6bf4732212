// Oracle: ray, triangle test, QBVH build and traversal, two-level scene queries.
// Restates crates/renderer/src/math/ray.rs, crates/renderer/src/qbvh.rs and the
// intersection part of crates/renderer/src/scene/{mod,mesh}.rs.
#pragma once
#include "common.h"

namespace orc {

// ray.rs:6-11 (differentials and cone are carried for shading; traversal ignores them)
struct RayDiff {
  Vec3 rx_origin, ry_origin, rx_direction, ry_direction;
};
struct Ray {
  Vec3 origin, direction;
  bool has_diff = false;
  RayDiff diff;
  float cone_width = 0.0f, cone_spread = 0.0f;
};

struct TriHit {
  float t;
  Vec3 bary;
};

// math/mod.rs:136-141
inline float difference_of_products(float a, float b, float c, float d) {
  float cd = c * d;
  float dop = std::fma(a, b, -cd);
  float err = std::fma(-c, d, cd);
  return dop + err;
}
// math/mod.rs:143-146
inline float gamma_n(int n) {
  const float eps = std::numeric_limits<float>::epsilon() * 0.5f;
  float nf = (float)n;
  return (nf * eps) / (1.0f - nf * eps);
}
// math/mod.rs:148-156
inline int max_component_index(const Vec3& v) {
  if (v.x > v.y) return v.x > v.z ? 0 : 2;
  return v.y > v.z ? 1 : 2;
}

bool intersect_triangle(const Ray& ray, float t_max, const Vec3& v0, const Vec3& v1, const Vec3& v2,
                        TriHit* out);

// qbvh.rs:15-20, 29-51
static constexpr uint32_t kLeafBit = 1u << 31;
static constexpr uint32_t kEmptyChild = kLeafBit;
inline uint32_t encode_leaf(uint32_t offset, uint32_t count) { return kLeafBit | (count << 24) | offset; }

struct Bounds {
  Vec3 min = Vec3::splat(kInf), max = Vec3::splat(-kInf);
  Vec3 center() const { return 0.5f * (min + max); }
  Vec3 extent() const { return max - min; }
  float surface_area() const {
    Vec3 e = vmax(extent(), Vec3(0, 0, 0));
    return 2.0f * (e.x * e.y + e.x * e.z + e.y * e.z);
  }
  Bounds unite(const Bounds& o) const { Bounds b; b.min = vmin(min, o.min); b.max = vmax(max, o.max); return b; }
};

// qbvh.rs:53-63: lanes of the 4-wide node; layout of the C struct is
// bounds[6][4] (min_x, min_y, min_z, max_x, max_y, max_z), children[4], valid_mask.
struct QbvhNode {
  float b[6][4];
  uint32_t children[4];
  uint32_t valid_mask;
  uint32_t pad[3];
};
static_assert(sizeof(QbvhNode) == 128, "node layout");

struct Qbvh {
  std::vector<QbvhNode> nodes;
  std::vector<uint32_t> primitive_indices;
};

bool build_qbvh(const std::vector<Bounds>& prim_bounds, Qbvh* out);

struct TraversalStats {
  uint64_t nodes = 0;      // interior nodes whose 4-wide box test ran
  uint64_t triangles = 0;  // triangle tests
  uint64_t instances = 0;  // instance (BLAS) entries
};

// qbvh.rs:611-675. The callback gets (offset, count, t_max) and returns the new t_max;
// returning a negative value from `stop` requests early termination (any-hit).
template <class Leaf>
float traverse_qbvh(const Qbvh& q, const Ray& ray, float initial_t_max, Leaf&& leaf_cb, bool* stop,
                    TraversalStats* st);

struct Mesh {
  std::vector<Vec3> positions;
  std::vector<Vec3> normals;
  std::vector<Vec2> uvs;
  std::vector<uint32_t> indices;
  Bounds bounds;
  Qbvh qbvh;
  size_t triangle_count() const { return indices.size() / 3; }
  void triangle_positions(size_t t, Vec3* v) const {
    v[0] = positions[indices[3 * t]];
    v[1] = positions[indices[3 * t + 1]];
    v[2] = positions[indices[3 * t + 2]];
  }
};

struct Instance {
  uint32_t mesh_index;
  uint32_t material_index;
  Mat4 local_to_world, world_to_local;
  Mat3 normal_to_world;
  Bounds world_bounds;
};

struct SceneHit {
  int32_t instance = -1;
  int32_t triangle = -1;
  float t = kInf;
  Vec3 bary;
};

struct AuxRng;

struct Geometry {
  std::vector<Mesh> meshes;
  std::vector<Instance> instances;
  Qbvh tlas;
  // Per instance: the opacity of its material's alpha test (Material::
  // has_alpha_test / any_hit, untextured), 1 where the material has none.
  // Empty: no instance has one.
  std::vector<float> alpha;
  // scene/mod.rs:340-395 with closest_mesh_hit_with_filter (686-723): with an
  // AuxRng, a candidate hit on an alpha-tested instance draws u from it and
  // is kept iff u < opacity; without one every hit is kept.
  bool closest_hit(const Ray& ray, SceneHit* hit, TraversalStats* st = nullptr, AuxRng* aux = nullptr) const;
  // First accepted hit in the same visit order; used for occlusion-only queries.
  bool any_hit(const Ray& ray, float t_max, SceneHit* hit, TraversalStats* st = nullptr) const;
};

Bounds transform_bounds(const Bounds& b, const Mat4& m);

}  // namespace orc

#include "traverse_impl.h"
