// Host-side SG light-tree builder (binned SAOH, 12 bins, one emitter per leaf).
//
// Restates crates/renderer/src/light_tree/builder.rs:58-765 and the cluster
// algebra of crates/renderer/src/math/sg.rs:203-214, 325-346 for emissive
// triangles, point lights and spot lights.
// Node order is the reference's: an interior node is reserved before its left
// then right subtree (pre-order).  The tree is full (every interior node has
// two children), so a subtree over k emitters holds 2k - 1 nodes and the
// right child of node i with a left part of k emitters is node i + 2k: the
// two subtrees write disjoint node and emitter ranges, and large ones are
// built on separate threads with the same result as one thread.
// `sort_unstable_by` on centroids
// (builder.rs:486-490, 758-762) has no defined order for equal keys; here
// equal centroids keep their emitter registration order.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <numeric>
#include <exception>
#include <thread>
#include <vector>

#include "host_scene.h"

namespace tpt {
namespace {

constexpr int kBins = 12;
constexpr float kPi = 3.14159265358979323846f;
constexpr float kSgSharpnessMax = 2.1990233e12f;  // 2^41, sg.rs:26

struct V3 {
  float x, y, z;
};
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 mul(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 mulv(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 divs(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(V3 a) { return mulv(a, 1.0f / length(a)); }
inline V3 normalize_or_zero(V3 a) {
  float r = 1.0f / length(a);
  return (std::isfinite(r) && r > 0.0f) ? mulv(a, r) : V3{0, 0, 0};
}
inline V3 vmin(V3 a, V3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
inline V3 vabs(V3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline float comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
// sg.rs:314-316
inline float luminance(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

struct Box {
  V3 lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
  void grow(const Box& o) { lo = vmin(lo, o.lo); hi = vmax(hi, o.hi); }
  float area() const {
    V3 e = vmax(sub(hi, lo), V3{0, 0, 0});
    return 2.0f * (e.x * e.y + e.x * e.z + e.y * e.z);
  }
};

// sg.rs:203-214
float vmf_axis_length_to_sharpness(float axis_length) {
  float r = std::fmin(std::fmax(axis_length, 0.0f), 1.0f);
  if (std::isnan(axis_length)) r = axis_length;
  if (r >= 1.0f) return kSgSharpnessMax;
  float one_minus = 1.0f - r * r;
  if (one_minus <= 0.0f) return kSgSharpnessMax;
  float lambda = r * (3.0f - r * r) / one_minus;
  return std::fmin(std::fmax(lambda, 0.0f), kSgSharpnessMax);
}

// builder.rs:244-343 (Conty & Kulla 2018 orientation bounds)
struct Cone {
  V3 axis{0, 0, 1};
  float theta_o = 0, theta_e = 0;
  bool valid = false;
  float measure() const {
    if (!valid) return 0.0f;
    float to = std::fmin(std::fmax(theta_o, 0.0f), kPi);
    float te = std::fmin(std::fmax(theta_e, 0.0f), kPi * 0.5f);
    float tw = std::fmin(to + te, kPi);
    float co = std::cos(to), so = std::sin(to);
    return 2.0f * kPi * (1.0f - co) + 0.5f * kPi * (2.0f * tw * so - std::cos(to - 2.0f * tw) - 2.0f * to * so + co);
  }
  static Cone merge(Cone a, Cone b) {
    if (!a.valid) return b;
    if (!b.valid) return a;
    float theta_e = std::fmax(a.theta_e, b.theta_e);
    if (!(a.theta_o >= b.theta_o)) std::swap(a, b);
    float cos_d = std::fmin(std::fmax(dot(a.axis, b.axis), -1.0f), 1.0f);
    float theta_d = std::acos(cos_d);
    if (std::fmin(theta_d + b.theta_o, kPi) <= a.theta_o) return Cone{a.axis, a.theta_o, theta_e, true};
    float theta_o = std::fmin((a.theta_o + theta_d + b.theta_o) * 0.5f, kPi);
    if (theta_o >= kPi - 1e-5f) return Cone{a.axis, kPi, theta_e, true};
    V3 rot = cross(a.axis, b.axis);
    V3 axis;
    if (dot(rot, rot) > 1.0e-12f) {
      float theta_r = theta_o - a.theta_o;
      V3 k = normalize(rot);
      float cr = std::cos(theta_r), sr = std::sin(theta_r);
      axis = normalize_or_zero(add(add(mulv(a.axis, cr), mulv(cross(k, a.axis), sr)), mulv(k, dot(k, a.axis) * (1.0f - cr))));
    } else {
      axis = a.axis;
    }
    return Cone{dot(axis, axis) > 0.0f ? axis : a.axis, theta_o, theta_e, true};
  }
};

struct Leaf {
  uint32_t inst, tri;
  float flux;
  V3 mu;
  float sigma_s2;
  V3 nu_bar;
  Box aabb;
  float radius;
  Cone cone;
  V3 centroid;
  float area;
  uint32_t order;
};

// builder.rs:357-456
struct Cluster {
  float flux = 0;
  V3 mu{0, 0, 0};
  float sigma_s2 = 0;
  V3 nu_bar{0, 0, 0};
  Box aabb;
  float radius = 0;
  Cone cone;

  // sg.rs:325-346
  void absorb(float f, V3 m, float s2, V3 nb) {
    float total = flux + f;
    if (total <= 0.0f) { mu = {0, 0, 0}; sigma_s2 = 0; nu_bar = {0, 0, 0}; flux = 0; return; }
    float wl = flux / total, wr = f / total;
    V3 nmu = add(mul(wl, mu), mul(wr, m));
    V3 d = sub(mu, m);
    float ns = wl * sigma_s2 + wr * s2 + wl * wr * dot(d, d);
    V3 nnu = add(mul(wl, nu_bar), mul(wr, nb));
    mu = nmu; sigma_s2 = ns; nu_bar = nnu; flux = total;
  }
  void merge_leaf(const Leaf& l) {
    if (flux + l.flux <= 0.0f) return;
    if (flux <= 0.0f) {
      flux = l.flux; mu = l.mu; sigma_s2 = l.sigma_s2; nu_bar = l.nu_bar; aabb = l.aabb; cone = l.cone;
      return;
    }
    absorb(l.flux, l.mu, l.sigma_s2, l.nu_bar);
    aabb.grow(l.aabb);
    cone = Cone::merge(cone, l.cone);
  }
  void merge_with(const Cluster& o) {
    if (o.flux <= 0.0f) return;
    if (flux <= 0.0f) { *this = o; return; }
    absorb(o.flux, o.mu, o.sigma_s2, o.nu_bar);
    aabb.grow(o.aabb);
    cone = Cone::merge(cone, o.cone);
  }
  void finish_radius() {
    if (flux <= 0.0f) { radius = 0; return; }
    V3 e = vmax(vabs(sub(aabb.hi, mu)), vabs(sub(aabb.lo, mu)));
    radius = length(e);
  }
};

// Subtrees of at least this many emitters may go to another thread.
constexpr size_t kParallelMin = 1024;

class TreeBuilder {
 public:
  // `out` is sized to 2n - 1 nodes by the caller; `threads` caps the threads
  // working at once (the caller's included).
  TreeBuilder(std::vector<LightNodeHost>* out, int threads) : nodes_(*out), spare_(std::max(0, threads - 1)) {}

  // Builds the subtree over L[0, n) at node `idx`.
  void build(Leaf* L, size_t n, uint32_t parent, uint32_t idx) {
    if (n <= 1) {
      put_leaf(L[0], parent, idx);
      return;
    }
    Cluster total;
    for (size_t i = 0; i < n; ++i) total.merge_leaf(L[i]);
    total.finish_radius();
    size_t split;
    if (!best_split(L, n, total, &split)) {
      // median split along the longest centroid extent (builder.rs:471-492)
      V3 mn{INFINITY, INFINITY, INFINITY}, mx{-INFINITY, -INFINITY, -INFINITY};
      for (size_t i = 0; i < n; ++i) { mn = vmin(mn, L[i].centroid); mx = vmax(mx, L[i].centroid); }
      V3 d = sub(mx, mn);
      int axis = (d.x >= d.y && d.x >= d.z) ? 0 : (d.y >= d.z ? 1 : 2);
      sort_axis(L, n, axis);
      split = n / 2;
    }
    split = std::min(std::max<size_t>(split, 1), n - 1);
    const uint32_t l = idx + 1, r = idx + 2 * (uint32_t)split;
    LightNodeHost& nd = nodes_[idx];
    nd = LightNodeHost{};
    nd.left = l;
    nd.right = r;
    nd.parent = parent;
    fill_cluster(nd, total.flux, total.mu, total.sigma_s2, total.nu_bar, total.radius);
    nd.leaf_instance = kInvalidNode;
    nd.leaf_triangle = kInvalidNode;
    nd.area = 0.0f;
    std::thread t;
    bool threaded = false;
    if (split >= kParallelMin && n - split >= kParallelMin && take_thread()) {
      try {
        t = std::thread([=] { build(L, split, idx, l); });
        threaded = true;
      } catch (const std::exception&) {
        spare_.fetch_add(1);  // no thread could be started: build both halves here
      }
    }
    if (threaded) {
      build(L + split, n - split, idx, r);
      t.join();
      spare_.fetch_add(1);
    } else {
      build(L, split, idx, l);
      build(L + split, n - split, idx, r);
    }
  }

 private:
  static void fill_cluster(LightNodeHost& nd, float flux, V3 mu, float s2, V3 nu_bar, float radius) {
    nd.flux = flux;
    nd.mu[0] = mu.x; nd.mu[1] = mu.y; nd.mu[2] = mu.z;
    nd.sigma_s2 = s2;
    nd.lambda = vmf_axis_length_to_sharpness(length(nu_bar));
    V3 nu = dot(nu_bar, nu_bar) > 0.0f ? normalize(nu_bar) : V3{0, 0, 1};
    nd.nu[0] = nu.x; nd.nu[1] = nu.y; nd.nu[2] = nu.z;
    nd.radius = radius;
  }

  bool take_thread() {
    int k = spare_.load();
    while (k > 0)
      if (spare_.compare_exchange_weak(k, k - 1)) return true;
    return false;
  }

  void put_leaf(const Leaf& l, uint32_t parent, uint32_t idx) {
    LightNodeHost nd{};
    fill_cluster(nd, l.flux, l.mu, l.sigma_s2, l.nu_bar, l.radius);
    nd.left = nd.right = kInvalidNode;
    nd.parent = parent;
    nd.leaf_instance = l.inst;
    nd.leaf_triangle = l.tri;
    nd.area = l.area;
    nodes_[idx] = nd;
  }

  static void sort_axis(Leaf* L, size_t n, int axis) {
    std::sort(L, L + n, [axis](const Leaf& a, const Leaf& b) {
      float ca = comp(a.centroid, axis), cb = comp(b.centroid, axis);
      if (ca < cb) return true;
      if (cb < ca) return false;
      return a.order < b.order;
    });
  }

  // builder.rs:661-765
  static bool best_split(Leaf* L, size_t n, const Cluster& total, size_t* out) {
    if (n < 2) return false;
    V3 cmin{INFINITY, INFINITY, INFINITY}, cmax{-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = 0; i < n; ++i) { cmin = vmin(cmin, L[i].centroid); cmax = vmax(cmax, L[i].centroid); }
    V3 ext = sub(cmax, cmin);
    if (std::fmax(std::fmax(ext.x, ext.y), ext.z) <= 0.0f) return false;
    float parent_area = std::fmax(std::fmax(total.aabb.area(), 0.0f), 1.0e-30f);
    float parent_cone = std::fmax(total.cone.measure(), 1.0e-30f);
    float best_cost = INFINITY;
    int best_axis = 0;
    size_t best_split = 0;
    for (int axis = 0; axis < 3; ++axis) {
      if (comp(ext, axis) <= 0.0f) continue;
      Cluster bins[kBins];
      uint32_t count[kBins] = {0};
      float inv = (float)kBins / comp(ext, axis);
      float lo = comp(cmin, axis);
      for (size_t i = 0; i < n; ++i) {
        float key = (comp(L[i].centroid, axis) - lo) * inv;
        size_t k = std::isnan(key) || key <= 0.0f ? 0 : (key >= 4294967295.0f ? (size_t)kBins - 1 : (size_t)key);
        k = std::min<size_t>(k, kBins - 1);
        bins[k].merge_leaf(L[i]);
        count[k] += 1;
      }
      Cluster prefix[kBins], suffix[kBins];
      uint32_t pc[kBins], sc[kBins];
      Cluster acc;
      uint32_t ac = 0;
      for (int i = 0; i < kBins; ++i) { acc.merge_with(bins[i]); ac += count[i]; prefix[i] = acc; pc[i] = ac; }
      Cluster sacc;
      uint32_t scn = 0;
      for (int i = kBins - 1; i >= 0; --i) { sacc.merge_with(bins[i]); scn += count[i]; suffix[i] = sacc; sc[i] = scn; }
      for (int s = 1; s < kBins; ++s) {
        if (pc[s - 1] == 0 || sc[s] == 0) continue;
        const Cluster& l = prefix[s - 1];
        const Cluster& r = suffix[s];
        float cost = l.flux * std::fmax(l.aabb.area(), 0.0f) * l.cone.measure() +
                     r.flux * std::fmax(r.aabb.area(), 0.0f) * r.cone.measure();
        if (!std::isfinite(cost)) continue;
        float norm = cost / (parent_area * parent_cone);
        if (norm < best_cost) { best_cost = norm; best_axis = axis; best_split = pc[s - 1]; }
      }
    }
    if (!std::isfinite(best_cost)) return false;
    sort_axis(L, n, best_axis);
    *out = std::min(std::max<size_t>(best_split, 1), n - 1);
    return true;
  }

  std::vector<LightNodeHost>& nodes_;
  std::atomic<int> spare_;
};

}  // namespace

void make_spot_light(const float* position, const float* direction, const float* color, float intensity,
                     float total_width_rad, float falloff_start_rad, HostSpotLight* out) {
  const float pi = 3.14159274101257324f;  // f32::consts::PI
  const float total_width = std::fmin(std::fmax(total_width_rad, 0.0f), pi);
  const float falloff_start = std::fmin(std::fmax(falloff_start_rad, 0.0f), total_width);
  const V3 d{direction[0], direction[1], direction[2]};
  const V3 n = mulv(d, 1.0f / length(d));  // glam normalize
  for (int k = 0; k < 3; ++k) {
    out->position[k] = position[k];
    out->color[k] = color[k];
  }
  out->direction[0] = n.x;
  out->direction[1] = n.y;
  out->direction[2] = n.z;
  out->intensity = intensity;
  out->cos_total_width = std::cos(total_width);
  out->cos_falloff_start = std::cos(falloff_start);
}

// Scene::register_area_light_triangles (scene/mod.rs:649-683): the area-light
// registry BDPT samples its light subpaths from.
void register_area_lights(const HostSceneView& s, std::vector<HostAreaLight>* out, float* weight_sum) {
  out->clear();
  float sum = 0.0f;
  for (uint32_t ii = 0; ii < s.num_instances; ++ii) {
    const HostInstance& inst = s.instances[ii];
    const HostMaterial& mat = s.materials[inst.material];
    if (!mat.may_emit()) continue;
    const float max_em = mat.max_emission();
    if (max_em <= 0.0f) continue;
    const HostMesh& m = s.meshes[inst.mesh];
    for (uint32_t t = 0; t < m.num_triangles; ++t) {
      V3 p[3];
      for (int k = 0; k < 3; ++k) {
        const float* v = m.positions + 3 * (size_t)m.indices[3 * (size_t)t + k];
        float w[3];
        transform_point_glam(inst.local_to_world, v, w);
        p[k] = V3{w[0], w[1], w[2]};
      }
      const float area = 0.5f * length(cross(sub(p[1], p[0]), sub(p[2], p[0])));
      const float weight = area * max_em;
      if (weight <= 0.0f) continue;
      sum += weight;
      out->push_back(HostAreaLight{ii, t, area, weight, sum});
    }
  }
  *weight_sum = sum;
}

// Scene::register_area_light_triangles (scene/mod.rs:649-683) + build_light_tree
// (builder.rs:58-99): emitters in instance/triangle order, leaves with flux > 0.
bool build_light_tree_host(const HostSceneView& s, LightTreeHost* out, int threads) {
  out->nodes.clear();
  out->root = kInvalidNode;
  std::vector<Leaf> leaves;
  for (uint32_t ii = 0; ii < s.num_instances; ++ii) {
    const HostInstance& inst = s.instances[ii];
    const HostMaterial& mat = s.materials[inst.material];
    float max_em = mat.max_emission();
    if (!mat.may_emit() || max_em <= 0.0f) continue;
    const HostMesh& m = s.meshes[inst.mesh];
    for (uint32_t t = 0; t < m.num_triangles; ++t) {
      V3 p[3];
      for (int k = 0; k < 3; ++k) {
        const float* v = m.positions + 3 * (size_t)m.indices[3 * (size_t)t + k];
        float w[3];
        transform_point_glam(inst.local_to_world, v, w);
        p[k] = V3{w[0], w[1], w[2]};
      }
      // registration weight: triangle_area * max_emission (scene/mod.rs:668-673)
      float reg_area = 0.5f * length(cross(sub(p[1], p[0]), sub(p[2], p[0])));
      if (!(reg_area * max_em > 0.0f)) continue;
      // triangle_leaf (builder.rs:127-187)
      V3 e1 = sub(p[1], p[0]), e2 = sub(p[2], p[0]);
      V3 gn = cross(e1, e2);
      float area_doubled = length(gn);
      if (area_doubled <= 0.0f) continue;
      V3 n_geom = divs(gn, area_doubled);
      float area = 0.5f * area_doubled;
      float phi = max_em * area;
      if (!(phi > 0.0f)) continue;
      Leaf L;
      L.inst = ii;
      L.tri = t;
      L.flux = phi;
      L.mu = divs(add(add(p[0], p[1]), p[2]), 3.0f);
      L.sigma_s2 = (dot(e1, e1) + dot(e2, e2) - dot(e1, e2)) / 18.0f;
      L.radius = std::fmax(std::fmax(length(sub(p[0], L.mu)), length(sub(p[1], L.mu))), length(sub(p[2], L.mu)));
      L.aabb.lo = vmin(vmin(p[0], p[1]), p[2]);
      L.aabb.hi = vmax(vmax(p[0], p[1]), p[2]);
      L.nu_bar = mulv(n_geom, 0.5f);
      L.cone = Cone{n_geom, 0.0f, kPi * 0.5f, true};
      L.centroid = L.mu;
      L.area = reg_area;
      L.order = (uint32_t)leaves.size();
      leaves.push_back(L);
    }
  }
  // point_leaf / spot_leaf (builder.rs:189-242), kept when their flux is > 0
  for (uint32_t i = 0; i < s.num_points; ++i) {
    const HostPointLight& pl = s.points[i];
    const V3 c{pl.color[0], pl.color[1], pl.color[2]};
    const float phi = std::fmax(luminance(c) * pl.intensity, 0.0f);
    if (!(phi > 0.0f)) continue;
    Leaf L;
    L.inst = kLeafPoint;
    L.tri = i;
    L.flux = phi;
    L.mu = V3{pl.position[0], pl.position[1], pl.position[2]};
    L.sigma_s2 = 0.0f;
    L.nu_bar = V3{0, 0, 0};
    L.aabb.lo = L.mu;
    L.aabb.hi = L.mu;
    L.radius = 0.0f;
    L.cone = Cone{V3{0, 0, 1}, kPi, 0.0f, true};  // undirected: theta_o = pi
    L.centroid = L.mu;
    L.area = 0.0f;
    L.order = (uint32_t)leaves.size();
    leaves.push_back(L);
  }
  for (uint32_t i = 0; i < s.num_spots; ++i) {
    const HostSpotLight& sl = s.spots[i];
    const V3 c{sl.color[0], sl.color[1], sl.color[2]};
    const float phi = std::fmax(luminance(c) * sl.intensity, 0.0f);
    if (!(phi > 0.0f)) continue;
    const V3 dir{sl.direction[0], sl.direction[1], sl.direction[2]};
    const float cos_total = std::fmin(std::fmax(sl.cos_total_width, -1.0f), 1.0f);
    const float mean_len = std::fmin(std::fmax((1.0f + cos_total) * 0.5f, 0.0f), 1.0f);
    Leaf L;
    L.inst = kLeafSpot;
    L.tri = i;
    L.flux = phi;
    L.mu = V3{sl.position[0], sl.position[1], sl.position[2]};
    L.sigma_s2 = 0.0f;
    L.nu_bar = mul(mean_len, dir);
    L.aabb.lo = L.mu;
    L.aabb.hi = L.mu;
    L.radius = 0.0f;
    L.cone = Cone{dir, 0.0f, std::acos(cos_total), true};
    L.centroid = L.mu;
    L.area = 0.0f;
    L.order = (uint32_t)leaves.size();
    leaves.push_back(L);
  }
  if (leaves.empty()) return false;
  if (threads <= 0) {
    const unsigned hc = std::thread::hardware_concurrency();
    threads = hc ? (int)hc : 1;
  }
  out->nodes.assign(2 * leaves.size() - 1, LightNodeHost{});
  TreeBuilder b(&out->nodes, threads);
  b.build(leaves.data(), leaves.size(), kInvalidNode, 0);
  out->root = 0;
  // fixup_parents (builder.rs:628-644)
  out->nodes[out->root].parent = kInvalidNode;
  for (uint32_t i = 0; i < out->nodes.size(); ++i) {
    if (out->nodes[i].left != kInvalidNode) out->nodes[out->nodes[i].left].parent = i;
    if (out->nodes[i].right != kInvalidNode) out->nodes[out->nodes[i].right].parent = i;
  }
  return true;
}

}  // namespace tpt
