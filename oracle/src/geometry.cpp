// Oracle: triangle test, QBVH builder and scene queries.
#include "geometry.h"
#include "sampler.h"

namespace orc {

// crates/renderer/src/math/ray.rs:107-209 (pbrt-v4 watertight test with f64 fallback)
bool intersect_triangle(const Ray& ray, float t_max, const Vec3& v0, const Vec3& v1, const Vec3& v2,
                        TriHit* out) {
  if (length_squared(cross(v2 - v0, v1 - v0)) == 0.0f) return false;
  Vec3 p0t = v0 - ray.origin, p1t = v1 - ray.origin, p2t = v2 - ray.origin;
  int kz = max_component_index(vabs(ray.direction));
  int kx = kz + 1; if (kx == 3) kx = 0;
  int ky = kx + 1; if (ky == 3) ky = 0;
  Vec3 d(ray.direction[kx], ray.direction[ky], ray.direction[kz]);
  if (d.z == 0.0f) return false;
  p0t = Vec3(p0t[kx], p0t[ky], p0t[kz]);
  p1t = Vec3(p1t[kx], p1t[ky], p1t[kz]);
  p2t = Vec3(p2t[kx], p2t[ky], p2t[kz]);
  float sx = -d.x / d.z, sy = -d.y / d.z, sz = 1.0f / d.z;
  p0t.x += sx * p0t.z; p0t.y += sy * p0t.z;
  p1t.x += sx * p1t.z; p1t.y += sy * p1t.z;
  p2t.x += sx * p2t.z; p2t.y += sy * p2t.z;
  float e0 = difference_of_products(p1t.x, p2t.y, p1t.y, p2t.x);
  float e1 = difference_of_products(p2t.x, p0t.y, p2t.y, p0t.x);
  float e2 = difference_of_products(p0t.x, p1t.y, p0t.y, p1t.x);
  if (e0 == 0.0f || e1 == 0.0f || e2 == 0.0f) {
    e0 = (float)((double)p2t.y * (double)p1t.x - (double)p2t.x * (double)p1t.y);
    e1 = (float)((double)p0t.y * (double)p2t.x - (double)p0t.x * (double)p2t.y);
    e2 = (float)((double)p1t.y * (double)p0t.x - (double)p1t.x * (double)p0t.y);
  }
  if ((e0 < 0.0f || e1 < 0.0f || e2 < 0.0f) && (e0 > 0.0f || e1 > 0.0f || e2 > 0.0f)) return false;
  float det = e0 + e1 + e2;
  if (det == 0.0f) return false;
  p0t.z *= sz; p1t.z *= sz; p2t.z *= sz;
  float t_scaled = e0 * p0t.z + e1 * p1t.z + e2 * p2t.z;
  if ((det < 0.0f && (t_scaled >= 0.0f || t_scaled < t_max * det)) ||
      (det > 0.0f && (t_scaled <= 0.0f || t_scaled > t_max * det)))
    return false;
  float inv_det = 1.0f / det;
  float b0 = e0 * inv_det, b1 = e1 * inv_det, b2 = e2 * inv_det;
  float t = t_scaled * inv_det;
  float max_zt = max_element(vabs(Vec3(p0t.z, p1t.z, p2t.z)));
  float delta_z = gamma_n(3) * max_zt;
  float max_xt = max_element(vabs(Vec3(p0t.x, p1t.x, p2t.x)));
  float max_yt = max_element(vabs(Vec3(p0t.y, p1t.y, p2t.y)));
  float delta_x = gamma_n(5) * (max_xt + max_zt);
  float delta_y = gamma_n(5) * (max_yt + max_zt);
  float delta_e = 2.0f * (gamma_n(2) * max_xt * max_yt + delta_y * max_xt + delta_x * max_yt);
  float max_e = max_element(vabs(Vec3(e0, e1, e2)));
  float delta_t = 3.0f * (gamma_n(3) * max_e * max_zt + delta_e * max_zt + delta_z * max_e) * std::fabs(inv_det);
  if (t <= delta_t) return false;
  out->t = t;
  out->bary = Vec3(b0, b1, b2);
  return true;
}

// ---------------------------------------------------------------------------
// QBVH builder: crates/renderer/src/qbvh.rs:144-549.  The recursion is the
// reference's; rayon only parallelises it and its reductions (bounds union,
// integer counts) are order independent.  `sort_unstable_by` in the forced
// median split (qbvh.rs:282-286) has no defined order for equal centroids; here
// equal centroids are ordered by primitive index.

namespace {
constexpr int kBins = 16;
constexpr size_t kTargetLeaf = 4;
constexpr size_t kMaxLeaf = 16;

struct BPrim {
  uint32_t index;
  Bounds bounds;
  Vec3 centroid;
};

struct BNode {
  Bounds bounds;
  uint32_t count = 0;  // leaf when children empty
  std::vector<BNode> children;
  bool leaf = true;
};

struct Bin {
  Bounds bounds;
  uint32_t count = 0;
};

struct BinSplit {
  int axis;
  float cmin, cmax;
  int bin_split;
  float cost;
};

Bounds bounds_of(const BPrim* p, size_t n) {
  Bounds b;
  for (size_t i = 0; i < n; ++i) b = b.unite(p[i].bounds);
  return b;
}
Bounds centroid_bounds_of(const BPrim* p, size_t n) {
  Bounds b;
  for (size_t i = 0; i < n; ++i) {
    Bounds c; c.min = p[i].centroid; c.max = p[i].centroid;
    b = b.unite(c);
  }
  return b;
}
size_t bin_index(float c, float cmin, float inv) {
  float raw = (c - cmin) * inv;
  float cl = raw;
  if (!(cl >= 0.0f)) cl = std::isnan(raw) ? raw : 0.0f;  // Rust clamp keeps NaN
  if (cl > (float)(kBins - 1)) cl = (float)(kBins - 1);
  if (std::isnan(cl)) return 0;  // `as usize` maps NaN to 0
  return (size_t)cl;
}

bool evaluate_bins(const Bin* bins, float parent_area, int* split_out, float* cost_out) {
  Bounds lb[kBins], rb[kBins];
  uint32_t lc[kBins], rc[kBins];
  Bounds acc; uint32_t ac = 0;
  for (int i = 0; i < kBins; ++i) { acc = acc.unite(bins[i].bounds); ac += bins[i].count; lb[i] = acc; lc[i] = ac; }
  acc = Bounds(); ac = 0;
  for (int i = kBins - 1; i >= 0; --i) { acc = acc.unite(bins[i].bounds); ac += bins[i].count; rb[i] = acc; rc[i] = ac; }
  (void)rc;
  uint32_t total = lc[kBins - 1];
  if (total <= 1) return false;
  float best = kInf;
  int best_split = -1;
  for (int s = 0; s < kBins - 1; ++s) {
    uint32_t nl = lc[s], nr = total - nl;
    if (nl == 0 || nr == 0) continue;
    float al = lb[s].surface_area(), ar = rb[s + 1].surface_area();
    float cost = 1.0f + 1.0f * (al * (float)nl + ar * (float)nr) / parent_area;
    if (cost < best) { best = cost; best_split = s; }
  }
  if (best_split < 0) return false;
  *split_out = best_split;
  *cost_out = best;
  return true;
}

bool find_best_binary_split(const BPrim* p, size_t n, const Bounds& parent, BinSplit* out) {
  if (n <= 1) return false;
  Bounds cb = centroid_bounds_of(p, n);
  float parent_area = fmax_num(parent.surface_area(), 1.0e-30f);
  bool have = false;
  for (int axis = 0; axis < 3; ++axis) {
    float cmin = cb.min[axis], cmax = cb.max[axis];
    if (cmax - cmin <= 0.0f) continue;
    Bin bins[kBins];
    float extent = fmax_num(cmax - cmin, 1.0e-30f);
    float inv = (float)kBins / extent;
    for (size_t i = 0; i < n; ++i) {
      size_t b = bin_index(p[i].centroid[axis], cmin, inv);
      bins[b].bounds = bins[b].bounds.unite(p[i].bounds);
      bins[b].count += 1;
    }
    int s; float cost;
    if (!evaluate_bins(bins, parent_area, &s, &cost)) continue;
    if (!have || cost < out->cost) {
      *out = BinSplit{axis, cmin, cmax, s, cost};
      have = true;
    }
  }
  return have;
}

size_t partition_in_place(BPrim* p, size_t n, const BinSplit& sp) {
  float extent = fmax_num(sp.cmax - sp.cmin, 1.0e-30f);
  float inv = (float)kBins / extent;
  size_t left = 0, right = n;
  while (left < right) {
    size_t b = bin_index(p[left].centroid[sp.axis], sp.cmin, inv);
    if ((int)b <= sp.bin_split) {
      ++left;
    } else {
      --right;
      std::swap(p[left], p[right]);
    }
  }
  return left;
}

BNode make_leaf(const Bounds& b, size_t n) { BNode l; l.bounds = b; l.count = (uint32_t)n; l.leaf = true; return l; }

BNode build_node(BPrim* p, size_t n);
std::vector<BNode> split_into_children(BPrim* p, size_t n);

BNode make_leaf_or_force_split(BPrim* p, size_t n, const Bounds& b) {
  if (n <= kMaxLeaf) return make_leaf(b, n);
  size_t mid = n / 2;
  Vec3 e = b.extent();
  int axis = (e.x >= e.y && e.x >= e.z) ? 0 : (e.y >= e.z ? 1 : 2);
  std::sort(p, p + n, [axis](const BPrim& a, const BPrim& c) {
    float ca = a.centroid[axis], cc = c.centroid[axis];
    if (ca < cc) return true;
    if (cc < ca) return false;
    return a.index < c.index;
  });
  BNode node; node.bounds = b; node.leaf = false;
  node.children = split_into_children(p, mid);
  auto r = split_into_children(p + mid, n - mid);
  for (auto& c : r) node.children.push_back(std::move(c));
  return node;
}

BNode build_node(BPrim* p, size_t n) {
  Bounds b = bounds_of(p, n);
  if (n <= kTargetLeaf) return make_leaf(b, n);
  BinSplit sp;
  if (!find_best_binary_split(p, n, b, &sp)) return make_leaf_or_force_split(p, n, b);
  if (sp.cost >= 1.0f * (float)n && n <= kMaxLeaf) return make_leaf(b, n);
  size_t mid = partition_in_place(p, n, sp);
  if (mid == 0 || mid == n) return make_leaf_or_force_split(p, n, b);
  BNode node; node.bounds = b; node.leaf = false;
  node.children = split_into_children(p, mid);
  auto r = split_into_children(p + mid, n - mid);
  for (auto& c : r) node.children.push_back(std::move(c));
  return node;
}

std::vector<BNode> split_into_children(BPrim* p, size_t n) {
  std::vector<BNode> out;
  if (n == 0) return out;
  Bounds b = bounds_of(p, n);
  if (n <= kTargetLeaf) { out.push_back(build_node(p, n)); return out; }
  BinSplit sp;
  if (!find_best_binary_split(p, n, b, &sp)) { out.push_back(build_node(p, n)); return out; }
  if (sp.cost >= 1.0f * (float)n && n <= kMaxLeaf) { out.push_back(build_node(p, n)); return out; }
  size_t mid = partition_in_place(p, n, sp);
  if (mid == 0 || mid == n) { out.push_back(build_node(p, n)); return out; }
  out.push_back(build_node(p, mid));
  out.push_back(build_node(p + mid, n - mid));
  return out;
}

QbvhNode empty_node() {
  QbvhNode n;
  for (int s = 0; s < 4; ++s) {
    for (int a = 0; a < 3; ++a) { n.b[a][s] = kInf; n.b[3 + a][s] = -kInf; }
    n.children[s] = kEmptyChild;
  }
  n.valid_mask = 0;
  n.pad[0] = n.pad[1] = n.pad[2] = 0;
  return n;
}

// qbvh.rs:491-516 (pre-order numbering, children in order)
uint32_t flatten(const BNode& node, uint32_t prim_offset, std::vector<QbvhNode>& nodes, uint32_t* total) {
  if (node.leaf) { *total = node.count; return encode_leaf(prim_offset, node.count); }
  uint32_t idx = (uint32_t)nodes.size();
  nodes.push_back(empty_node());
  QbvhNode nn = empty_node();
  uint32_t cur = prim_offset;
  for (size_t i = 0; i < node.children.size(); ++i) {
    const BNode& ch = node.children[i];
    uint32_t cnt = 0;
    uint32_t ref = flatten(ch, cur, nodes, &cnt);
    nn.b[0][i] = ch.bounds.min.x; nn.b[1][i] = ch.bounds.min.y; nn.b[2][i] = ch.bounds.min.z;
    nn.b[3][i] = ch.bounds.max.x; nn.b[4][i] = ch.bounds.max.y; nn.b[5][i] = ch.bounds.max.z;
    nn.children[i] = ref;
    nn.valid_mask |= 1u << i;
    cur += cnt;
  }
  nodes[idx] = nn;
  *total = cur - prim_offset;
  return idx;
}
}  // namespace

bool build_qbvh(const std::vector<Bounds>& prim_bounds, Qbvh* out) {
  out->nodes.clear();
  out->primitive_indices.clear();
  if (prim_bounds.empty()) return false;
  std::vector<BPrim> prims(prim_bounds.size());
  for (size_t i = 0; i < prims.size(); ++i) {
    prims[i].index = (uint32_t)i;
    prims[i].bounds = prim_bounds[i];
    prims[i].centroid = prim_bounds[i].center();
  }
  BNode root = build_node(prims.data(), prims.size());
  out->primitive_indices.resize(prims.size());
  for (size_t i = 0; i < prims.size(); ++i) out->primitive_indices[i] = prims[i].index;
  uint32_t total = 0;
  flatten(root, 0, out->nodes, &total);
  return true;
}

// scene/mod.rs:869-893
Bounds transform_bounds(const Bounds& b, const Mat4& m) {
  Vec3 corners[8] = {
      Vec3(b.min.x, b.min.y, b.min.z), Vec3(b.min.x, b.min.y, b.max.z), Vec3(b.min.x, b.max.y, b.min.z),
      Vec3(b.min.x, b.max.y, b.max.z), Vec3(b.max.x, b.min.y, b.min.z), Vec3(b.max.x, b.min.y, b.max.z),
      Vec3(b.max.x, b.max.y, b.min.z), Vec3(b.max.x, b.max.y, b.max.z)};
  Vec3 first = m.transform_point3(corners[0]);
  Bounds r; r.min = first; r.max = first;
  for (int i = 1; i < 8; ++i) {
    Vec3 c = m.transform_point3(corners[i]);
    r.min = vmin(r.min, c);
    r.max = vmax(r.max, c);
  }
  return r;
}

// scene/mod.rs:340-395 and 686-723
bool Geometry::closest_hit(const Ray& ray, SceneHit* hit, TraversalStats* st, AuxRng* aux) const {
  *hit = SceneHit();
  if (instances.empty()) return false;
  bool found = false;
  traverse_qbvh(
      tlas, ray, kInf,
      [&](uint32_t offset, uint32_t count, float cur_t_max) -> float {
        float t_max = cur_t_max;
        for (uint32_t oi = offset; oi < offset + count; ++oi) {
          uint32_t ii = tlas.primitive_indices[oi];
          const Instance& inst = instances[ii];
          Ray lr;
          lr.origin = inst.world_to_local.transform_point3(ray.origin);
          lr.direction = inst.world_to_local.transform_vector3(ray.direction);
          const Mesh& mesh = meshes[inst.mesh_index];
          if (st) st->instances++;
          // Material::has_alpha_test of the instance's material
          const float alpha = aux && !this->alpha.empty() ? this->alpha[ii] : 1.0f;
          bool mesh_found = false;
          TriHit best{};
          uint32_t best_tri = 0;
          traverse_qbvh(
              mesh.qbvh, lr, t_max,
              [&](uint32_t off2, uint32_t cnt2, float cur2) -> float {
                float tm = cur2;
                for (uint32_t k = off2; k < off2 + cnt2; ++k) {
                  uint32_t tri = mesh.qbvh.primitive_indices[k];
                  Vec3 v[3];
                  mesh.triangle_positions(tri, v);
                  if (st) st->triangles++;
                  TriHit h;
                  if (intersect_triangle(lr, tm, v[0], v[1], v[2], &h)) {
                    // any_hit: alpha >= 1 || u < alpha (alpha = the clamped opacity)
                    if (alpha < 1.0f && !(aux->next_f32() < alpha)) continue;
                    tm = h.t;
                    best = h;
                    best_tri = tri;
                    mesh_found = true;
                  }
                }
                return tm;
              },
              nullptr, st);
          if (mesh_found) {
            t_max = best.t;
            hit->instance = (int32_t)ii;
            hit->triangle = (int32_t)best_tri;
            hit->t = best.t;
            hit->bary = best.bary;
            found = true;
          }
        }
        return t_max;
      },
      nullptr, st);
  return found;
}

bool Geometry::any_hit(const Ray& ray, float t_max_in, SceneHit* hit, TraversalStats* st) const {
  *hit = SceneHit();
  if (instances.empty()) return false;
  bool stop = false;
  traverse_qbvh(
      tlas, ray, t_max_in,
      [&](uint32_t offset, uint32_t count, float cur_t_max) -> float {
        for (uint32_t oi = offset; oi < offset + count && !stop; ++oi) {
          uint32_t ii = tlas.primitive_indices[oi];
          const Instance& inst = instances[ii];
          Ray lr;
          lr.origin = inst.world_to_local.transform_point3(ray.origin);
          lr.direction = inst.world_to_local.transform_vector3(ray.direction);
          const Mesh& mesh = meshes[inst.mesh_index];
          if (st) st->instances++;
          traverse_qbvh(
              mesh.qbvh, lr, cur_t_max,
              [&](uint32_t off2, uint32_t cnt2, float cur2) -> float {
                for (uint32_t k = off2; k < off2 + cnt2; ++k) {
                  uint32_t tri = mesh.qbvh.primitive_indices[k];
                  Vec3 v[3];
                  mesh.triangle_positions(tri, v);
                  if (st) st->triangles++;
                  TriHit h;
                  if (intersect_triangle(lr, cur2, v[0], v[1], v[2], &h)) {
                    hit->instance = (int32_t)ii;
                    hit->triangle = (int32_t)tri;
                    hit->t = h.t;
                    hit->bary = h.bary;
                    stop = true;
                    return cur2;
                  }
                }
                return cur2;
              },
              &stop, st);
        }
        return cur_t_max;
      },
      &stop, st);
  return stop;
}

}  // namespace orc
