// Oracle: QBVH traversal (restates crates/renderer/src/qbvh.rs:574-675).
#pragma once

namespace orc {

// wide::f32x4::fast_min / fast_max on SSE (minps / maxps): a NaN operand in
// either lane yields the second operand.
inline float fast_min(float a, float b) { return a < b ? a : b; }
inline float fast_max(float a, float b) { return a > b ? a : b; }

// qbvh.rs:574-576
inline float safe_inv(float d) { return d == 0.0f ? kInf : 1.0f / d; }

// qbvh.rs:578-607
inline uint32_t intersect_4_aabbs(const QbvhNode& n, const Vec3& o, const Vec3& inv, float t_max,
                                  float tmin_out[4]) {
  uint32_t bits = 0;
  for (int s = 0; s < 4; ++s) {
    float t1x = (n.b[0][s] - o.x) * inv.x;
    float t2x = (n.b[3][s] - o.x) * inv.x;
    float t1y = (n.b[1][s] - o.y) * inv.y;
    float t2y = (n.b[4][s] - o.y) * inv.y;
    float t1z = (n.b[2][s] - o.z) * inv.z;
    float t2z = (n.b[5][s] - o.z) * inv.z;
    float tmin_x = fast_min(t1x, t2x), tmax_x = fast_max(t1x, t2x);
    float tmin_y = fast_min(t1y, t2y), tmax_y = fast_max(t1y, t2y);
    float tmin_z = fast_min(t1z, t2z), tmax_z = fast_max(t1z, t2z);
    float tmin = fast_max(fast_max(fast_max(tmin_x, tmin_y), tmin_z), 0.0f);
    float tmax = fast_min(fast_min(fast_min(tmax_x, tmax_y), tmax_z), t_max);
    if (tmin <= tmax) bits |= 1u << s;
    tmin_out[s] = tmin;
  }
  return bits & n.valid_mask;
}

template <class Leaf>
float traverse_qbvh(const Qbvh& q, const Ray& ray, float initial_t_max, Leaf&& leaf_cb, bool* stop,
                    TraversalStats* st) {
  if (q.nodes.empty()) {
    if (q.primitive_indices.empty()) return initial_t_max;
    return leaf_cb(0u, (uint32_t)q.primitive_indices.size(), initial_t_max);
  }
  Vec3 inv(safe_inv(ray.direction.x), safe_inv(ray.direction.y), safe_inv(ray.direction.z));
  float closest_t = initial_t_max;
  uint32_t stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    uint32_t node_index = stack[--sp];
    const QbvhNode& node = q.nodes[node_index];
    float tmin[4];
    if (st) st->nodes++;
    uint32_t bits = intersect_4_aabbs(node, ray.origin, inv, closest_t, tmin);
    if (bits == 0) continue;
    float ht[4];
    uint32_t hc[4];
    int n = 0;
    for (int s = 0; s < 4; ++s) {
      if (!(bits & (1u << s))) continue;
      ht[n] = tmin[s];
      hc[n] = node.children[s];
      ++n;
    }
    for (int i = 1; i < n; ++i) {
      int j = i;
      while (j > 0 && ht[j - 1] > ht[j]) {
        std::swap(ht[j - 1], ht[j]);
        std::swap(hc[j - 1], hc[j]);
        --j;
      }
    }
    for (int k = n - 1; k >= 0; --k) {
      uint32_t c = hc[k];
      if (c & kLeafBit) {
        uint32_t count = (c >> 24) & 0x7Fu;
        if (count == 0) continue;
        closest_t = leaf_cb(c & 0xFFFFFFu, count, closest_t);
        if (stop && *stop) return closest_t;
      } else {
        if (sp >= 128) return closest_t;  // the reference debug-asserts; never reached by built trees
        stack[sp++] = c;
      }
    }
  }
  return closest_t;
}

}  // namespace orc
