// SG light tree on the device: spherical-Gaussian math (math/sg.rs), the
// node-to-SG-light projection and diffuse importance (light_tree/lobe.rs:233-283),
// stochastic descent and reverse pmf (light_tree/traversal.rs:26-143).
#pragma once
#include "render_types.h"
#include "vmath.cuh"

namespace tpt {

constexpr float kSgSharpnessMaxF = 2.1990233e12f;  // 2^41 (sg.rs:26)
constexpr float kFltMinPositive = 1.17549435e-38f;
constexpr float kFltEpsilon = 1.1920929e-7f;

using DevLightNode = DevLightNodeRec;

struct SgLobe {
  V3 axis;
  float sharpness;
  float log_amplitude;
};

// sg.rs:51-58 (Higham)
__device__ __forceinline__ float expm1_over_x(float x) {
  const float u = expf(x);
  if (u == 1.0f) return 1.0f;
  const float y = u - 1.0f;
  return fabsf(x) < 1.0f ? y / logf(u) : y / x;
}

// sg.rs:62-90: the VSGL polynomial erf (restated coefficients of a published approximation)
__device__ __forceinline__ float sg_erf(float x) {
  if (fabsf(x) >= 4.0f) return copysignf(1.0f, x);
  if (fabsf(x) > 1.0f) {
    const float a = fabsf(x);
    const float p = ((((((2.5890768e-5f * a + -5.648746e-4f) * a + 5.6679556e-3f) * a + -3.5175983e-2f) * a +
                       1.5432939e-1f) * a + 9.156747e-1f) * a + 1.6284595f) * a;
    const float y = 1.0f - exp2f(-p);
    return copysignf(y, x);
  }
  const float x2 = x * x;
  return (((((-5.5885315e-4f * x2 + 4.9073556e-3f) * x2 + -2.6703065e-2f) * x2 + 1.1279922e-1f) * x2 +
           -3.76123e-1f) * x2 + 1.12837916709551257390f) * x;  // FRAC_2_SQRT_PI
}

// sg.rs:117-119
__device__ __forceinline__ float sg_integral(float k) { return 4.0f * kPiF * expm1_over_x(-2.0f * k); }

// sg.rs:134-151
__device__ __forceinline__ SgLobe sg_product(V3 a1, float k1, V3 a2, float k2) {
  const V3 axis = a1 * k1 + a2 * k2;
  const float sharp = length(axis);
  const V3 d = a1 - a2;
  const float len2 = dot(d, d);
  const float denom = fmaxf(sharp + k1 + k2, kFltMinPositive);
  SgLobe l;
  l.log_amplitude = -k1 * k2 * len2 / denom;
  l.axis = sharp > kFltMinPositive ? axis / sharp : V3{0.0f, 0.0f, 1.0f};
  l.sharpness = sharp;
  return l;
}

// sg.rs:239-278
__device__ __forceinline__ float upper_sg_cc_over_2pi(float s) {
  if (s <= 0.5f) {
    return (((((((-1.0f / 362880.0f) * s + 1.0f / 40320.0f) * s - 1.0f / 5040.0f) * s + 1.0f / 720.0f) * s -
              1.0f / 120.0f) * s + 1.0f / 24.0f) * s - 1.0f / 6.0f) * s + 0.5f;
  }
  return (expm1f(-s) + s) / (s * s);
}
__device__ __forceinline__ float lower_sg_cc_over_2pi(float s) {
  const float e = expf(-s);
  if (s <= 0.5f) {
    return e * (((((((((1.0f / 403200.0f) * s - 1.0f / 45360.0f) * s + 1.0f / 5760.0f) * s - 1.0f / 840.0f) * s +
                     1.0f / 144.0f) * s - 1.0f / 30.0f) * s + 1.0f / 8.0f) * s - 1.0f / 3.0f) * s + 0.5f);
  }
  return e * (-expm1f(-s) - s * e) / (s * s);
}

// sg.rs:288-306
__device__ __forceinline__ float sg_clamped_cosine_product_over_pi(float z, float s) {
  const float t = s * sqrtf(0.5f * ((s + 2.736083f) * s + 17.021297f) / (((s + 4.0100827f) * s + 15.219156f) * s + 76.0879f));
  const float tz = t * z;
  const float inv_sqrt_pi = 0.5641896f;
  const float clamp_min = 0.5f * kFltEpsilon;
  float lerp = 0.5f * (z * (1.0f - sg_erf(-tz)) + (1.0f - sg_erf(t))) -
               0.5f * inv_sqrt_pi * expf(-tz * tz) * expm1f(t * t * (z * z - 1.0f)) / fmaxf(t, kFltMinPositive);
  lerp = clampf(lerp, clamp_min, 1.0f);
  const float lower = lower_sg_cc_over_2pi(s);
  const float upper = upper_sg_cc_over_2pi(s);
  return 2.0f * (lower + (upper - lower) * lerp);
}

// lobe.rs:233-272: the cluster as an SG light seen from (p, n).  Returns 0 weight for "None".
__device__ __forceinline__ bool sg_light_for_node(V3 p, V3 n, const DevLightNode& node, float& w, SgLobe& lobe) {
  if (node.flux <= 0.0f) return false;
  const V3 d = V3{node.mu[0], node.mu[1], node.mu[2]} - p;
  const float r2 = dot(d, d);
  if (r2 <= 0.0f) return false;
  const float inv_r = 1.0f / sqrtf(r2);
  const float cos_below = fmaxf(-(dot(n, d)) * inv_r, 0.0f);
  const float bound_var = 0.5f * node.radius * node.radius;
  float sigma2 = node.sigma_s2 * (1.0f - cos_below) + bound_var * cos_below;
  const float min_sigma2 = r2 / kSgSharpnessMaxF;
  if (sigma2 < min_sigma2) sigma2 = min_sigma2;
  const V3 axis = d * inv_r;
  const float sharp = clampf(r2 / sigma2, 0.0f, kSgSharpnessMaxF);
  lobe = sg_product(-V3{node.nu[0], node.nu[1], node.nu[2]}, node.lambda, axis, sharp);
  const float sg_norm = fmaxf(sg_integral(node.lambda), 1.0e-30f);
  const float w_amp = node.flux / (2.0f * kPiF * sigma2 * sg_norm);
  w = w_amp * expf(lobe.log_amplitude);
  return isfinite(w) && w > 0.0f;
}

// lobe.rs:276-283
__device__ __forceinline__ float diffuse_importance(float rho, V3 n, float w, const SgLobe& lobe) {
  if (rho <= 0.0f || w <= 0.0f) return 0.0f;
  const float cosine = clampf(dot(lobe.axis, n), -1.0f, 1.0f);
  const float integral = sg_clamped_cosine_product_over_pi(cosine, lobe.sharpness) * kPiF;
  return rho * w * integral;
}

// Light-tree query of a shading point (light_tree/importance.rs:20-48).  Only
// diffuse lobes are built by the materials in scope (NormalizedLambert); a
// material without a query skips the tree (returns false from build_query).
struct TreeQuery {
  V3 p, n;
  float rho;  // luminance of the diffuse albedo
};

__device__ __forceinline__ float node_importance(const TreeQuery& q, const DevLightNode& node) {
  float w;
  SgLobe lobe;
  if (!sg_light_for_node(q.p, q.n, node, w, lobe)) return 0.0f;
  return diffuse_importance(q.rho, q.n, w, lobe);
}

__device__ __forceinline__ DevLightNode load_node(const DevLightNode* nodes, uint32_t i) {
  DevLightNode n;
  const float4* src = reinterpret_cast<const float4*>(nodes + i);
  float4* dst = reinterpret_cast<float4*>(&n);
  dst[0] = __ldg(src);
  dst[1] = __ldg(src + 1);
  dst[2] = __ldg(src + 2);
  dst[3] = __ldg(src + 3);
  return n;
}

// traversal.rs:26-92.  Returns the leaf node index (or kInvalid) and its pmf.
static __device__ __noinline__ uint32_t sample_light_tree(const DevLightNode* nodes, uint32_t root, const TreeQuery& q,
                                                      float u, float& pmf) {
  u = clampf(u, 0.0f, 1.0f - kFltEpsilon);
  uint32_t idx = root;
  pmf = 1.0f;
  for (int guard = 0; guard < 4096; ++guard) {
    const DevLightNode node = load_node(nodes, idx);
    if (node.leaf_instance != 0xFFFFFFFFu) return idx;
    const DevLightNode L = load_node(nodes, node.left), R = load_node(nodes, node.right);
    const float il = node_importance(q, L), ir = node_importance(q, R);
    const float total = il + ir;
    float p_left;
    if (total <= 0.0f) {
      const float lf = fmaxf(L.flux, 0.0f), rf = fmaxf(R.flux, 0.0f);
      const float tf = lf + rf;
      if (tf <= 0.0f) return 0xFFFFFFFFu;
      p_left = lf / tf;
      if (u < p_left) {
        u /= fmaxf(p_left, kFltMinPositive);
        pmf *= p_left;
        idx = node.left;
      } else {
        u = (u - p_left) / fmaxf(1.0f - p_left, kFltMinPositive);
        pmf *= 1.0f - p_left;
        idx = node.right;
      }
      continue;
    }
    p_left = il / total;
    if (u < p_left) {
      u /= fmaxf(p_left, kFltMinPositive);
      pmf *= p_left;
      idx = node.left;
    } else {
      u = (u - p_left) / fmaxf(1.0f - p_left, kFltMinPositive);
      pmf *= 1.0f - p_left;
      idx = node.right;
    }
    u = clampf(u, 0.0f, 1.0f - kFltEpsilon);
  }
  return 0xFFFFFFFFu;  // deeper than 4096 levels: treated as no sample
}

// traversal.rs:97-143
static __device__ __noinline__ float pdf_for_leaf(const DevLightNode* nodes, const TreeQuery& q, uint32_t leaf) {
  if (leaf == 0xFFFFFFFFu) return 0.0f;
  float pmf = 1.0f;
  uint32_t child = leaf;
  uint32_t parent = __ldg(&nodes[leaf].parent);
  for (int guard = 0; guard < 4096 && parent != 0xFFFFFFFFu; ++guard) {
    const DevLightNode P = load_node(nodes, parent);
    const DevLightNode L = load_node(nodes, P.left), R = load_node(nodes, P.right);
    const float il = node_importance(q, L), ir = node_importance(q, R);
    const float total = il + ir;
    float p_left;
    if (total <= 0.0f) {
      const float lf = fmaxf(L.flux, 0.0f), rf = fmaxf(R.flux, 0.0f);
      const float tf = lf + rf;
      if (tf <= 0.0f) return 0.0f;
      p_left = lf / tf;
    } else {
      p_left = il / total;
    }
    pmf *= (child == P.left) ? p_left : 1.0f - p_left;
    child = parent;
    parent = P.parent;
  }
  return pmf;
}

// sg.rs:314-316
__device__ __forceinline__ float luminance(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

}  // namespace tpt
