// EnvironmentLight on the device (light/environment.rs:133-239, 301-333,
// 464-525): radiance lookup, pdf and hierarchical sample warping through the
// mip pyramid built on the host (host/env_build.cpp), with the reference's
// float operation order (the transcendental functions are CUDA's).
#pragma once
#include "render_types.h"
#include "vmath.cuh"

namespace tpt {

constexpr float kEnvOneMinusEps = 1.0f - 1.1920929e-7f;  // 1 - f32::EPSILON

// glam Mat3 * Vec3 (x_axis * v.x + y_axis * v.y + z_axis * v.z), column-major m
__device__ __forceinline__ V3 env_mat_mul(const float* m, V3 v) {
  return V3{(m[0] * v.x + m[3] * v.y) + m[6] * v.z, (m[1] * v.x + m[4] * v.y) + m[7] * v.z,
            (m[2] * v.x + m[5] * v.y) + m[8] * v.z};
}

__device__ __forceinline__ V3 env_uv_to_direction(float u, float v) {
  const float phi = u * kTauF, theta = v * kPiF;
  const float st = sinf(theta);
  return V3{st * sinf(phi), cosf(theta), st * cosf(phi)};
}

__device__ __forceinline__ void env_direction_to_uv(V3 d, float& u, float& v) {
  const V3 dir = normalize_or_zero(d);
  const float y = clampf(dir.y, -1.0f, 1.0f);
  const float theta = acosf(y);
  float phi = atan2f(dir.x, dir.z);
  if (phi < 0.0f) phi += kTauF;
  u = clampf(phi / kTauF, 0.0f, 1.0f);
  v = clampf(theta / kPiF, 0.0f, 1.0f);
}

__device__ __forceinline__ uint32_t env_pixel_coord(float t, uint32_t size) {
  const float c = clampf(t, 0.0f, 1.0f);
  const uint32_t idx = (uint32_t)(c * (float)size);
  return min(idx, size - 1);
}

__device__ __forceinline__ float env_texel_weight(const DevEnvDist& d, uint32_t i, uint32_t j) {
  const uint32_t* leaf = d.levels + 3 * (d.num_levels - 1);
  return __ldg(d.weights + __ldg(leaf + 2) + (size_t)j * __ldg(leaf) + i);
}

// EnvironmentLight::radiance
__device__ __forceinline__ V3 env_radiance(const DevEnvironment& E, V3 dir) {
  float u, v;
  env_direction_to_uv(env_mat_mul(E.inv_rot, dir), u, v);
  const uint32_t i = env_pixel_coord(u, E.width), j = env_pixel_coord(v, E.height);
  const float* p = E.pixels + 3 * ((size_t)j * E.width + i);
  return V3{E.scale * __ldg(p), E.scale * __ldg(p + 1), E.scale * __ldg(p + 2)};
}

// pdf_with_distribution (solid-angle density of sampling `dir`)
__device__ __forceinline__ float env_pdf(const DevEnvironment& E, const DevEnvDist& d, V3 dir) {
  if (d.total_weight <= 0.0f) return 0.0f;
  float u, v;
  env_direction_to_uv(env_mat_mul(E.inv_rot, dir), u, v);
  const float st = sinf(v * kPiF);
  if (st <= 0.0f) return 0.0f;
  const uint32_t i = env_pixel_coord(u, E.width), j = env_pixel_coord(v, E.height);
  const float w = env_texel_weight(d, i, j);
  if (w <= 0.0f) return 0.0f;
  const float p2d = w / d.total_weight * (float)E.width * (float)E.height;
  return p2d / (kTauF * kPiF * st);
}

// hsw_step: descend from texel (i, j) of level l-1 into level l, rescaling u, v
__device__ __forceinline__ bool env_hsw_step(const DevEnvDist& d, uint32_t l, uint32_t& i, uint32_t& j, float& u,
                                             float& v) {
  const uint32_t pw = __ldg(d.levels + 3 * (l - 1)), ph = __ldg(d.levels + 3 * (l - 1) + 1);
  const uint32_t cw = __ldg(d.levels + 3 * l), chh = __ldg(d.levels + 3 * l + 1);
  const float* c = d.weights + __ldg(d.levels + 3 * l + 2);
  const uint32_t si = cw / pw, sj = chh / ph;
  uint32_t ci = i * si, cj = j * sj;
  if (sj == 2) {
    float w_top = 0.0f, w_bot = 0.0f;
    for (uint32_t di = 0; di < si; ++di) {
      w_top += __ldg(c + (size_t)cj * cw + ci + di);
      w_bot += __ldg(c + (size_t)(cj + 1) * cw + ci + di);
    }
    const float total = w_top + w_bot;
    if (total <= 0.0f) return false;
    const float p_top = w_top / total;
    if (v < p_top) {
      v = clampf(v / p_top, 0.0f, kEnvOneMinusEps);
    } else {
      v = clampf((v - p_top) / (1.0f - p_top), 0.0f, kEnvOneMinusEps);
      cj += 1;
    }
  }
  if (si == 2) {
    const float w_left = __ldg(c + (size_t)cj * cw + ci), w_right = __ldg(c + (size_t)cj * cw + ci + 1);
    const float total = w_left + w_right;
    if (total <= 0.0f) return false;
    const float p_left = w_left / total;
    if (u < p_left) {
      u = clampf(u / p_left, 0.0f, kEnvOneMinusEps);
    } else {
      u = clampf((u - p_left) / (1.0f - p_left), 0.0f, kEnvOneMinusEps);
      ci += 1;
    }
  }
  i = ci;
  j = cj;
  return true;
}

// sample_with_distribution: direction, radiance and solid-angle pdf
__device__ __forceinline__ bool env_sample(const DevEnvironment& E, const DevEnvDist& d, float us0, float us1,
                                           V3& wi, V3& radiance, float& pdf) {
  if (d.total_weight <= 0.0f) return false;
  float u = clampf(us0, 0.0f, 1.0f), v = clampf(us1, 0.0f, 1.0f);
  uint32_t i = 0, j = 0;
  for (uint32_t l = 1; l < d.num_levels; ++l)
    if (!env_hsw_step(d, l, i, j, u, v)) return false;
  if (i >= E.width || j >= E.height) return false;
  const float w = env_texel_weight(d, i, j);
  if (w <= 0.0f) return false;
  const float u_cont = ((float)i + u) / (float)E.width;
  const float v_cont = ((float)j + v) / (float)E.height;
  wi = env_mat_mul(E.rot, env_uv_to_direction(clampf(u_cont, 0.0f, kEnvOneMinusEps),
                                                clampf(v_cont, 0.0f, kEnvOneMinusEps)));
  const float st = sinf(v_cont * kPiF);
  if (st <= 0.0f) return false;
  const float p2d = w / d.total_weight * (float)E.width * (float)E.height;
  pdf = p2d / (kTauF * kPiF * st);
  const float* p = E.pixels + 3 * ((size_t)j * E.width + i);
  radiance = V3{E.scale * __ldg(p), E.scale * __ldg(p + 1), E.scale * __ldg(p + 2)};
  return true;
}

}  // namespace tpt
