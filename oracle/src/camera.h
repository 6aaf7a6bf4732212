// Oracle: pinhole camera (crates/renderer/src/scene/camera.rs:21-96, math/mod.rs:13-24).
#pragma once
#include "geometry.h"

namespace orc {

inline float sample_tent_1d(float u) {
  u = clampf(u, 0.0f, 1.0f);
  if (u < 0.5f) return std::sqrt(2.0f * u) - 1.0f;
  return 1.0f - std::sqrt(2.0f - 2.0f * u);
}

struct Camera {
  Vec3 eye, forward, right, image_up;
  float tan_half_fov_y = 0, exposure = 1;

  static Camera make(const Vec3& eye, const Vec3& look_at, const Vec3& up, float fov_y, float exposure) {
    Camera c;
    c.eye = eye;
    c.forward = normalize(look_at - eye);
    c.right = normalize(cross(c.forward, up));
    c.image_up = normalize(cross(c.right, c.forward));
    c.tan_half_fov_y = std::tan(0.5f * fov_y);
    c.exposure = exposure;
    return c;
  }

  Vec3 direction_for_sample(uint32_t rx, uint32_t ry, float px, float py) const {
    float fx = (float)rx, fy = (float)ry;
    float aspect = fx / fy;
    float sensor_x = ((2.0f * px / fx) - 1.0f) * aspect * tan_half_fov_y;
    float sensor_y = (1.0f - (2.0f * py / fy)) * tan_half_fov_y;
    return normalize(forward + sensor_x * right + sensor_y * image_up);
  }

  float pixel_spread_angle(uint32_t rx, uint32_t ry) const {
    float fx = (float)rx, fy = (float)ry;
    float aspect = fx / fy;
    float dx = 2.0f * aspect * tan_half_fov_y / fx;
    float dy = 2.0f * tan_half_fov_y / fy;
    return std::atan(fmax_num(dx, dy));
  }

  static float differential_scale(uint32_t spp) {
    float s = (float)(spp < 1 ? 1 : spp);
    return fmax_num(1.0f / std::sqrt(s), 0.125f);
  }

  Ray generate_ray_differential(uint32_t rx, uint32_t ry, uint32_t pxi, uint32_t pyi, Vec2 us, uint32_t spp) const {
    float px = ((float)pxi + 0.5f) + 0.5f * sample_tent_1d(us.x);
    float py = ((float)pyi + 0.5f) + 0.5f * sample_tent_1d(us.y);
    Vec3 dir = direction_for_sample(rx, ry, px, py);
    Vec3 rxd = direction_for_sample(rx, ry, px + 1.0f, py);
    Vec3 ryd = direction_for_sample(rx, ry, px, py + 1.0f);
    float scale = differential_scale(spp);
    Ray r;
    r.origin = eye;
    r.direction = dir;
    r.has_diff = true;
    r.diff.rx_origin = eye;
    r.diff.ry_origin = eye;
    r.diff.rx_direction = normalize_or_zero(dir + scale * (rxd - dir));
    r.diff.ry_direction = normalize_or_zero(dir + scale * (ryd - dir));
    r.cone_width = 0.0f;
    r.cone_spread = fmax_num(pixel_spread_angle(rx, ry) * scale, 0.0f);
    return r;
  }
};

}  // namespace orc
