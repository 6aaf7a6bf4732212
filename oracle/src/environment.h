// Oracle (test infrastructure): EnvironmentLight (light/environment.rs) --
// equirectangular map with a rotation about +y and two mip-pyramid sampling
// distributions (luminance x sin(theta), and its MIS-compensated variant).
#pragma once
#include <cstdint>
#include <vector>

#include "common.h"

namespace orc {

struct EnvDistribution {
  struct Level {
    uint32_t width, height;
    std::vector<float> weights;
  };
  std::vector<Level> levels;  // coarsest (1 x 1) first (build_distribution, :398-462)
  uint32_t padded_width = 0, padded_height = 0;
  float total_weight = 0.0f;
  float texel_weight(uint32_t i, uint32_t j) const {
    const Level& leaf = levels.back();
    return leaf.weights[(size_t)j * leaf.width + i];
  }
};

struct EnvSample {
  Vec3 direction, radiance;
  float u, v, pdf;
};

struct Environment {
  uint32_t width = 0, height = 0;
  float scale = 1.0f, rotate_y = 0.0f;
  float rot[9], inv_rot[9];  // Mat3::from_rotation_y(+-rotate_y), column-major
  std::vector<Vec3> pixels;
  EnvDistribution dist, mis;

  // EnvironmentLight::from_pixels (:46-82)
  static Environment from_pixels(uint32_t width, uint32_t height, const float* rgb, float scale, float rotate_y);
  float total_power() const;                      // :128-131
  Vec3 radiance(Vec3 direction) const;            // :133-139
  float pdf(Vec3 direction) const { return pdf_with(dist, direction); }
  float pdf_mis_compensated(Vec3 direction) const { return pdf_with(mis, direction); }
  bool sample(float u, float v, EnvSample* out) const { return sample_with(dist, u, v, out); }
  bool sample_mis_compensated(float u, float v, EnvSample* out) const { return sample_with(mis, u, v, out); }
  float pdf_with(const EnvDistribution& d, Vec3 direction) const;                    // :157-179
  bool sample_with(const EnvDistribution& d, float u, float v, EnvSample* out) const;  // :181-238
};

// direction_to_uv / uv_to_direction (:316-333)
void env_direction_to_uv(Vec3 direction, float* u, float* v);
Vec3 env_uv_to_direction(float u, float v);

}  // namespace orc
