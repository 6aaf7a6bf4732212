// Host construction of EnvironmentLight's sampling distributions
// (light/environment.rs:46-82, 301-462): the per-texel weights, the
// MIS-compensated weights and their mip pyramids, in the reference's float
// operation order so that the device samples the same texels with the same
// probabilities.
#pragma once
#include <cstdint>
#include <vector>

namespace tpt {

struct EnvPyramid {
  std::vector<float> weights;    // all levels, coarsest (1 x 1) first
  std::vector<uint32_t> levels;  // width, height, offset per level
  float total_weight = 0.0f;
};

struct EnvHost {
  uint32_t width = 0, height = 0;
  float scale = 1.0f;
  float rot[9], inv_rot[9];  // Mat3::from_rotation_y(+-rotate_y), column-major
  EnvPyramid dist, mis;
  float total_power = 0.0f;  // EnvironmentLight::total_power
};

// pixels: width * height RGB.  Returns false for an empty map.
bool build_environment(uint32_t width, uint32_t height, const float* pixels, float scale, float rotate_y,
                       EnvHost* out);

}  // namespace tpt
