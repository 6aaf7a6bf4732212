// EnvironmentLight's distributions on the host (light/environment.rs).
//
// environment_weights (:347-356): luminance clamped at 0 times the sine of the
// row centre's polar angle.  mis_compensated_environment_weights (:358-375):
// the same minus the solid-angle-weighted mean luminance (:377-392), kept only
// above max(|mean|, 1) * 1e-6.  build_distribution (:398-462): weights padded
// to power-of-two sizes and summed 2 x 2 (2 x 1 or 1 x 2 once a side is 1)
// level by level up to one root texel, whose value is the total weight.
#include "env_build.h"

#include <algorithm>
#include <cmath>

namespace tpt {

namespace {

constexpr float kPi = 3.14159274101257324f;
constexpr float kTau = 6.28318548202514648f;

float luminance(const float* c) { return 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]; }
float positive_luminance(const float* c) { return std::fmax(luminance(c), 0.0f); }

float row_sin_theta(uint32_t j, uint32_t height) {
  const float v = ((float)j + 0.5f) / (float)height;
  return std::sin(v * kPi);
}

uint32_t next_pow2(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

void build_pyramid(uint32_t width, uint32_t height, const std::vector<float>& w, EnvPyramid* out) {
  const uint32_t pw = next_pow2(width), ph = next_pow2(height);
  struct Level {
    uint32_t w, h;
    std::vector<float> v;
  };
  std::vector<Level> levels;
  Level leaf{pw, ph, std::vector<float>((size_t)pw * ph, 0.0f)};
  for (uint32_t j = 0; j < height; ++j)
    for (uint32_t i = 0; i < width; ++i) leaf.v[(size_t)j * pw + i] = std::fmax(w[(size_t)j * width + i], 0.0f);
  levels.push_back(std::move(leaf));
  while (levels.back().w > 1 || levels.back().h > 1) {
    const Level& f = levels.back();
    const uint32_t si = f.w > 1 ? 2 : 1, sj = f.h > 1 ? 2 : 1;
    Level c{f.w / si, f.h / sj, {}};
    c.v.assign((size_t)c.w * c.h, 0.0f);
    for (uint32_t j = 0; j < c.h; ++j)
      for (uint32_t i = 0; i < c.w; ++i) {
        float sum = 0.0f;
        for (uint32_t dj = 0; dj < sj; ++dj)
          for (uint32_t di = 0; di < si; ++di) sum += f.v[(size_t)(j * sj + dj) * f.w + (i * si + di)];
        c.v[(size_t)j * c.w + i] = sum;
      }
    levels.push_back(std::move(c));
  }
  std::reverse(levels.begin(), levels.end());
  out->weights.clear();
  out->levels.clear();
  for (const Level& l : levels) {
    out->levels.push_back(l.w);
    out->levels.push_back(l.h);
    out->levels.push_back((uint32_t)out->weights.size());
    out->weights.insert(out->weights.end(), l.v.begin(), l.v.end());
  }
  out->total_weight = levels[0].v[0];
}

// Mat3::from_rotation_y: columns (c, 0, -s), (0, 1, 0), (s, 0, c)
void rotation_y(float angle, float* m) {
  const float s = std::sin(angle), c = std::cos(angle);
  const float cols[9] = {c, 0.0f, -s, 0.0f, 1.0f, 0.0f, s, 0.0f, c};
  for (int k = 0; k < 9; ++k) m[k] = cols[k];
}

}  // namespace

bool build_environment(uint32_t width, uint32_t height, const float* pixels, float scale, float rotate_y,
                       EnvHost* out) {
  if (width == 0 || height == 0 || !pixels) return false;
  out->width = width;
  out->height = height;
  out->scale = scale;
  rotation_y(rotate_y, out->rot);
  rotation_y(-rotate_y, out->inv_rot);
  const size_t n = (size_t)width * height;
  std::vector<float> w(n), wm(n);
  for (uint32_t j = 0; j < height; ++j) {
    const float st = row_sin_theta(j, height);
    for (uint32_t i = 0; i < width; ++i) w[(size_t)j * width + i] = positive_luminance(pixels + 3 * ((size_t)j * width + i)) * st;
  }
  // solid_angle_mean_luminance
  float weighted_sum = 0.0f, weight_sum = 0.0f;
  for (uint32_t j = 0; j < height; ++j) {
    const float st = row_sin_theta(j, height);
    weight_sum += st * (float)width;
    for (uint32_t i = 0; i < width; ++i) weighted_sum += positive_luminance(pixels + 3 * ((size_t)j * width + i)) * st;
  }
  const float mean = weight_sum > 0.0f ? weighted_sum / weight_sum : 0.0f;
  const float eps = std::fmax(std::fabs(mean), 1.0f) * 1.0e-6f;
  for (uint32_t j = 0; j < height; ++j) {
    const float st = row_sin_theta(j, height);
    for (uint32_t i = 0; i < width; ++i) {
      const float comp = positive_luminance(pixels + 3 * ((size_t)j * width + i)) - mean;
      wm[(size_t)j * width + i] = comp > eps ? comp * st : 0.0f;
    }
  }
  build_pyramid(width, height, w, &out->dist);
  build_pyramid(width, height, wm, &out->mis);
  const float texel_solid_angle = kTau * kPi / ((float)width * (float)height);
  out->total_power = out->dist.total_weight * scale * texel_solid_angle;
  return true;
}

}  // namespace tpt
