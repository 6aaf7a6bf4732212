// Oracle (test infrastructure): EnvironmentLight, restating
// crates/renderer/src/light/environment.rs (from_pixels :46-82, total_power
// :128-131, radiance :133-139, pdf_with_distribution :157-179,
// sample_with_distribution :181-238, row_sin_theta :305-308, pixel_coord
// :310-314, uv_to_direction :316-321, direction_to_uv :323-333, weights
// :347-392, build_distribution :398-462, hsw_step :464-525).  glam's
// Mat3::from_rotation_y and Mat3 * Vec3 are written out with their column
// layout and summation order.
#include "environment.h"

#include <algorithm>
#include <cmath>

namespace orc {

namespace {

constexpr float kPiE = 3.14159274101257324f;
constexpr float kTauE = 6.28318548202514648f;
constexpr float kOneMinusEps = 1.0f - 1.1920929e-7f;

float luminance(Vec3 v) { return 0.2126f * v.x + 0.7152f * v.y + 0.0722f * v.z; }
float positive_luminance(Vec3 v) { return std::fmax(luminance(v), 0.0f); }

float row_sin_theta(uint32_t j, uint32_t height) {
  const float v = ((float)j + 0.5f) / (float)height;
  return std::sin(v * kPiE);
}

uint32_t pixel_coord(float t, uint32_t size) {
  const float c = clampf(t, 0.0f, 1.0f);
  const uint32_t idx = (uint32_t)(c * (float)size);
  return std::min(idx, size - 1);
}

uint32_t next_power_of_two(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

EnvDistribution build_distribution(uint32_t width, uint32_t height, const std::vector<float>& pixel_weights) {
  EnvDistribution d;
  d.padded_width = next_power_of_two(width);
  d.padded_height = next_power_of_two(height);
  std::vector<EnvDistribution::Level> levels;
  EnvDistribution::Level leaf{d.padded_width, d.padded_height,
                              std::vector<float>((size_t)d.padded_width * d.padded_height, 0.0f)};
  for (uint32_t j = 0; j < height; ++j)
    for (uint32_t i = 0; i < width; ++i)
      leaf.weights[(size_t)j * d.padded_width + i] = std::fmax(pixel_weights[(size_t)j * width + i], 0.0f);
  levels.push_back(std::move(leaf));
  while (levels.back().width > 1 || levels.back().height > 1) {
    const EnvDistribution::Level& finer = levels.back();
    const uint32_t scale_i = finer.width > 1 ? 2 : 1, scale_j = finer.height > 1 ? 2 : 1;
    EnvDistribution::Level coarse{finer.width / scale_i, finer.height / scale_j, {}};
    coarse.weights.assign((size_t)coarse.width * coarse.height, 0.0f);
    for (uint32_t j = 0; j < coarse.height; ++j)
      for (uint32_t i = 0; i < coarse.width; ++i) {
        float sum = 0.0f;
        for (uint32_t dj = 0; dj < scale_j; ++dj)
          for (uint32_t di = 0; di < scale_i; ++di)
            sum += finer.weights[(size_t)(j * scale_j + dj) * finer.width + (i * scale_i + di)];
        coarse.weights[(size_t)j * coarse.width + i] = sum;
      }
    levels.push_back(std::move(coarse));
  }
  std::reverse(levels.begin(), levels.end());
  d.total_weight = levels[0].weights[0];
  d.levels = std::move(levels);
  return d;
}

// hsw_step: from texel (pi, pj) of the parent level into `child`
bool hsw_step(uint32_t parent_w, uint32_t parent_h, const EnvDistribution::Level& child, uint32_t* i, uint32_t* j,
              float* u, float* v) {
  const uint32_t scale_i = child.width / parent_w, scale_j = child.height / parent_h;
  uint32_t ci = *i * scale_i, cj = *j * scale_j;
  if (scale_j == 2) {
    float w_top = 0.0f, w_bot = 0.0f;
    for (uint32_t di = 0; di < scale_i; ++di) {
      w_top += child.weights[(size_t)cj * child.width + ci + di];
      w_bot += child.weights[(size_t)(cj + 1) * child.width + ci + di];
    }
    const float total = w_top + w_bot;
    if (total <= 0.0f) return false;
    const float p_top = w_top / total;
    if (*v < p_top) {
      *v = clampf(*v / p_top, 0.0f, kOneMinusEps);
    } else {
      *v = clampf((*v - p_top) / (1.0f - p_top), 0.0f, kOneMinusEps);
      cj += 1;
    }
  }
  if (scale_i == 2) {
    const float w_left = child.weights[(size_t)cj * child.width + ci];
    const float w_right = child.weights[(size_t)cj * child.width + ci + 1];
    const float total = w_left + w_right;
    if (total <= 0.0f) return false;
    const float p_left = w_left / total;
    if (*u < p_left) {
      *u = clampf(*u / p_left, 0.0f, kOneMinusEps);
    } else {
      *u = clampf((*u - p_left) / (1.0f - p_left), 0.0f, kOneMinusEps);
      ci += 1;
    }
  }
  *i = ci;
  *j = cj;
  return true;
}

void rotation_y(float angle, float* m) {
  const float s = std::sin(angle), c = std::cos(angle);
  const float cols[9] = {c, 0.0f, -s, 0.0f, 1.0f, 0.0f, s, 0.0f, c};
  std::copy(cols, cols + 9, m);
}

Vec3 mat_mul(const float* m, Vec3 v) {
  return Vec3((m[0] * v.x + m[3] * v.y) + m[6] * v.z, (m[1] * v.x + m[4] * v.y) + m[7] * v.z,
              (m[2] * v.x + m[5] * v.y) + m[8] * v.z);
}

}  // namespace

Vec3 env_uv_to_direction(float u, float v) {
  const float phi = u * kTauE, theta = v * kPiE;
  const float st = std::sin(theta);
  return Vec3(st * std::sin(phi), std::cos(theta), st * std::cos(phi));
}

void env_direction_to_uv(Vec3 direction, float* u, float* v) {
  const Vec3 dir = normalize_or_zero(direction);
  const float y = clampf(dir.y, -1.0f, 1.0f);
  const float theta = std::acos(y);
  float phi = std::atan2(dir.x, dir.z);
  if (phi < 0.0f) phi += kTauE;
  *u = clampf(phi / kTauE, 0.0f, 1.0f);
  *v = clampf(theta / kPiE, 0.0f, 1.0f);
}

Environment Environment::from_pixels(uint32_t width, uint32_t height, const float* rgb, float scale,
                                     float rotate_y) {
  Environment e;
  e.width = width;
  e.height = height;
  e.scale = scale;
  e.rotate_y = rotate_y;
  e.pixels.resize((size_t)width * height);
  for (size_t k = 0; k < e.pixels.size(); ++k) e.pixels[k] = Vec3(rgb[3 * k], rgb[3 * k + 1], rgb[3 * k + 2]);
  // environment_weights
  std::vector<float> w((size_t)width * height, 0.0f);
  for (uint32_t j = 0; j < height; ++j) {
    const float st = row_sin_theta(j, height);
    for (uint32_t i = 0; i < width; ++i) w[(size_t)j * width + i] = positive_luminance(e.pixels[(size_t)j * width + i]) * st;
  }
  // mis_compensated_environment_weights with solid_angle_mean_luminance
  float weighted_sum = 0.0f, weight_sum = 0.0f;
  for (uint32_t j = 0; j < height; ++j) {
    const float st = row_sin_theta(j, height);
    weight_sum += st * (float)width;
    for (uint32_t i = 0; i < width; ++i) weighted_sum += positive_luminance(e.pixels[(size_t)j * width + i]) * st;
  }
  const float mean = weight_sum > 0.0f ? weighted_sum / weight_sum : 0.0f;
  const float eps = std::fmax(std::fabs(mean), 1.0f) * 1.0e-6f;
  std::vector<float> wm((size_t)width * height, 0.0f);
  for (uint32_t j = 0; j < height; ++j) {
    const float st = row_sin_theta(j, height);
    for (uint32_t i = 0; i < width; ++i) {
      const float c = positive_luminance(e.pixels[(size_t)j * width + i]) - mean;
      wm[(size_t)j * width + i] = c > eps ? c * st : 0.0f;
    }
  }
  e.dist = build_distribution(width, height, w);
  e.mis = build_distribution(width, height, wm);
  rotation_y(rotate_y, e.rot);
  rotation_y(-rotate_y, e.inv_rot);
  return e;
}

float Environment::total_power() const {
  const float texel_solid_angle = kTauE * kPiE / ((float)width * (float)height);
  return dist.total_weight * scale * texel_solid_angle;
}

Vec3 Environment::radiance(Vec3 direction) const {
  float u, v;
  env_direction_to_uv(mat_mul(inv_rot, direction), &u, &v);
  const uint32_t i = pixel_coord(u, width), j = pixel_coord(v, height);
  return scale * pixels[(size_t)j * width + i];
}

float Environment::pdf_with(const EnvDistribution& d, Vec3 direction) const {
  if (d.total_weight <= 0.0f) return 0.0f;
  float u, v;
  env_direction_to_uv(mat_mul(inv_rot, direction), &u, &v);
  const float st = std::sin(v * kPiE);
  if (st <= 0.0f) return 0.0f;
  const uint32_t i = pixel_coord(u, width), j = pixel_coord(v, height);
  const float w = d.texel_weight(i, j);
  if (w <= 0.0f) return 0.0f;
  const float p2d = w / d.total_weight * (float)width * (float)height;
  return p2d / (kTauE * kPiE * st);
}

bool Environment::sample_with(const EnvDistribution& d, float us0, float us1, EnvSample* out) const {
  if (d.total_weight <= 0.0f) return false;
  float u = clampf(us0, 0.0f, 1.0f), v = clampf(us1, 0.0f, 1.0f);
  uint32_t i = 0, j = 0;
  for (size_t l = 1; l < d.levels.size(); ++l)
    if (!hsw_step(d.levels[l - 1].width, d.levels[l - 1].height, d.levels[l], &i, &j, &u, &v)) return false;
  if (i >= width || j >= height) return false;
  const float w = d.texel_weight(i, j);
  if (w <= 0.0f) return false;
  const float u_cont = ((float)i + u) / (float)width;
  const float v_cont = ((float)j + v) / (float)height;
  out->u = clampf(u_cont, 0.0f, kOneMinusEps);
  out->v = clampf(v_cont, 0.0f, kOneMinusEps);
  out->direction = mat_mul(rot, env_uv_to_direction(out->u, out->v));
  const float st = std::sin(v_cont * kPiE);
  if (st <= 0.0f) return false;
  const float p2d = w / d.total_weight * (float)width * (float)height;
  out->pdf = p2d / (kTauE * kPiE * st);
  out->radiance = scale * pixels[(size_t)j * width + i];
  return true;
}

}  // namespace orc
