// Spectral dispersion of OpenPBR transmission on the device
// (bsdf/dispersion.rs): the Cauchy IOR of an Abbe number, the camera's RGB
// spectral sensitivity over 400-720 nm in 10 nm steps normalised to unit
// integrals, and wavelength sampling proportional to that basis (weighted by
// the path throughput) or to one channel of it.  Every function keeps the
// reference's f32 operation order; glam's Vec3::lerp is a * (1 - t) + b * t.
#pragma once
#include "vmath.cuh"

namespace tpt {
namespace disp {

constexpr float kLambdaMin = 400.0f, kLambdaMax = 720.0f, kLambdaStep = 10.0f;
constexpr int kSamples = 33, kIntervals = 32;

// Canon 5D Mark II RGB spectral sensitivity at 400, 410, ..., 720 nm (Jiang,
// Liu, Gu and Suesstrunk, WACV 2013; Camera Spectral Sensitivity Database,
// DOI 10.5281/zenodo.3245883, CC BY-NC-SA 4.0): the table the reference
// samples (dispersion.rs:22-47).
static __constant__ float c_sens[3][kSamples] = {
    {0.0019f, 0.0045f, 0.0103f, 0.0055f, 0.0034f, 0.0021f, 0.0023f, 0.0039f, 0.0073f, 0.0118f, 0.0179f,
     0.0612f, 0.0874f, 0.1534f, 0.1686f, 0.1724f, 0.2003f, 0.3158f, 0.4514f, 0.5258f, 0.5989f, 0.4728f,
     0.4084f, 0.3562f, 0.292f,  0.226f,  0.1704f, 0.1372f, 0.0428f, 0.0087f, 0.0017f, 0.0007f, 0.0005f},
    {0.0036f, 0.0123f, 0.0377f, 0.0422f, 0.0565f, 0.0704f, 0.097f,  0.209f,  0.43f,   0.6381f, 0.692f,
     1.0f,    0.8735f, 0.9058f, 0.8326f, 0.8057f, 0.712f,  0.6467f, 0.5426f, 0.3935f, 0.2958f, 0.1287f,
     0.06f,   0.0402f, 0.0276f, 0.0182f, 0.0138f, 0.0143f, 0.0061f, 0.0017f, 0.0008f, 0.0006f, 0.0005f},
    {0.0127f, 0.0971f, 0.3516f, 0.4765f, 0.56f,   0.6476f, 0.7745f, 0.6759f, 0.6858f, 0.5932f, 0.3971f,
     0.3559f, 0.1617f, 0.0883f, 0.0551f, 0.0424f, 0.0269f, 0.0205f, 0.0159f, 0.0122f, 0.01f,   0.0054f,
     0.0036f, 0.0032f, 0.0029f, 0.0032f, 0.0032f, 0.0034f, 0.0013f, 0.0005f, 0.0004f, 0.0004f, 0.0004f}};

__device__ __forceinline__ V3 sens(int i) { return V3{c_sens[0][i], c_sens[1][i], c_sens[2][i]}; }

// camera_normalization_scale (dispersion.rs:203-219): 1 / trapezoid integral
__device__ __forceinline__ V3 norm_scale() {
  V3 integral = V3{0.0f, 0.0f, 0.0f};
  for (int i = 0; i < kIntervals; ++i) integral = integral + (0.5f * (sens(i) + sens(i + 1))) * kLambdaStep;
  return V3{1.0f / fmaxf(integral.x, 1.0e-8f), 1.0f / fmaxf(integral.y, 1.0e-8f), 1.0f / fmaxf(integral.z, 1.0e-8f)};
}

// cauchy_ior (dispersion.rs:50-60)
__device__ __forceinline__ float cauchy_ior(float lambda_nm, float n_d, float abbe_v) {
  if (abbe_v <= 0.0f) return n_d;
  const float lf = 486.13f, ld = 587.56f, lc = 656.27f;
  const float inv_lf2 = 1.0f / (lf * lf), inv_lc2 = 1.0f / (lc * lc), inv_ld2 = 1.0f / (ld * ld);
  const float b = (n_d - 1.0f) / (abbe_v * (inv_lf2 - inv_lc2));
  const float a = n_d - b * inv_ld2;
  return a + b / (lambda_nm * lambda_nm);
}

// camera_rgb_basis_at (dispersion.rs:154-167 times the scale)
__device__ __forceinline__ V3 basis_at(float lambda_nm, V3 scale) {
  const float position = (lambda_nm - kLambdaMin) / kLambdaStep;
  V3 s;
  if (position <= 0.0f) {
    s = sens(0);
  } else if (position >= (float)(kSamples - 1)) {
    s = sens(kSamples - 1);
  } else {
    const int lower = (int)floorf(position);
    const float t = position - (float)lower;
    s = sens(lower) * (1.0f - t) + sens(lower + 1) * t;
  }
  return s * scale;
}

// wavelength_interval_weights (dispersion.rs:91-115); returns the clamped total
__device__ __forceinline__ float interval_weights(V3 throughput, V3 scale, float* w) {
  throughput = V3{fmaxf(throughput.x, 0.0f), fmaxf(throughput.y, 0.0f), fmaxf(throughput.z, 0.0f)};
  const V3 weights = max_element(throughput) > 0.0f ? throughput : V3{1.0f, 1.0f, 1.0f};
  float sum = 0.0f;
  float s0 = fmaxf(dot(sens(0) * scale, weights), 0.0f);
  for (int i = 0; i < kIntervals; ++i) {
    const float s1 = fmaxf(dot(sens(i + 1) * scale, weights), 0.0f);
    w[i] = 0.5f * (s0 + s1) * kLambdaStep;
    sum += w[i];
    s0 = s1;
  }
  if (sum <= 0.0f)
    for (int i = 0; i < kIntervals; ++i) w[i] = (kLambdaMax - kLambdaMin) / (float)kIntervals;
  float total = 0.0f;
  for (int i = 0; i < kIntervals; ++i) total += w[i];
  return fmaxf(total, 1.0e-8f);
}

// camera_channel_interval_weights (dispersion.rs:117-131)
__device__ __forceinline__ float channel_weights(int ch, V3 scale, float* w) {
  const float sc = ch == 0 ? scale.x : (ch == 1 ? scale.y : scale.z);
  float sum = 0.0f;
  float s0 = fmaxf(c_sens[ch][0] * sc, 0.0f);
  for (int i = 0; i < kIntervals; ++i) {
    const float s1 = fmaxf(c_sens[ch][i + 1] * sc, 0.0f);
    w[i] = 0.5f * (s0 + s1) * kLambdaStep;
    sum += w[i];
    s0 = s1;
  }
  if (sum <= 0.0f)
    for (int i = 0; i < kIntervals; ++i) w[i] = (kLambdaMax - kLambdaMin) / (float)kIntervals;
  float total = 0.0f;
  for (int i = 0; i < kIntervals; ++i) total += w[i];
  return fmaxf(total, 1.0e-8f);
}

// sample_interval (dispersion.rs:133-152) and the wavelength it maps to
__device__ __forceinline__ float sample_interval(const float* w, float total, float u, float& pdf) {
  const float target = clampf(u, 0.0f, 1.0f - 1.1920929e-7f) * total;
  float sum = 0.0f;
  int idx = 0;
  for (int i = 0; i < kIntervals; ++i) {
    idx = i;
    if (target < sum + w[i]) break;
    sum += w[i];
  }
  const float iw = fmaxf(w[idx], 1.0e-8f);
  const float local = clampf((target - sum) / iw, 0.0f, 1.0f);
  pdf = iw / (total * kLambdaStep);
  return clampf(kLambdaMin + kLambdaStep * ((float)idx + local), kLambdaMin, kLambdaMax);
}

// sample_dispersion_wavelength_weighted (dispersion.rs:67-74): (lambda, basis / pdf)
__device__ __forceinline__ float sample_wavelength_weighted(float u, V3 throughput, V3& basis_over_pdf) {
  const V3 scale = norm_scale();
  float w[kIntervals];
  const float total = interval_weights(throughput, scale, w);
  float pdf;
  const float lambda = sample_interval(w, total, u, pdf);
  basis_over_pdf = basis_at(lambda, scale) / fmaxf(pdf, 1.0e-8f);
  return lambda;
}

// sample_camera_channel_wavelength (dispersion.rs:76-81)
__device__ __forceinline__ float sample_channel_wavelength(int ch, float u) {
  float w[kIntervals];
  const float total = channel_weights(ch, norm_scale(), w);
  float pdf;
  return sample_interval(w, total, u, pdf);
}

// camera_spectral_interval_midpoint_nm
__device__ __forceinline__ float interval_midpoint(int i) { return kLambdaMin + kLambdaStep * ((float)i + 0.5f); }

}  // namespace disp
}  // namespace tpt
