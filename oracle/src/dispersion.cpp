// Oracle (test infrastructure): bsdf/dispersion.rs restated; see dispersion.h.
// Vec3::lerp is glam's `self * (1 - s) + rhs * s`; sums run in index order as
// the reference's iterator folds do.
#include "dispersion.h"

namespace orc {

namespace {

constexpr float kLambdaF = 486.13f;  // Fraunhofer F, d and C lines (dispersion.rs:5-7)
constexpr float kLambdaD = 587.56f;
constexpr float kLambdaC = 656.27f;
constexpr float kLambdaRange = kLambdaMaxNm - kLambdaMinNm;
constexpr float kF32Epsilon = 1.1920929e-7f;

// Canon 5D Mark II RGB spectral sensitivity, 400-720 nm in 10 nm steps
// (Jiang, Liu, Gu and Suesstrunk, "What is the Space of Spectral Sensitivity
// Functions for Digital Color Cameras?", WACV 2013; Camera Spectral Sensitivity
// Database, DOI 10.5281/zenodo.3245883, CC BY-NC-SA 4.0): the table the
// reference samples, dispersion.rs:22-47.
const float kSensR[kSpectralSamples] = {
    0.0019f, 0.0045f, 0.0103f, 0.0055f, 0.0034f, 0.0021f, 0.0023f, 0.0039f, 0.0073f, 0.0118f, 0.0179f,
    0.0612f, 0.0874f, 0.1534f, 0.1686f, 0.1724f, 0.2003f, 0.3158f, 0.4514f, 0.5258f, 0.5989f, 0.4728f,
    0.4084f, 0.3562f, 0.292f,  0.226f,  0.1704f, 0.1372f, 0.0428f, 0.0087f, 0.0017f, 0.0007f, 0.0005f};
const float kSensG[kSpectralSamples] = {
    0.0036f, 0.0123f, 0.0377f, 0.0422f, 0.0565f, 0.0704f, 0.097f,  0.209f,  0.43f,   0.6381f, 0.692f,
    1.0f,    0.8735f, 0.9058f, 0.8326f, 0.8057f, 0.712f,  0.6467f, 0.5426f, 0.3935f, 0.2958f, 0.1287f,
    0.06f,   0.0402f, 0.0276f, 0.0182f, 0.0138f, 0.0143f, 0.0061f, 0.0017f, 0.0008f, 0.0006f, 0.0005f};
const float kSensB[kSpectralSamples] = {
    0.0127f, 0.0971f, 0.3516f, 0.4765f, 0.56f,   0.6476f, 0.7745f, 0.6759f, 0.6858f, 0.5932f, 0.3971f,
    0.3559f, 0.1617f, 0.0883f, 0.0551f, 0.0424f, 0.0269f, 0.0205f, 0.0159f, 0.0122f, 0.01f,   0.0054f,
    0.0036f, 0.0032f, 0.0029f, 0.0032f, 0.0032f, 0.0034f, 0.0013f, 0.0005f, 0.0004f, 0.0004f, 0.0004f};

Vec3 sens_sample(int i) { return Vec3(kSensR[i], kSensG[i], kSensB[i]); }

// camera_normalization_scale (dispersion.rs:203-219): 1 / trapezoid integral
Vec3 normalization_scale() {
  Vec3 integral(0, 0, 0);
  for (int i = 0; i < kSpectralIntervals; ++i)
    integral += 0.5f * (sens_sample(i) + sens_sample(i + 1)) * kLambdaStepNm;
  return Vec3(1.0f / fmax_num(integral.x, 1.0e-8f), 1.0f / fmax_num(integral.y, 1.0e-8f),
              1.0f / fmax_num(integral.z, 1.0e-8f));
}

// the scale and the normalised table, computed once (the reference caches the
// scale in a OnceLock)
struct Basis {
  Vec3 scale;
  Vec3 sample[kSpectralSamples];
  Basis() {
    scale = normalization_scale();
    for (int i = 0; i < kSpectralSamples; ++i) sample[i] = sens_sample(i) * scale;
  }
};
const Basis& basis() {
  static const Basis b;
  return b;
}
Vec3 basis_sample(int i) { return basis().sample[i]; }

// camera_rgb_sensitivity_at (dispersion.rs:154-167)
Vec3 sensitivity_at(float lambda_nm) {
  const float position = (lambda_nm - kLambdaMinNm) / kLambdaStepNm;
  if (position <= 0.0f) return sens_sample(0);
  const int max_index = kSpectralSamples - 1;
  if (position >= (float)max_index) return sens_sample(max_index);
  const int lower = (int)std::floor(position);
  const float t = position - (float)lower;
  return sens_sample(lower) * (1.0f - t) + sens_sample(lower + 1) * t;
}

// wavelength_interval_weights (dispersion.rs:91-115)
void interval_weights(Vec3 throughput, float* w) {
  throughput = vmax(throughput, Vec3(0, 0, 0));
  const Vec3 weights = max_element(throughput) > 0.0f ? throughput : Vec3(1, 1, 1);
  float sum = 0.0f;
  for (int i = 0; i < kSpectralIntervals; ++i) {
    const float s0 = fmax_num(dot(basis_sample(i), weights), 0.0f);
    const float s1 = fmax_num(dot(basis_sample(i + 1), weights), 0.0f);
    w[i] = 0.5f * (s0 + s1) * kLambdaStepNm;
    sum += w[i];
  }
  if (sum <= 0.0f)
    for (int i = 0; i < kSpectralIntervals; ++i) w[i] = kLambdaRange / (float)kSpectralIntervals;
}

// camera_channel_interval_weights (dispersion.rs:117-131)
void channel_weights(int channel, float* w) {
  float sum = 0.0f;
  for (int i = 0; i < kSpectralIntervals; ++i) {
    const float s0 = fmax_num(basis_sample(i)[channel < 2 ? channel : 2], 0.0f);
    const float s1 = fmax_num(basis_sample(i + 1)[channel < 2 ? channel : 2], 0.0f);
    w[i] = 0.5f * (s0 + s1) * kLambdaStepNm;
    sum += w[i];
  }
  if (sum <= 0.0f)
    for (int i = 0; i < kSpectralIntervals; ++i) w[i] = kLambdaRange / (float)kSpectralIntervals;
}

float weights_total(const float* w) {
  float total = 0.0f;
  for (int i = 0; i < kSpectralIntervals; ++i) total += w[i];
  return fmax_num(total, 1.0e-8f);
}

// sample_interval (dispersion.rs:133-152)
void sample_interval(const float* w, float u, int* index, float* local, float* pdf) {
  const float total = weights_total(w);
  const float target = clampf(u, 0.0f, 1.0f - kF32Epsilon) * total;
  float sum = 0.0f;
  int idx = 0;
  for (int i = 0; i < kSpectralIntervals; ++i) {
    if (target < sum + w[i]) {
      idx = i;
      break;
    }
    sum += w[i];
    idx = i;
  }
  const float iw = fmax_num(w[idx], 1.0e-8f);
  *index = idx;
  *local = clampf((target - sum) / iw, 0.0f, 1.0f);
  *pdf = iw / (total * kLambdaStepNm);
}

float interval_lambda(int index, float local) {
  return clampf(kLambdaMinNm + kLambdaStepNm * ((float)index + local), kLambdaMinNm, kLambdaMaxNm);
}

}  // namespace

float cauchy_ior(float lambda_nm, float n_d, float abbe_v) {
  if (abbe_v <= 0.0f) return n_d;
  const float inv_lf2 = 1.0f / (kLambdaF * kLambdaF);
  const float inv_lc2 = 1.0f / (kLambdaC * kLambdaC);
  const float inv_ld2 = 1.0f / (kLambdaD * kLambdaD);
  const float b = (n_d - 1.0f) / (abbe_v * (inv_lf2 - inv_lc2));
  const float a = n_d - b * inv_ld2;
  return a + b / (lambda_nm * lambda_nm);
}

float sample_dispersion_wavelength_weighted(float u, Vec3 throughput, Vec3* basis_over_pdf) {
  float w[kSpectralIntervals];
  interval_weights(throughput, w);
  int index;
  float local, pdf;
  sample_interval(w, u, &index, &local, &pdf);
  const float lambda = interval_lambda(index, local);
  *basis_over_pdf = camera_rgb_basis_at(lambda) / fmax_num(pdf, 1.0e-8f);
  return lambda;
}

float sample_camera_channel_wavelength(int channel, float u) {
  float w[kSpectralIntervals];
  channel_weights(channel, w);
  int index;
  float local, pdf;
  sample_interval(w, u, &index, &local, &pdf);
  return interval_lambda(index, local);
}

Vec3 camera_rgb_basis_at(float lambda_nm) { return sensitivity_at(lambda_nm) * basis().scale; }

// camera_wavelength_sampling_pdf (dispersion.rs:83-89)
float camera_wavelength_sampling_pdf(float lambda_nm, Vec3 throughput) {
  float w[kSpectralIntervals];
  interval_weights(throughput, w);
  float total = 0.0f;
  for (int i = 0; i < kSpectralIntervals; ++i) total += w[i];
  total = fmax_num(total, 1.0e-8f);
  const float position = clampf((lambda_nm - kLambdaMinNm) / kLambdaStepNm, 0.0f,
                                (float)kSpectralIntervals - kF32Epsilon);
  // (32 - EPSILON rounds to 32 in f32: the last interval takes lambda = 720)
  const int interval = std::min((int)std::floor(position), kSpectralIntervals - 1);
  return w[interval] / (total * kLambdaStepNm);
}

float camera_spectral_interval_midpoint_nm(int index) {
  return kLambdaMinNm + kLambdaStepNm * ((float)index + 0.5f);
}

}  // namespace orc
