// Oracle (test infrastructure): spectral dispersion of OpenPBR transmission,
// restating crates/renderer/src/bsdf/dispersion.rs -- the Cauchy IOR of an
// Abbe number (cauchy_ior :50-60), the camera's RGB spectral sensitivity over
// 400-720 nm in 10 nm steps (the Canon 5D Mark II table of Jiang et al.,
// WACV 2013, :16-47) normalised to unit integrals (:203-219), wavelength
// sampling proportional to the camera basis weighted by the path throughput
// (:67-74, :91-115, :133-152) and per camera channel (:76-81, :117-131).
#pragma once
#include "common.h"

namespace orc {

constexpr float kLambdaMinNm = 400.0f;
constexpr float kLambdaMaxNm = 720.0f;
constexpr float kLambdaStepNm = 10.0f;
constexpr int kSpectralSamples = 33;
constexpr int kSpectralIntervals = 32;

float cauchy_ior(float lambda_nm, float n_d, float abbe_v);
// (lambda, basis / pdf): a wavelength drawn proportional to the camera basis
// dotted with the (clamped) path throughput
float sample_dispersion_wavelength_weighted(float u, Vec3 throughput, Vec3* basis_over_pdf);
float sample_camera_channel_wavelength(int channel, float u);
Vec3 camera_rgb_basis_at(float lambda_nm);
float camera_wavelength_sampling_pdf(float lambda_nm, Vec3 throughput);
float camera_spectral_interval_midpoint_nm(int index);

}  // namespace orc
