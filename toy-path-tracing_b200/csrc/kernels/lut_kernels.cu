// GPU construction of the OpenPBR lookup tables (bsdf/directional_albedo.rs):
//
//   dielectric directional albedo  1 M cells x 64 hemisphere samples
//   conductor energy compensation  4096 cells x 256 VNDF samples
//   dielectric energy compensation 32768 cells x 4096 VNDF samples (R + T)
//
// One thread per cell sums its samples in the reference's order, so each cell
// is bit-identical to the reference loop: the only transcendental inputs (the
// sample directions' sines and cosines) come precomputed from the host math
// library, everything else is +, *, / and sqrt, correctly rounded on both
// sides (the library is compiled with -fmad=false).  The reference builds these
// on the CPU with rayon at scene preparation; here they take milliseconds.
#include "../api/internal.h"
#include "../device/openpbr.cuh"

namespace tpt {

namespace {
using namespace opbr;

__device__ __forceinline__ float cell_center(int index, int resolution) {
  return ((float)index + 0.5f) / (float)resolution;
}
__device__ __forceinline__ float ggx_g1(V3 w, float ax, float ay) {
  const float l = ggx_lambda(w, ax, ay);
  if (!isfinite(l)) return 0.0f;
  return 1.0f / (1.0f + l);
}
__device__ __forceinline__ float pdf_wm_vndf(V3 wo, V3 wm, float ax, float ay) {  // smith_ggx.rs:63-77
  if (!(wo.z > 0.0f) || wm.z <= 0.0f) return 0.0f;
  const float d = ggx_d(wm, ax, ay);
  const float g1 = ggx_g1(wo, ax, ay);
  const float c = fmaxf(dot(wo, wm), 0.0f);
  if (d <= 0.0f || g1 <= 0.0f || c <= 0.0f) return 0.0f;
  return d * g1 * c / wo.z;
}
// sample_wm_vndf (smith_ggx.rs:80-123) with cos/sin of 2 pi u.y given
__device__ __forceinline__ bool sample_wm_vndf(V3 wo, float ax, float ay, float ux, float cphi, float sphi, V3& out) {
  if (wo.z <= 0.0f) return false;
  ax = fmaxf(ax, kMinAlpha);
  ay = fmaxf(ay, kMinAlpha);
  const V3 wo_std = normalize_or_zero(V3{ax * wo.x, ay * wo.y, wo.z});
  if (length_sq(wo_std) == 0.0f) return false;
  const float lensq = wo_std.x * wo_std.x + wo_std.y * wo_std.y;
  const V3 t1 = lensq > 0.0f ? V3{-wo_std.y, wo_std.x, 0.0f} / sqrtf(lensq) : V3{1.0f, 0.0f, 0.0f};
  const V3 t2 = cross(wo_std, t1);
  const float r = sqrtf(clampf(ux, 0.0f, 1.0f));
  const float p1 = r * cphi;
  float p2 = r * sphi;
  const float s = 0.5f * (1.0f + wo_std.z);
  p2 = (1.0f - s) * sqrtf(fmaxf(1.0f - p1 * p1, 0.0f)) + s * p2;
  const V3 nh = p1 * t1 + p2 * t2 + sqrtf(fmaxf(1.0f - p1 * p1 - p2 * p2, 0.0f)) * wo_std;
  const V3 wm = normalize_or_zero(V3{ax * nh.x, ay * nh.y, fmaxf(nh.z, 0.0f)});
  if (length_sq(wm) == 0.0f || wm.z <= 0.0f) return false;
  out = wm;
  return true;
}

// DielectricGgxBsdf reflection-only eval (dielectric_ggx.rs:133-163), front face
__device__ __forceinline__ float dielectric_reflection_eval(float eta, float ax, float ay, V3 wo, V3 wi) {
  if (!(wo.z > 0.0f) || eta <= 0.0f) return 0.0f;
  if (!(wo.z * wi.z > 0.0f)) return 0.0f;
  V3 wm;
  if (!half_vector(wo, wi, wm)) return 0.0f;
  const float cos_wo_wm = dot(wo, wm);
  if (cos_wo_wm <= 0.0f) return 0.0f;
  const float cos_o = fabsf(wo.z), cos_i = fabsf(wi.z);
  if (cos_o <= 0.0f || cos_i <= 0.0f) return 0.0f;
  const float d = ggx_d(wm, ax, ay);
  if (d <= 0.0f) return 0.0f;
  const float g = ggx_g2(wo, wi, ax, ay);
  if (g <= 0.0f) return 0.0f;
  const float f = fresnel_dielectric(cos_wo_wm, 1.0f, eta);
  return d * g * f / (4.0f * cos_o * cos_i);
}

// alpha_xy_from_roughness (directional_albedo.rs:358-370)
__device__ __forceinline__ void alpha_xy(float roughness, float anisotropy, float& ax, float& ay) {
  roughness = clampf(roughness, 0.0f, 1.0f);
  anisotropy = clampf(anisotropy, -1.0f, 1.0f);
  const float alpha = roughness * roughness;
  const float aspect = sqrtf(1.0f - 0.9f * fabsf(anisotropy));
  float x, y;
  if (anisotropy >= 0.0f) {
    x = alpha / aspect;
    y = alpha * aspect;
  } else {
    x = alpha * aspect;
    y = alpha / aspect;
  }
  ax = clampf(x, kMinAlpha, 1.0f);
  ay = clampf(y, kMinAlpha, 1.0f);
}

constexpr int kLutBlock = 128;

// DielectricGgxDirectionalAlbedoLut::build (directional_albedo.rs:134-167, 292-325)
__global__ void __launch_bounds__(kLutBlock) lut_da_kernel(float eta, const float* __restrict__ dirs,
                                                           const float* __restrict__ phi_cs, float* __restrict__ out) {
  __shared__ float sd[64 * 3];
  for (int k = threadIdx.x; k < 64 * 3; k += blockDim.x) sd[k] = dirs[k];
  __syncthreads();
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (uint32_t)(64 * 16 * 64 * 16)) return;
  const int ia = idx % 16, ir = (idx / 16) % 64, ip = (idx / 1024) % 16, ic = idx / 16384;
  const float sqrt_cos = cell_center(ic, 64);
  const float cos_theta = sqrt_cos * sqrt_cos;
  const float sin_theta = sqrtf(fmaxf(1.0f - cos_theta * cos_theta, 0.0f));
  const V3 wo = V3{sin_theta * phi_cs[2 * ip], sin_theta * phi_cs[2 * ip + 1], cos_theta};
  const float roughness = cell_center(ir, 64);
  const float anisotropy = 2.0f * cell_center(ia, 16) - 1.0f;
  float ax, ay;
  alpha_xy(roughness, anisotropy, ax, ay);
  float val;
  if (!(wo.z > 0.0f)) {
    val = 0.0f;
  } else if (fmaxf(ax, ay) < kSmoothAlpha) {
    val = fresnel_dielectric(clampf(wo.z, 0.0f, 1.0f), 1.0f, eta);
  } else {
    ax = fmaxf(ax, kMinAlpha);
    ay = fmaxf(ay, kMinAlpha);
    constexpr float kUniformHemispherePdf = 1.0f / (2.0f * kPiF);
    float sum = 0.0f;
    for (int k = 0; k < 64; ++k) {
      const V3 wi = V3{sd[3 * k], sd[3 * k + 1], sd[3 * k + 2]};
      sum += dielectric_reflection_eval(eta, ax, ay, wo, wi) * fmaxf(wi.z, 0.0f) / kUniformHemispherePdf;
    }
    val = clampf(sum / 64.0f, 0.0f, 1.0f);
  }
  out[idx] = val;
}

// ConductorGgxEnergyCompensationLut::build (directional_albedo.rs:700-730, 781-822)
__global__ void __launch_bounds__(kLutBlock) lut_cec_kernel(const float* __restrict__ u, const float* __restrict__ cs,
                                                            float* __restrict__ e) {
  const uint32_t index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= 64u * 64u) return;
  const int ic = index % 64, ir = index / 64;
  const float sqrt_cos = cell_center(ic, 64);
  const float cos_theta = sqrt_cos * sqrt_cos;
  const float roughness = cell_center(ir, 64);
  const float alpha = clampf(roughness * roughness, kMinAlpha, 1.0f);
  float val;
  if (cos_theta <= 0.0f) {
    val = 0.0f;
  } else if (alpha < kSmoothAlpha) {
    val = 1.0f;
  } else {
    const float sin_theta = sqrtf(fmaxf(1.0f - cos_theta * cos_theta, 0.0f));
    const V3 wo = V3{sin_theta, 0.0f, cos_theta};
    const float g1 = ggx_g1(wo, alpha, alpha);
    if (g1 <= 0.0f) {
      val = 0.0f;
    } else {
      float sum = 0.0f;
      for (int k = 0; k < 256; ++k) {
        float term = 0.0f;
        V3 wm;
        if (sample_wm_vndf(wo, alpha, alpha, __ldg(u + k), __ldg(cs + 2 * k), __ldg(cs + 2 * k + 1), wm)) {
          const float c = dot(wo, wm);
          if (!(c <= 0.0f)) {
            const V3 wi = reflect_local(wo, wm);
            if (!(wi.z <= 0.0f)) term = ggx_g2(wo, wi, alpha, alpha) / g1;
          }
        }
        sum += term;
      }
      val = clampf(sum / 256.0f, 0.0f, 1.0f);
    }
  }
  e[index] = val;
}

// DielectricGgxBsdf::sample_rough (dielectric_ggx.rs:509-588), front face, no
// energy-compensation table: the weight's x and whether it transmitted.
__device__ __forceinline__ bool dielectric_sample_rough(float eta, float a, V3 wo, float uc, float ux, float cphi,
                                                        float sphi, float& wx, bool& transmitted) {
  const float eta_rel = 1.0f / eta;
  V3 wm;
  if (!sample_wm_vndf(wo, a, a, ux, cphi, sphi, wm)) return false;
  const float cos_wo_wm = dot(wo, wm);
  if (cos_wo_wm <= 0.0f) return false;
  const float f = fresnel_dielectric(cos_wo_wm, 1.0f, eta);
  const float g1 = ggx_g1(wo, a, a);
  if (g1 <= 0.0f) return false;
  float pr = fmaxf(f, 0.0f), pt = fmaxf(1.0f - f, 0.0f);
  const float sum = pr + pt;
  if (sum <= 0.0f) return false;
  pr /= sum;
  pt /= sum;
  if (uc < pr) {
    const V3 wi = reflect_local(wo, wm);
    if (!(wi.z > 0.0f)) return false;
    const float g2 = ggx_g2(wo, wi, a, a);
    const float pdf_wm = pdf_wm_vndf(wo, wm, a, a);
    if (pdf_wm <= 0.0f) return false;
    const float pdf = pr * pdf_wm / (4.0f * cos_wo_wm);
    if (pdf <= 0.0f) return false;
    wx = f * g2 / (pr * g1);
    transmitted = false;
    return true;
  }
  // refract_about_wm (dielectric_ggx.rs:723-738)
  const float cos_o = dot(wo, wm);
  if (cos_o <= 0.0f) return false;
  const float sin2_t = eta_rel * eta_rel * fmaxf(1.0f - cos_o * cos_o, 0.0f);
  if (sin2_t >= 1.0f) return false;
  const float cos_t = sqrtf(fmaxf(1.0f - sin2_t, 0.0f));
  const V3 wi = normalize_or_zero(-eta_rel * wo + (eta_rel * cos_o - cos_t) * wm);
  if (length_sq(wi) == 0.0f) return false;
  if (wi.z >= 0.0f) return false;
  const float cos_wi_wm = dot(wi, wm);
  const float den = cos_wi_wm + eta_rel * cos_wo_wm;
  if (fabsf(den) < 1.0e-6f) return false;
  const float g2 = ggx_g2(wo, wi, a, a);
  const float pdf_wm = pdf_wm_vndf(wo, wm, a, a);
  if (pdf_wm <= 0.0f) return false;
  const float pdf = pt * pdf_wm * fabsf(cos_wi_wm) / (den * den);
  if (pdf <= 0.0f) return false;
  const float radiance_scale = 1.0f / (eta_rel * eta_rel);
  wx = radiance_scale * (1.0f - f) * g2 / (pt * g1);
  transmitted = true;
  return true;
}

// DielectricGgxEnergyCompensationLut::build (directional_albedo.rs:871-898, 977-1023)
__global__ void __launch_bounds__(kLutBlock) lut_dec_kernel(const float* __restrict__ uc, const float* __restrict__ ux,
                                                            const float* __restrict__ cs, float* __restrict__ e) {
  const uint32_t index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= 32u * 32u * 32u) return;
  const int ic = index % 32, ir = (index / 32) % 32, ie = index / 1024;
  const float sqrt_cos = cell_center(ic, 32);
  const float cos_theta = sqrt_cos * sqrt_cos;
  const float roughness = cell_center(ir, 32);
  // dielectric_ec_axis_to_eta (directional_albedo.rs:855-863)
  const float t = clampf(cell_center(ie, 32), 0.0f, 1.0f);
  const float eta = t >= 0.5f ? 1.0f + (t - 0.5f) * 2.0f * (3.0f - 1.0f)
                              : 1.0f / (1.0f + (0.5f - t) * 2.0f * (3.0f - 1.0f));
  const float alpha = clampf(roughness * roughness, kMinAlpha, 1.0f);
  float val;
  if (cos_theta <= 0.0f || eta <= 0.0f) {
    val = 0.0f;
  } else if (alpha < kSmoothAlpha) {
    val = 1.0f;
  } else {
    const float sin_theta = sqrtf(fmaxf(1.0f - cos_theta * cos_theta, 0.0f));
    const V3 wo = V3{sin_theta, 0.0f, cos_theta};
    const float inv_eta_sq = 1.0f / (eta * eta);
    const float a = fmaxf(alpha, kMinAlpha);
    float sum = 0.0f;
    for (int k = 0; k < 4096; ++k) {
      float wx;
      bool tr;
      if (!dielectric_sample_rough(eta, a, wo, __ldg(uc + k), __ldg(ux + k), __ldg(cs + 2 * k), __ldg(cs + 2 * k + 1),
                                   wx, tr))
        continue;
      if (!isfinite(wx)) continue;
      sum += wx * (tr ? inv_eta_sq : 1.0f);
    }
    val = clampf(sum / 4096.0f, 0.0f, 1.0f);
  }
  e[index] = val;
}
}  // namespace

cudaError_t launch_lut_dielectric_albedo(float eta, const float* dirs, const float* phi_cs, float* out,
                                         cudaStream_t s) {
  const unsigned n = 64u * 16u * 64u * 16u;
  lut_da_kernel<<<(n + kLutBlock - 1) / kLutBlock, kLutBlock, 0, s>>>(eta, dirs, phi_cs, out);
  return cudaGetLastError();
}
cudaError_t launch_lut_conductor_e(const float* u, const float* cs, float* e, cudaStream_t s) {
  lut_cec_kernel<<<(4096 + kLutBlock - 1) / kLutBlock, kLutBlock, 0, s>>>(u, cs, e);
  return cudaGetLastError();
}
cudaError_t launch_lut_dielectric_e(const float* uc, const float* ux, const float* cs, float* e, cudaStream_t s) {
  lut_dec_kernel<<<(32768 + kLutBlock - 1) / kLutBlock, kLutBlock, 0, s>>>(uc, ux, cs, e);
  return cudaGetLastError();
}

}  // namespace tpt
