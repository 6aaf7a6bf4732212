// OpenPBR BSDF on the device: evaluation, pdf and sampling of the lowered
// material (DevOpenPbr) in the shading frame.
//
// Restates crates/renderer/src/bsdf/open_pbr.rs (layer_weights 334-406,
// lobe_probabilities 408-437, eval/pdf/sample 224-332, the lobes 560-1022 and
// 1427-1518, finalize_rough_sample 1997-2027, pick_lobe 2043-2070),
// bsdf/eon.rs:60-197, bsdf/smith_ggx.rs:8-175 and the table lookups of
// bsdf/directional_albedo.rs.  Everything that depends on the material alone is
// computed once on the host; OpbrVertex holds what depends on the outgoing
// direction; eval_pdf then evaluates each lobe once for a direction pair and
// shares the half vector and the GGX terms between the metal and specular
// lobes.  The arithmetic order of every term follows the reference (the
// library is compiled with -fmad=false).
#pragma once
#include "render_types.h"
#include "dispersion.cuh"
#include "thin_film.h"
#include "vmath.cuh"

namespace tpt {
namespace opbr {

constexpr float kSmoothAlpha = 1.0e-3f;
constexpr float kMinAlpha = 1.0e-4f;
constexpr float kFracPi2 = 1.57079637050628662f;
constexpr float kMsEps = 1.0e-6f;
constexpr float kRcpPi = 1.0f / kPiF;
constexpr float kC1Fon = 0.5f - 2.0f / (3.0f * kPiF);
constexpr float kC2Fon = 2.0f / 3.0f - 28.0f / (15.0f * kPiF);
constexpr float kEonEps = 1.0e-7f;
constexpr uint32_t kFlagReflection = 1u, kFlagTransmission = 2u, kFlagDiffuse = 4u, kFlagGlossy = 8u,
                   kFlagDelta = 16u;

__device__ __forceinline__ float lum(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
__device__ __forceinline__ V3 splat(float s) { return V3{s, s, s}; }
__device__ __forceinline__ V3 vmaxv(V3 a, V3 b) { return V3{fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
__device__ __forceinline__ V3 vdiv(V3 a, V3 b) { return V3{a.x / b.x, a.y / b.y, a.z / b.z}; }
__device__ __forceinline__ V3 clamp01(V3 v) {
  return V3{fminf(fmaxf(v.x, 0.0f), 1.0f), fminf(fmaxf(v.y, 0.0f), 1.0f), fminf(fmaxf(v.z, 0.0f), 1.0f)};
}
__device__ __forceinline__ V3 ld3(const float* p) { return V3{p[0], p[1], p[2]}; }
// llvm.powi expansions: x^5 = x * x^4, x^6 = x^2 * x^4 with x^4 = x^2 * x^2.
__device__ __forceinline__ float powi5(float x) {
  const float x2 = x * x;
  return x * (x2 * x2);
}
__device__ __forceinline__ float powi6(float x) {
  const float x2 = x * x;
  return x2 * (x2 * x2);
}

// math/mod.rs:50-71
__device__ __forceinline__ float fresnel_dielectric(float cos_i, float eta_i, float eta_t) {
  cos_i = clampf(cos_i, -1.0f, 1.0f);
  if (cos_i < 0.0f) {
    const float t = eta_i;
    eta_i = eta_t;
    eta_t = t;
    cos_i = -cos_i;
  }
  const float sin_i = sqrtf(fmaxf(1.0f - cos_i * cos_i, 0.0f));
  const float sin_t = (eta_i / eta_t) * sin_i;
  if (sin_t >= 1.0f) return 1.0f;
  const float cos_t = sqrtf(fmaxf(1.0f - sin_t * sin_t, 0.0f));
  const float r_par = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t);
  const float r_perp = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t);
  return 0.5f * (r_par * r_par + r_perp * r_perp);
}

// ---- smith_ggx.rs -------------------------------------------------------------
__device__ __forceinline__ float ggx_d(V3 wm, float ax, float ay) {
  if (wm.z <= 0.0f) return 0.0f;
  const float term = wm.x * wm.x / (ax * ax) + wm.y * wm.y / (ay * ay) + wm.z * wm.z;
  const float denom = kPiF * ax * ay * term * term;
  return denom <= 0.0f ? 0.0f : 1.0f / denom;
}
__device__ __forceinline__ float ggx_lambda(V3 w, float ax, float ay) {
  const float c = fabsf(w.z);
  if (c <= 0.0f) return __int_as_float(0x7f800000);
  const float term = 1.0f + (ax * ax * w.x * w.x + ay * ay * w.y * w.y) / (c * c);
  return 0.5f * (-1.0f + sqrtf(term));
}
__device__ __forceinline__ float ggx_g2(V3 wo, V3 wi, float ax, float ay) {
  const float lo = ggx_lambda(wo, ax, ay), li = ggx_lambda(wi, ax, ay);
  if (!isfinite(lo) || !isfinite(li)) return 0.0f;
  return 1.0f / (1.0f + lo + li);
}
__device__ __forceinline__ V3 reflect_local(V3 wo, V3 wm) { return normalize_or_zero(-wo + 2.0f * dot(wo, wm) * wm); }
__device__ __forceinline__ bool half_vector(V3 wo, V3 wi, V3& wm) {
  const V3 m = normalize_or_zero(wo + wi);
  if (length_sq(m) == 0.0f) return false;
  wm = m.z < 0.0f ? -m : m;
  return true;
}
__device__ __forceinline__ bool sample_wm_bounded_vndf(V3 wo, float ax, float ay, float u0, float u1, V3& out) {
  if (wo.z <= 0.0f) return false;
  ax = fmaxf(ax, kMinAlpha);
  ay = fmaxf(ay, kMinAlpha);
  const V3 wo_std = normalize_or_zero(V3{ax * wo.x, ay * wo.y, wo.z});
  if (length_sq(wo_std) == 0.0f) return false;
  const float phi = kTauF * u0;
  const float a = clampf(fminf(ax, ay), 0.0f, 1.0f);
  const float s = 1.0f + sqrtf(wo.x * wo.x + wo.y * wo.y);
  const float a2 = a * a, s2 = s * s;
  const float k = (1.0f - a2) * s2 / (s2 + a2 * wo.z * wo.z);
  const float lower = wo.z > 0.0f ? -k * wo_std.z : -wo_std.z;
  const float z = __fmaf_rn(lower, u1, 1.0f - u1);
  const float sin_theta = sqrtf(clampf(1.0f - z * z, 0.0f, 1.0f));
  const V3 o_std = V3{sin_theta * cosf(phi), sin_theta * sinf(phi), z};
  const V3 wm_std = wo_std + o_std;
  const V3 wm = normalize_or_zero(V3{ax * wm_std.x, ay * wm_std.y, wm_std.z});
  if (length_sq(wm) == 0.0f || wm.z <= 0.0f) return false;
  out = wm;
  return true;
}
__device__ __forceinline__ float pdf_wm_bounded_vndf(V3 wo, V3 wm, float ax, float ay) {
  if (wo.z <= 0.0f || wm.z <= 0.0f) return 0.0f;
  ax = fmaxf(ax, kMinAlpha);
  ay = fmaxf(ay, kMinAlpha);
  const float a = clampf(fminf(ax, ay), 0.0f, 1.0f);
  const float s = 1.0f + sqrtf(wo.x * wo.x + wo.y * wo.y);
  const float a2 = a * a, s2 = s * s;
  const float k = (1.0f - a2) * s2 / (s2 + a2 * wo.z * wo.z);
  const float t = sqrtf(ax * ax * wo.x * wo.x + ay * ay * wo.y * wo.y + wo.z * wo.z);
  const float denom = k * wo.z + t;
  if (denom <= 0.0f) return 0.0f;
  return 2.0f * ggx_d(wm, ax, ay) * fmaxf(dot(wo, wm), 0.0f) / denom;
}
__device__ __forceinline__ float ggx_g1(V3 w, float ax, float ay) {
  const float l = ggx_lambda(w, ax, ay);
  if (!isfinite(l)) return 0.0f;
  return 1.0f / (1.0f + l);
}
// smith_ggx.rs:62-75
__device__ __forceinline__ float pdf_wm_vndf(V3 wo, V3 wm, float ax, float ay) {
  if (!(wo.z > 0.0f) || wm.z <= 0.0f) return 0.0f;
  const float d = ggx_d(wm, ax, ay);
  const float g1 = ggx_g1(wo, ax, ay);
  const float c = fmaxf(dot(wo, wm), 0.0f);
  if (d <= 0.0f || g1 <= 0.0f || c <= 0.0f) return 0.0f;
  return d * g1 * c / wo.z;
}
// sample_wm_vndf, Heitz 2018 (smith_ggx.rs:77-123)
__device__ __forceinline__ bool sample_wm_vndf(V3 wo, float ax, float ay, float u0, float u1, V3& out) {
  if (wo.z <= 0.0f) return false;
  ax = fmaxf(ax, kMinAlpha);
  ay = fmaxf(ay, kMinAlpha);
  const V3 wo_std = normalize_or_zero(V3{ax * wo.x, ay * wo.y, wo.z});
  if (length_sq(wo_std) == 0.0f) return false;
  const float lensq = wo_std.x * wo_std.x + wo_std.y * wo_std.y;
  const V3 t1 = lensq > 0.0f ? V3{-wo_std.y, wo_std.x, 0.0f} / sqrtf(lensq) : V3{1.0f, 0.0f, 0.0f};
  const V3 t2 = cross(wo_std, t1);
  const float r = sqrtf(clampf(u0, 0.0f, 1.0f));
  const float phi = kTauF * u1;
  const float p1 = r * cosf(phi);
  float p2 = r * sinf(phi);
  const float s = 0.5f * (1.0f + wo_std.z);
  p2 = (1.0f - s) * sqrtf(fmaxf(1.0f - p1 * p1, 0.0f)) + s * p2;
  const V3 nh = p1 * t1 + p2 * t2 + sqrtf(fmaxf(1.0f - p1 * p1 - p2 * p2, 0.0f)) * wo_std;
  const V3 wm = normalize_or_zero(V3{ax * nh.x, ay * nh.y, fmaxf(nh.z, 0.0f)});
  if (length_sq(wm) == 0.0f || wm.z <= 0.0f) return false;
  out = wm;
  return true;
}
// math/mod.rs:83-100 (refraction about +z) and refract_about (open_pbr.rs:2043-2058)
__device__ __forceinline__ bool refract_z(V3 wo, float eta, V3& out) {
  if (wo.z <= 0.0f) return false;
  const float sin2_o = fmaxf(1.0f - wo.z * wo.z, 0.0f);
  const float sin2_t = eta * eta * sin2_o;
  if (sin2_t >= 1.0f) return false;
  const float cos_t = sqrtf(fmaxf(1.0f - sin2_t, 0.0f));
  const V3 wi = normalize_or_zero(V3{-eta * wo.x, -eta * wo.y, -cos_t});
  if (length_sq(wi) == 0.0f) return false;
  out = wi;
  return true;
}
__device__ __forceinline__ bool refract_about(V3 wo, V3 wm, float eta, V3& out) {
  const float cos_o = dot(wo, wm);
  if (cos_o <= 0.0f) return false;
  const float sin2_t = eta * eta * fmaxf(1.0f - cos_o * cos_o, 0.0f);
  if (sin2_t >= 1.0f) return false;
  const float cos_t = sqrtf(fmaxf(1.0f - sin2_t, 0.0f));
  const V3 wi = normalize_or_zero(-eta * wo + (eta * cos_o - cos_t) * wm);
  if (length_sq(wi) == 0.0f) return false;
  out = wi;
  return true;
}
// math/mod.rs:26-40
__device__ __forceinline__ V3 sample_cosine_hemisphere(float u0, float u1) {
  const float r = sqrtf(clampf(u0, 0.0f, 1.0f));
  const float phi = kTauF * u1;
  const float dx = r * cosf(phi), dy = r * sinf(phi);
  return V3{dx, dy, sqrtf(fmaxf(1.0f - (dx * dx + dy * dy), 0.0f))};
}
__device__ __forceinline__ float cosine_pdf(float c) { return fmaxf(c, 0.0f) / kPiF; }

// ---- table lookups (directional_albedo.rs:388-408, 203-238, 750-779, 928-974)
__device__ __forceinline__ DevLerpAxis axis_lerp(float value, int resolution) {
  const float position = clampf(value, 0.0f, 1.0f) * (float)resolution - 0.5f;
  if (position <= 0.0f) return DevLerpAxis{0u, 0u, 0.0f};
  const int max_index = resolution - 1;
  if (position >= (float)max_index) return DevLerpAxis{(uint32_t)max_index, (uint32_t)max_index, 0.0f};
  const int lower = (int)floorf(position);
  return DevLerpAxis{(uint32_t)lower, (uint32_t)lower + 1u, position - (float)lower};
}

// DielectricGgxDirectionalAlbedoLut::lookup(w, roughness proxy, anisotropy 0)
static __device__ __noinline__ float da_lookup(const float* __restrict__ tab, float eta, bool smooth, DevLerpAxis r, V3 w) {
  if (w.z <= 0.0f) return 0.0f;
  if (smooth) return fresnel_dielectric(clampf(w.z, 0.0f, 1.0f), 1.0f, eta);
  const float sqrt_cos = sqrtf(clampf(w.z, 0.0f, 1.0f));
  const float phi = ((w.x == 0.0f && w.y == 0.0f) ? 0.0f : atan2f(fabsf(w.y), fabsf(w.x))) / kFracPi2;
  const DevLerpAxis c = axis_lerp(sqrt_cos, 64), p = axis_lerp(phi, 16);
  const uint32_t ci[2] = {c.lo, c.hi}, pi[2] = {p.lo, p.hi}, ri[2] = {r.lo, r.hi};
  const float cw[2] = {1.0f - c.t, c.t}, pw[2] = {1.0f - p.t, p.t}, rw[2] = {1.0f - r.t, r.t};
  float value = 0.0f;
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y)
#pragma unroll
      for (int z = 0; z < 2; ++z) {
        // anisotropy 0 sits at position 7.5 of its 16 cells: indices 7 and 8, weights 1/2
        const float* row = tab + ((size_t)(ci[x] * 16u + pi[y]) * 64u + ri[z]) * 16u;
        const float wxyz = cw[x] * pw[y] * rw[z];
        value += wxyz * 0.5f * __ldg(row + 7);
        value += wxyz * 0.5f * __ldg(row + 8);
      }
  return clampf(value, 0.0f, 1.0f);
}

// DielectricGgxEnergyCompensationLut::lookup_e with the material's axes
__device__ __forceinline__ float dec_lookup_e(const float* __restrict__ e, const DevMsFace& f, float cos_theta) {
  const float sqrt_cos = sqrtf(clampf(cos_theta, 0.0f, 1.0f));
  const DevLerpAxis c = axis_lerp(sqrt_cos, 32);
  const uint32_t hi[2] = {f.eta_axis.lo, f.eta_axis.hi}, ri[2] = {f.r_axis.lo, f.r_axis.hi}, ci[2] = {c.lo, c.hi};
  const float hw[2] = {1.0f - f.eta_axis.t, f.eta_axis.t}, rw[2] = {1.0f - f.r_axis.t, f.r_axis.t},
              cw[2] = {1.0f - c.t, c.t};
  float value = 0.0f;
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y)
#pragma unroll
      for (int z = 0; z < 2; ++z) value += hw[x] * rw[y] * cw[z] * __ldg(e + (hi[x] * 32u + ri[y]) * 32u + ci[z]);
  return clampf(value, 0.0f, 1.0f);
}

// ConductorGgxEnergyCompensationLut::lookup_e
__device__ __forceinline__ float cec_lookup_e(const float* __restrict__ e, DevLerpAxis r, float cos_theta) {
  const float sqrt_cos = sqrtf(clampf(cos_theta, 0.0f, 1.0f));
  const DevLerpAxis c = axis_lerp(sqrt_cos, 64);
  const uint32_t ci[2] = {c.lo, c.hi}, ri[2] = {r.lo, r.hi};
  const float cw[2] = {1.0f - c.t, c.t}, rw[2] = {1.0f - r.t, r.t};
  float value = 0.0f;
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y) value += cw[x] * rw[y] * __ldg(e + ri[y] * 64u + ci[x]);
  return clampf(value, 0.0f, 1.0f);
}

// ---- EON diffuse (eon.rs) with rho = 1 ---------------------------------------
__device__ __forceinline__ float e_fon_approx(float mu, float r) {
  const float mc = 1.0f - mu;
  const float g = mc * (0.05710853f + mc * (0.49188188f + mc * (-0.33218145f + mc * 0.071443f)));
  return (1.0f + r * g) / (1.0f + kC1Fon * r);
}
__device__ __forceinline__ float f_eon_white(float r, V3 wo, V3 wi) {
  const float mu_o = wo.z, mu_i = wi.z;
  const float s = dot(wo, wi) - mu_i * mu_o;
  const float s_over_t = s > 0.0f ? s / fmaxf(mu_o, mu_i) : s;
  const float af = 1.0f / (1.0f + kC1Fon * r);
  const float f_ss = 1.0f * (kRcpPi * af * (1.0f + r * s_over_t));
  const float e_fo = e_fon_approx(mu_o, r), e_fi = e_fon_approx(mu_i, r);
  const float avg_ef = af * (1.0f + kC2Fon * r);
  const float oma = 1.0f - avg_ef;
  const float rho_ms = 1.0f * 1.0f * avg_ef / (1.0f - 1.0f * oma);
  const float scale = kRcpPi * fmaxf(1.0f - e_fo, kEonEps) * fmaxf(1.0f - e_fi, kEonEps) / fmaxf(oma, kEonEps);
  return f_ss + rho_ms * scale;
}
struct Ltc {
  float a, b, c, d;
};
__device__ __forceinline__ Ltc ltc_coeffs(float mu, float r) {
  Ltc l;
  l.a = 1.0f + r * (0.303392f + (-0.518982f + 0.111709f * mu) * mu + (-0.276266f + 0.335918f * mu) * r);
  l.b = r * (-1.16407f + 1.15859f * mu + (0.150815f - 0.150105f * mu) * r) / (mu * mu * mu - 1.43545f);
  l.c = 1.0f + r * (0.20013f + (-0.506373f + 0.261777f * mu) * mu);
  l.d = r * (0.540852f + (-1.01625f + 0.475392f * mu) * mu) / (-1.0743f + (0.0725628f + mu) * mu);
  return l;
}
__device__ __forceinline__ void ltc_basis(V3 wo, float& xx, float& xy) {
  const float len_sqr = wo.x * wo.x + wo.y * wo.y;
  if (len_sqr > 0.0f) {
    const float inv = 1.0f / sqrtf(len_sqr);
    xx = wo.x * inv;
    xy = wo.y * inv;
  } else {
    xx = 1.0f;
    xy = 0.0f;
  }
}
__device__ __forceinline__ float cltc_pdf(V3 wo, V3 wi, float r) {
  float xx, xy;
  ltc_basis(wo, xx, xy);
  const float yx = -xy, yy = xx;
  const V3 w = V3{xx * wi.x + xy * wi.y, yx * wi.x + yy * wi.y, wi.z};
  const Ltc l = ltc_coeffs(wo.z, r);
  const float det_m = l.c * (l.a - l.b * l.d);
  const V3 wh = V3{l.c * (w.x - l.b * w.z), (l.a - l.b * l.d) * w.y, -l.c * (l.d * w.x - l.a * w.z)};
  const float lensq = fmaxf(dot(wh, wh), 1.0e-30f);
  const float vz = 1.0f / sqrtf(l.d * l.d + 1.0f);
  const float s = 0.5f * (1.0f + vz);
  const float q = det_m / lensq;
  return q * q * fmaxf(wh.z, 0.0f) / (kPiF * s);
}
__device__ __forceinline__ float eon_pdf(float r, float r_pow01, V3 wo, V3 wi) {
  const float mu = wo.z;
  const float p_u = r_pow01 * (0.162925f + (-0.372058f + (0.538233f - 0.290822f * mu) * mu) * mu);
  const float p_c = 1.0f - p_u;
  return p_u * (1.0f / (2.0f * kPiF)) + p_c * cltc_pdf(wo, wi, r);
}
// EonBsdf::sample up to its validity test; the OpenPBR layer recomputes pdf and f.
static __device__ __noinline__ bool eon_sample_dir(float r, float r_pow01, V3 wo, float u1, float u2, V3& wi_out) {
  const float mu = wo.z;
  const float p_u = r_pow01 * (0.162925f + (-0.372058f + (0.538233f - 0.290822f * mu) * mu) * mu);
  const float p_c = 1.0f - p_u;
  V3 wi;
  float pdf_c;
  if (u1 < p_u) {
    const float u1n = u1 / p_u;
    const float st = sqrtf(fmaxf(1.0f - u1n * u1n, 0.0f));
    const float phi = 2.0f * kPiF * u2;
    wi = V3{st * cosf(phi), st * sinf(phi), u1n};
    pdf_c = cltc_pdf(wo, wi, r);
  } else {
    const float u1n = (u1 - p_u) / fmaxf(p_c, 1.0e-30f);
    const Ltc l = ltc_coeffs(wo.z, r);
    const float radius = sqrtf(u1n);
    const float phi = 2.0f * kPiF * u2;
    const float x0 = radius * cosf(phi), y0 = radius * sinf(phi);
    const float vz = 1.0f / sqrtf(l.d * l.d + 1.0f);
    const float s = 0.5f * (1.0f + vz);
    const float edge = sqrtf(fmaxf(1.0f - y0 * y0, 0.0f));
    const float x = -((1.0f - s) * edge + s * x0);
    const float y = y0;
    const V3 wh = V3{x, y, sqrtf(fmaxf(1.0f - (x * x + y * y), 0.0f))};
    const float pdf_wh = wh.z / (kPiF * s);
    const V3 w_ltc = V3{l.a * wh.x + l.b * wh.z, l.c * wh.y, l.d * wh.x + wh.z};
    const float len = length(w_ltc);
    const float det_m = l.c * (l.a - l.b * l.d);
    pdf_c = pdf_wh * (len * len * len) / det_m;
    const V3 v = w_ltc / len;
    float xx, xy;
    ltc_basis(wo, xx, xy);
    const float yx = -xy, yy = xx;
    wi = V3{xx * v.x + yx * v.y, xy * v.x + yy * v.y, v.z};
  }
  const float pdf = p_u * (1.0f / (2.0f * kPiF)) + p_c * pdf_c;
  if (pdf <= 0.0f || wi.z <= 0.0f) return false;
  wi_out = wi;
  return true;
}

// ---- fuzz (open_pbr.rs:148-205, 2070-2123) ------------------------------------
__device__ __forceinline__ float zeltner_albedo(float ndot_v, float roughness) {
  const float x = clampf(ndot_v, 0.0f, 1.0f), y = clampf(roughness, 0.01f, 1.0f);
  const float s = y * (0.0206607f + 1.58491f * y) / (0.0379424f + y * (1.32227f + y));
  const float m = y * (-0.193854f + y * (-1.14885f + y * (1.7932f - 0.95943f * y * y))) / (0.046391f + y);
  const float o = y * (0.000654023f + (-0.0207818f + 0.119681f * y) * y) / (1.26264f + y * (-1.92021f + y));
  const float q = (x - m) / s;
  return expf(-0.5f * (q * q)) / (s * sqrtf(2.0f * kPiF)) + o;
}
__device__ __forceinline__ float zeltner_a_inv(float ndot_v, float roughness) {
  const float x = clampf(ndot_v, 0.0f, 1.0f), y = clampf(roughness, 0.01f, 1.0f);
  return (2.58126f * x + 0.813703f * y) * y / (1.0f + 0.310327f * x * x + 2.60994f * x * y);
}
__device__ __forceinline__ float zeltner_b_inv(float ndot_v, float roughness) {
  const float x = clampf(ndot_v, 0.0f, 1.0f), y = clampf(roughness, 0.01f, 1.0f);
  return sqrtf(1.0f - x) * (y - 1.0f) * y * y * y / (0.0000254053f + 1.71228f * x - 1.71506f * x * y + 1.34174f * y * y);
}
__device__ __forceinline__ float eval_ltc(V3 wi, float a_inv, float b_inv) {
  V3 w = V3{a_inv * wi.x + b_inv * wi.z, a_inv * wi.y, wi.z};
  const float len = length(w);
  if (len <= 0.0f) return 0.0f;
  w = w / len;
  if (w.z <= 0.0f) return 0.0f;
  const float det = a_inv * a_inv;
  const float jac = det / (len * len * len);
  return (w.z / kPiF) * jac;
}
__device__ __forceinline__ float phi_of(V3 v) {
  const float p = atan2f(v.y, v.x);
  return p < 0.0f ? p + 2.0f * kPiF : p;
}
__device__ __forceinline__ V3 rotate_z(V3 v, float angle) {
  const float s = sinf(angle), c = cosf(angle);
  return V3{c * v.x - s * v.y, s * v.x + c * v.y, v.z};
}
// fuzz eval (returns the scalar of the splat) and pdf for wo.z, wi.z > 0
static __device__ __noinline__ void fuzz_eval_pdf(float r, V3 wo, V3 wi, float& f, float& pdf) {
  const V3 w = rotate_z(wi, -phi_of(wo));
  const float a = zeltner_a_inv(wo.z, r), b = zeltner_b_inv(wo.z, r);
  const float v = eval_ltc(w, a, b);
  f = zeltner_albedo(wo.z, r) * v / fmaxf(wi.z, 1.0e-6f);
  pdf = v;
}
static __device__ __noinline__ bool fuzz_sample_dir(float r, V3 wo, float u0, float u1, V3& wi) {
  if (wo.z <= 0.0f) return false;
  const float a = zeltner_a_inv(wo.z, r), b = zeltner_b_inv(wo.z, r);
  const float phi = 2.0f * kPiF * u0;
  const float ct = sqrtf(u1), st = sqrtf(fmaxf(1.0f - u1, 0.0f));
  const V3 w = V3{cosf(phi) * st, sinf(phi) * st, ct};
  const V3 ws = normalize_or_zero(V3{w.x / a - w.z * b / a, w.y / a, w.z});
  if (ws.z <= 0.0f) return false;
  const V3 v = rotate_z(ws, phi_of(wo));
  if (v.z <= 0.0f) return false;
  wi = v;
  return true;
}

// ---- open_pbr.rs helpers ------------------------------------------------------
__device__ __forceinline__ float weighted_fresnel_ratio(float c, float eta_ti, float eta_tp) {
  eta_ti = fmaxf(eta_ti, 1.0e-4f);
  eta_tp = fmaxf(eta_tp, 1.0e-4f);
  if (eta_tp >= 1.0f) return fresnel_dielectric(c, 1.0f, eta_tp);
  const float cc = clampf(c, 0.0f, 1.0f);
  const float mu2_t = 1.0f - (1.0f - cc * cc) / (eta_ti * eta_ti);
  if (mu2_t <= 0.0f) return 1.0f;
  return fresnel_dielectric(sqrtf(mu2_t), 1.0f, 1.0f / eta_tp);
}
__device__ __forceinline__ float refracted_cos(float mu, float eta) {
  const float m = clampf(mu, 0.0f, 1.0f);
  const float sin2_t = fmaxf(1.0f - m * m, 0.0f) / fmaxf(eta * eta, kMsEps);
  return sqrtf(fmaxf(1.0f - sin2_t, 0.0f));
}

// Per-vertex state: everything of OpenPbrBsdf that depends on wo only.
struct OpbrVertex {
  const DevOpenPbr* m;
  const float* cec_e;
  const float* dec_e;
  V3 wo;
  uint32_t face;       // 0 front, 1 back
  float dk_cos;        // |wo.z| of the vertex the BSDF was built for
  float below_fuzz_s;  // max(1 - fuzz * E_fuzz, 0)
  float e_coat;        // coat albedo (with multiple scattering)
  float e_spec;        // specular albedo (with multiple scattering)
  float dec_eo[2];     // dielectric E(wo) of the specular and coat lobes
  float cec_eo;        // conductor E(wo)
  V3 darkening;
  V3 tw_r, tw_t;  // thin_wall_coefficients(|wo.z|) of thin-walled materials
  float q_coat, q_metal, q_spec, q_btdf, q_fuzz, q_diff, q_total;
  // the path state of the shading vertex (ShadingVertex::path_throughput and
  // wavelength_lock, lock < 0: none); read by dispersive transmission only
  V3 thr;
  float lock;
};

// LayerWeights below the coat for a given coat tint (open_pbr.rs:334-406);
// the diffuse BTDF's weight is zero (subsurface is forced to 0 on add)
struct Below {
  V3 metal, spec, btdf, diff;
};
__device__ __forceinline__ Below weights_below(const OpbrVertex& s, V3 tint) {
  const DevOpenPbr& m = *s.m;
  const V3 one = V3{1.0f, 1.0f, 1.0f};
  const V3 below_fuzz = splat(s.below_fuzz_s);
  V3 under_coat = below_fuzz;
  if (m.coat > 0.0f) {
    const V3 thr = s.darkening * tint * splat(fmaxf(1.0f - s.e_coat, 0.0f));
    under_coat = below_fuzz * (one * (1.0f - m.coat) + thr * m.coat);
  }
  Below b;
  b.metal = m.metalness * under_coat;
  const V3 below_metal = (1.0f - m.metalness) * under_coat;
  const V3 sc = ld3(m.specular_color);
  b.spec = below_metal * sc;
  const V3 below_spec = below_metal * vmaxv(one - sc * s.e_spec, V3{0.0f, 0.0f, 0.0f});
  const V3 trans_tint = (m.flags & kOpbrThinWalled) ? one : ld3(m.trans_color);
  b.btdf = below_spec * m.transmission * trans_tint;
  const V3 below_trans = below_spec * (1.0f - m.transmission);
  b.diff = below_trans * ((1.0f - 0.0f) * m.base) * ld3(m.base_color);
  return b;
}

__device__ __forceinline__ float spec_fresnel(const DevOpenPbr& m, uint32_t face, float c) {
  const DevFresnelFace& f = m.fres[face];
  const float unc = weighted_fresnel_ratio(c, f.unc_ti, f.unc_tp);
  if (m.coat_clamped <= 0.0f) return unc;
  const float coated = weighted_fresnel_ratio(c, f.coat_ti, f.coat_tp);
  return unc + (coated - unc) * m.coat_clamped;
}

__device__ __forceinline__ V3 from_film(film::F3 a) { return V3{a.x, a.y, a.z}; }
// A dielectric Fresnel blended with the thin film's reflectance over a base
// of eta `eta_base` (over the coat's eta where coated): spec_brdf_fresnel
// (open_pbr.rs:869-898) and spec_btdf_fresnel_with_eta (1120-1152).
__device__ __forceinline__ V3 filmed_dielectric(const DevOpenPbr& m, V3 no_film, float c, float eta_base) {
  film::F3 f = film::film_dielectric(c, 1.0f, m.film_ior, eta_base, m.film_thick);
  if (m.coat > 0.0f)
    f = film::lerp3(f, film::film_dielectric(c, m.coat_eta, m.film_ior, eta_base, m.film_thick),
                    clampf(m.coat, 0.0f, 1.0f));
  return no_film + (from_film(f) - no_film) * m.film_w;
}
// spec_brdf_fresnel: per channel once a film is present
__device__ __forceinline__ V3 spec_fresnel3(const DevOpenPbr& m, uint32_t face, float c) {
  const V3 no_film = splat(spec_fresnel(m, face, c));
  return (m.flags & kOpbrFilm) ? filmed_dielectric(m, no_film, c, m.trans_eta) : no_film;
}

// thin_wall_coefficients (open_pbr.rs:931-959, thin_wall_internal_fresnel
// 961-979) without thin film: reflectance and transmittance of the slab.
__device__ __forceinline__ void thin_wall_coeffs(const DevOpenPbr& m, uint32_t face, float cos_theta_o, V3& r_out,
                                                 V3& t_out) {
  const V3 one = V3{1.0f, 1.0f, 1.0f}, zero = V3{0.0f, 0.0f, 0.0f};
  const float eta = fmaxf(m.trans_eta, 1.0e-4f);
  const float eta_prime = fmaxf(m.trans_eta, 1.0e-4f);  // specular_eta = transmission_eta
  const float cos_o = clampf(cos_theta_o, 0.0f, 1.0f);
  const float sin2_o = fmaxf(1.0f - cos_o * cos_o, 0.0f);
  const float sin2_i = clampf(sin2_o / (eta * eta), 0.0f, 1.0f);
  const float cos_i = fmaxf(sqrtf(1.0f - sin2_i), 1.0e-4f);
  const V3 f_o = clamp01(spec_fresnel3(m, face, cos_o));
  V3 f_i = splat(weighted_fresnel_ratio(cos_i, 1.0f / fmaxf(eta, 1.0e-4f), 1.0f / fmaxf(eta_prime, 1.0e-4f)));
  if (m.flags & kOpbrFilm)
    f_i = f_i + (from_film(film::film_dielectric(cos_i, fmaxf(eta, 1.0e-4f), m.film_ior, 1.0f, m.film_thick)) - f_i) *
                    m.film_w;
  f_i = clamp01(f_i);
  const float e = 1.0f / cos_i;
  const V3 tc = clamp01(ld3(m.trans_color));
  const V3 a = V3{powf(tc.x, e), powf(tc.y, e), powf(tc.z, e)};
  const V3 a2 = a * a;
  const V3 f_i2_a2 = a2 * f_i * f_i;
  const V3 denom = vmaxv(one - f_i2_a2, splat(1.0e-6f));
  const V3 omfo = vmaxv(one - f_o, zero);
  const V3 omfi = vmaxv(one - f_i, zero);
  r_out = clamp01(f_o + vdiv(omfo * omfi * f_i * a2, denom));
  t_out = clamp01(omfo * omfi * a * (one + vdiv(f_i2_a2, denom)));
}

__device__ __forceinline__ float albedo_with_ms(const OpbrVertex& s, int lobe, bool alpha_rough, float ss) {
  if (s.wo.z <= 0.0f || !alpha_rough) return clampf(ss, 0.0f, 1.0f);
  const DevMsFace& f = s.m->ms[lobe][s.face];
  return clampf(ss + f.ms_factor * fmaxf(1.0f - s.dec_eo[lobe], 0.0f), 0.0f, 1.0f);
}

// Builds the per-vertex state (make_bsdf's view-dependent part, the albedos,
// layer weights without wi and the lobe probabilities) for outgoing direction
// `wo`.  `dk_cos` is |wo.z| of the shading vertex the BSDF was built for (the
// coat darkening reads it); it differs from |wo.z| only when the state is
// evaluated at another direction of the same BSDF (pdf_rev, importance layers).
static __device__ __noinline__ void init_vertex(OpbrVertex& s, const DevOpenPbr* mp, const float* cec_e,
                                                const float* dec_e, V3 wo, bool front_face, float dk_cos) {
  const DevOpenPbr& m = *mp;
  s.m = mp;
  s.cec_e = cec_e;
  s.dec_e = dec_e;
  s.wo = wo;
  s.face = front_face ? 0u : 1u;
  s.dk_cos = dk_cos;
  s.thr = V3{1.0f, 1.0f, 1.0f};
  s.lock = -1.0f;
  // coat_darkening_factor's view term (material/open_pbr.rs:836-857)
  s.darkening = V3{1.0f, 1.0f, 1.0f};
  if (m.flags & kOpbrDarkening) {
    const float ks = fresnel_dielectric(clampf(dk_cos, 0.0f, 1.0f), 1.0f, m.dk_eta);
    const float k = clampf(ks + (m.dk_kr - ks) * m.dk_rb, 0.0f, 1.0f);
    const V3 cc = ld3(m.coat_color);
    const V3 denom = vmaxv(V3{1.0f, 1.0f, 1.0f} - ld3(m.dk_e_base) * (k * cc), splat(1.0e-4f));
    const V3 delta_factor = vdiv(splat(fmaxf(1.0f - k, 0.0f)), denom);
    const V3 one = V3{1.0f, 1.0f, 1.0f};
    s.darkening = clamp01(one + (delta_factor - one) * m.dk_wd);
  }
  const bool spec_alpha_rough = !(fmaxf(m.spec_ax, m.spec_ay) < kSmoothAlpha);
  const bool coat_alpha_rough = !(fmaxf(m.coat_ax, m.coat_ay) < kSmoothAlpha);
  s.dec_eo[0] = spec_alpha_rough && wo.z > 0.0f ? dec_lookup_e(dec_e, m.ms[0][s.face], wo.z) : 0.0f;
  s.dec_eo[1] = (m.coat > 0.0f && coat_alpha_rough && wo.z > 0.0f) ? dec_lookup_e(dec_e, m.ms[1][s.face], wo.z) : 0.0f;
  s.cec_eo = (m.flags & kOpbrMetalRough) ? cec_lookup_e(cec_e, m.cond_r, wo.z) : 0.0f;
  const float e_fuzz = m.fuzz > 0.0f ? zeltner_albedo(clampf(wo.z, 0.0f, 1.0f), m.fuzz_roughness) : 0.0f;
  s.below_fuzz_s = fmaxf(1.0f - m.fuzz * e_fuzz, 0.0f);
  s.e_coat = 0.0f;
  if (m.coat > 0.0f && wo.z > 0.0f) {
    const float ss = da_lookup(m.coat_da, m.coat_da_eta, (m.flags & kOpbrCoatDaSmooth) != 0, m.coat_da_r, wo);
    s.e_coat = albedo_with_ms(s, 1, coat_alpha_rough, ss);
  }
  s.e_spec = 0.0f;
  if (wo.z > 0.0f) {
    const float ss = da_lookup(m.spec_da, m.spec_da_eta, (m.flags & kOpbrSpecDaSmooth) != 0, m.spec_da_r, wo);
    // thin-walled: the single-scattering albedo alone (open_pbr.rs:485-487)
    s.e_spec = (m.flags & kOpbrThinWalled) ? ss : albedo_with_ms(s, 0, spec_alpha_rough, ss);
  }
  if (m.flags & kOpbrThinWalled) thin_wall_coeffs(m, s.face, fabsf(wo.z), s.tw_r, s.tw_t);
  const Below b = weights_below(s, ld3(m.coat_color));
  s.q_coat = m.coat > 0.0f ? m.coat * s.below_fuzz_s : 0.0f;
  s.q_metal = lum(b.metal * (splat(0.5f) + 0.5f * ld3(m.base_color)));
  s.q_spec = lum(b.spec);
  s.q_btdf = (m.flags & kOpbrTrans) ? fmaxf(lum(b.btdf), 0.0f) : 0.0f;
  s.q_fuzz = fmaxf(lum(m.fuzz * ld3(m.fuzz_color)), 0.0f);
  s.q_diff = fmaxf(lum(b.diff), 0.0f);
  s.q_total = s.q_coat + s.q_metal + s.q_spec + s.q_btdf + s.q_fuzz + s.q_diff;
}

// metal_fresnel (open_pbr.rs:761-802): F82 tint, blended with the filmed
// conductor's reflectance when the material has a thin film
__device__ __forceinline__ V3 metal_fresnel(const DevOpenPbr& m, float c) {
  const V3 f0 = ld3(m.f0);
  const float om = 1.0f - clampf(c, 0.0f, 1.0f);
  const V3 fs = f0 + (V3{1.0f, 1.0f, 1.0f} - f0) * powi5(om);
  const float cc = clampf(c, 0.0f, 1.0f);
  const float corr = cc * powi6(1.0f - cc) / m.f82_denom;
  const V3 no_film = clamp01(m.specular * (fs - corr * ld3(m.f82_delta)));
  if (!(m.flags & kOpbrFilm)) return no_film;
  const film::F3 n = film::F3{m.metal_n[0], m.metal_n[1], m.metal_n[2]};
  const film::F3 k = film::F3{m.metal_k[0], m.metal_k[1], m.metal_k[2]};
  film::F3 f = film::film_conductor(c, 1.0f, m.film_ior, n, k, m.film_thick);
  if (m.coat > 0.0f)
    f = film::lerp3(f, film::film_conductor(c, m.coat_eta, m.film_ior, n, k, m.film_thick), clampf(m.coat, 0.0f, 1.0f));
  return no_film + (from_film(f) - no_film) * m.film_w;
}
__device__ __forceinline__ float refl_ms(const OpbrVertex& s, int lobe, float wi_z) {
  const DevMsFace& f = s.m->ms[lobe][s.face];
  const float e_i = dec_lookup_e(s.dec_e, f, wi_z);
  return f.ms_factor * (1.0f - s.dec_eo[lobe]) * (1.0f - e_i) / (kPiF * f.one_minus_e_avg_o);
}

// coat_absorb_tint (open_pbr.rs:453-464) for a (layer wo, wi) pair, wi.z > 0
__device__ __forceinline__ V3 coat_tint(const DevOpenPbr& m, V3 wo, V3 wi) {
  if (wo.z <= 0.0f || wi.z <= 0.0f) return V3{1.0f, 1.0f, 1.0f};
  const float mu_o = refracted_cos(wo.z, m.coat_eta), mu_i = refracted_cos(wi.z, m.coat_eta);
  const float e = 0.5f * (1.0f / fmaxf(mu_i, 1.0e-4f) + 1.0f / fmaxf(mu_o, 1.0e-4f));
  return V3{powf(fmaxf(m.coat_color[0], 0.0f), e), powf(fmaxf(m.coat_color[1], 0.0f), e),
            powf(fmaxf(m.coat_color[2], 0.0f), e)};
}

// ---- dispersion (open_pbr.rs:1223-1427, 1670-1928) --------------------------
// The transmission eta is a Cauchy function of wavelength.  make_bsdf sets
// transmission_eta = specular_eta, so the refraction eta and the Fresnel /
// multiple-scattering eta of one wavelength are the same number here, and the
// host-lowered constants of the non-dispersive path are replaced by their
// values at that eta: the Fresnel arguments, dielectric_ms_params'
// transmission half (over the energy-compensation tables; roughness_eq does
// not depend on eta, so its table axis is the lowered one).
__device__ __forceinline__ float f_avg_dielectric(float eta) {  // open_pbr.rs:2183-2191
  if (eta >= 1.0f) return clampf((eta - 1.0f) / (4.08567f + 1.00071f * eta), 0.0f, 1.0f);
  const float e = fmaxf(eta, kMsEps);
  const float v = 0.997118f + 0.1014f * e - 0.965241f * e * e - 0.130607f * e * e * e;
  return clampf(v, 0.0f, 1.0f);
}
__device__ __forceinline__ float dec_eta_to_axis(float eta) {  // directional_albedo.rs:845-853
  const float kMinInv = 1.0f / 3.0f, kMax = 3.0f;
  eta = clampf(eta, kMinInv, kMax);
  if (eta >= 1.0f) return 0.5f + 0.5f * ((eta - 1.0f) / (kMax - 1.0f));
  const float inv = 1.0f / eta;
  return 0.5f - 0.5f * ((inv - 1.0f) / (kMax - 1.0f));
}
// DielectricGgxEnergyCompensationLut::lookup_e_avg / lookup_e at given axes
__device__ __forceinline__ float dec_e_avg_at(const float* __restrict__ e_avg, DevLerpAxis r, DevLerpAxis h) {
  const uint32_t ri[2] = {r.lo, r.hi}, hi[2] = {h.lo, h.hi};
  const float rw[2] = {1.0f - r.t, r.t}, hw[2] = {1.0f - h.t, h.t};
  float value = 0.0f;
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y) value += hw[x] * rw[y] * __ldg(e_avg + hi[x] * 32u + ri[y]);
  return clampf(value, 0.0f, 1.0f);
}
__device__ __forceinline__ float dec_e_at(const float* __restrict__ e, DevLerpAxis h, DevLerpAxis r, float cos_theta) {
  DevMsFace f;
  f.eta_axis = h;
  f.r_axis = r;
  return dec_lookup_e(e, f, cos_theta);
}
// dielectric_ms_params (open_pbr.rs:583-636) with the transmission lobe weights (638-646)
struct TransMs {
  float eta_rel, one_minus_e_avg_t, ratio_r, ss, ms, total;
  DevLerpAxis eta_axis, eta_rel_axis;
};
__device__ __forceinline__ TransMs trans_ms_at(const OpbrVertex& s, float eta) {
  TransMs t;
  const float eta_o = s.face == 0u ? fmaxf(eta, 1.0e-4f) : 1.0f / fmaxf(eta, 1.0e-4f);
  t.eta_rel = 1.0f / eta_o;
  const DevLerpAxis r = s.m->ms[0][s.face].r_axis;
  const float* e_avg = s.dec_e + kDecTableLen;
  t.eta_axis = axis_lerp(dec_eta_to_axis(eta_o), 32);
  t.eta_rel_axis = axis_lerp(dec_eta_to_axis(t.eta_rel), 32);
  const float e_avg_o = dec_e_avg_at(e_avg, r, t.eta_axis);
  const float e_avg_t = dec_e_avg_at(e_avg, r, t.eta_rel_axis);
  const float om_o = fmaxf(1.0f - e_avg_o, kMsEps);
  t.one_minus_e_avg_t = fmaxf(1.0f - e_avg_t, kMsEps);
  const float f_avg_o = f_avg_dielectric(eta_o), f_avg_t = f_avg_dielectric(t.eta_rel);
  const float a = (1.0f - f_avg_o) / om_o;
  const float b = (1.0f - f_avg_t) * eta_o * eta_o / t.one_minus_e_avg_t;
  const float x = a + b > kMsEps ? b / (a + b) : 0.5f;
  t.ratio_r = clampf(1.0f - x * (1.0f - f_avg_o), 0.0f, 1.0f);
  t.ss = clampf(e_avg_o, 0.0f, 1.0f);
  t.ms = fmaxf(1.0f - e_avg_o, 0.0f) * clampf(1.0f - t.ratio_r, 0.0f, 1.0f);
  t.total = fmaxf(t.ss + t.ms, 1.0e-8f);
  return t;
}
// base_dielectric_fresnel (open_pbr.rs:902-929) at physical / prime etas
__device__ __forceinline__ float dielectric_fresnel_eta(const DevOpenPbr& m, uint32_t face, float c, float eta_ph,
                                                        float eta_pr) {
  const bool front = face == 0u;
  const float unc = front ? weighted_fresnel_ratio(c, eta_ph, eta_pr)
                          : weighted_fresnel_ratio(c, 1.0f / eta_ph, 1.0f / eta_pr);
  if (m.coat_clamped <= 0.0f) return unc;
  const float eta_bc = eta_ph / fmaxf(m.coat_eta, 1.0e-4f);
  const float eta_bcp = eta_pr / fmaxf(m.coat_eta, 1.0e-4f);
  float a = eta_bc, b = eta_bcp;
  if (m.coat_eta > eta_ph) {
    a = 1.0f / fmaxf(eta_bc, 1.0e-4f);
    b = 1.0f / fmaxf(eta_bcp, 1.0e-4f);
  }
  const float coated = front ? weighted_fresnel_ratio(c, a, b)
                             : weighted_fresnel_ratio(c, 1.0f / fmaxf(a, 1.0e-4f), 1.0f / fmaxf(b, 1.0e-4f));
  return unc + (coated - unc) * m.coat_clamped;
}
// The rough BTDF at one wavelength's eta (eval_spec_btdf_scalar_with_eta,
// spec_btdf_fresnel_with_eta, eval_dielectric_transmission_ms,
// pdf_specular_btdf_with_eta; open_pbr.rs:672-696, 1074-1222): the single-
// scattering value (ss_ok false when it is None), the multiple-scattering
// value and the pdf.
struct BtdfEta {
  bool ss_ok;
  V3 ss;
  float ms, pdf;
};
__device__ __forceinline__ BtdfEta btdf_at_eta(const OpbrVertex& s, V3 wi, bool importance, float eta) {
  const DevOpenPbr& m = *s.m;
  const V3 wo = s.wo;
  BtdfEta r;
  r.ss_ok = false;
  r.ss = V3{0.0f, 0.0f, 0.0f};
  const float eta_rel = s.face == 0u ? 1.0f / eta : eta;
  const TransMs t = trans_ms_at(s, eta);
  float pdf_ss = 0.0f;
  const V3 wmu = eta_rel * wo + wi;
  if (!(length_sq(wmu) < 1.0e-12f)) {
    V3 wm = normalize(wmu);
    if (wm.z < 0.0f) wm = -wm;
    const float co = dot(wo, wm);
    const float ci = dot(wi, wm);
    const float den = ci + eta_rel * co;
    if (!(co <= 0.0f) && !(fabsf(den) < 1.0e-6f)) {
      const float d = ggx_d(wm, m.spec_ax, m.spec_ay);
      const float g = ggx_g2(wo, wi, m.spec_ax, m.spec_ay);
      if (!(d <= 0.0f || g <= 0.0f)) {
        const float scale = importance ? 1.0f : 1.0f / (eta_rel * eta_rel);
        const float sc = d * g * fabsf(ci * co);
        const float denom = den * den * fabsf(wo.z) * fabsf(wi.z);
        if (!(denom <= 0.0f)) {
          const float scalar = sc * scale / denom;
          const V3 no_film = splat(dielectric_fresnel_eta(m, s.face, co, eta, eta));
          const V3 fr = (m.flags & kOpbrFilm) ? filmed_dielectric(m, no_film, co, eta) : no_film;
          r.ss = vmaxv(V3{1.0f, 1.0f, 1.0f} - fr, V3{0.0f, 0.0f, 0.0f}) * scalar;
          r.ss_ok = true;
        }
      }
      const float pdf_wm = pdf_wm_vndf(wo, wm, m.spec_ax, m.spec_ay);
      pdf_ss = pdf_wm <= 0.0f ? 0.0f : pdf_wm * fabsf(ci) / (den * den);
    }
  }
  const float e_o = dec_e_at(s.dec_e, t.eta_axis, m.ms[0][s.face].r_axis, wo.z);
  const float e_i = dec_e_at(s.dec_e, t.eta_rel_axis, m.ms[0][s.face].r_axis, fabsf(wi.z));
  const float ms_scale = importance ? 1.0f : 1.0f / (t.eta_rel * t.eta_rel);
  r.ms = (1.0f - t.ratio_r) * (1.0f - e_o) * (1.0f - e_i) * ms_scale / (kPiF * t.one_minus_e_avg_t);
  r.pdf = (t.ss * pdf_ss + t.ms * cosine_pdf(-wi.z)) / t.total;
  return r;
}
// A dispersive rough BTDF seen from the front of an unlocked path integrates
// over the camera basis (camera_dispersion_active, open_pbr.rs:1250-1312)
__device__ __forceinline__ bool camera_dispersion(const OpbrVertex& s) {
  return (s.m->flags & kOpbrDisp) && s.face == 0u && (s.m->flags & kOpbrTransRough) && s.lock < 0.0f;
}
// eval_spec_btdf_camera_integrated and pdf_specular_btdf_camera_mixture
static __device__ __noinline__ void btdf_camera(const OpbrVertex& s, V3 wi, bool importance, V3& f, float& pdf) {
  const V3 scale = disp::norm_scale();
  float w[disp::kIntervals];
  const float total = disp::interval_weights(s.thr, scale, w);
  f = V3{0.0f, 0.0f, 0.0f};
  pdf = 0.0f;
  for (int i = 0; i < disp::kIntervals; ++i) {
    const float lambda = disp::interval_midpoint(i);
    const float eta = disp::cauchy_ior(lambda, s.m->trans_eta, s.m->disp_abbe);
    const BtdfEta b = btdf_at_eta(s, wi, importance, eta);
    f = f + disp::basis_at(lambda, scale) * (b.ss + splat(b.ms)) * disp::kLambdaStep;
    const float p_lambda = w[i] / (total * disp::kLambdaStep);
    pdf += p_lambda * b.pdf * disp::kLambdaStep;
  }
}

// The specular BTDF and its pdf for wi below the surface (eval_spec_btdf,
// eval_thin_wall_spec_btdf, pdf_specular_btdf, open_pbr.rs:1024-1222);
// `importance` selects the transport mode's eta^2 scaling.
__device__ __forceinline__ void btdf_eval_pdf(const OpbrVertex& s, V3 wi, bool importance, V3& f, float& pdf,
                                              V3& f_thin) {
  const DevOpenPbr& m = *s.m;
  const V3 wo = s.wo;
  f = V3{0.0f, 0.0f, 0.0f};
  pdf = 0.0f;
  f_thin = V3{0.0f, 0.0f, 0.0f};
  if (!(m.flags & kOpbrTransRough)) return;  // spec_btdf_is_smooth: neither term
  if (m.flags & kOpbrThinWalled) {
    const V3 wim = V3{wi.x, wi.y, -wi.z};
    V3 wm;
    if (!half_vector(wo, wim, wm)) return;
    const float d = ggx_d(wm, m.tw_ax, m.tw_ay);
    const float g = ggx_g2(wo, wim, m.tw_ax, m.tw_ay);
    if (!(d <= 0.0f || g <= 0.0f)) f_thin = s.tw_t * (d * g / (4.0f * wo.z * fabsf(wi.z)));
    const float pdf_wm = pdf_wm_bounded_vndf(wo, wm, m.tw_ax, m.tw_ay);
    const float denom = 4.0f * fabsf(dot(wo, wm));
    pdf = denom > 0.0f ? pdf_wm / denom : 0.0f;
    return;
  }
  if (m.flags & kOpbrDisp) {
    if (camera_dispersion(s)) {
      btdf_camera(s, wi, importance, f, pdf);
      return;
    }
    if (s.lock >= 0.0f) {  // the path's locked wavelength
      const BtdfEta b = btdf_at_eta(s, wi, importance, disp::cauchy_ior(s.lock, m.trans_eta, m.disp_abbe));
      if (b.ss_ok) f = b.ss + splat(b.ms);
      pdf = b.pdf;
      return;
    }
  }
  const float eta_rel = m.teta_rel[s.face];
  const DevMsFace& fm = m.ms[0][s.face];
  // the single-scattering half, shared by eval and pdf (their validity tests agree)
  float pdf_ss = 0.0f;
  const V3 wmu = eta_rel * wo + wi;
  if (!(length_sq(wmu) < 1.0e-12f)) {
    V3 wm = normalize(wmu);
    if (wm.z < 0.0f) wm = -wm;
    const float co = dot(wo, wm);
    const float ci = dot(wi, wm);
    const float den = ci + eta_rel * co;
    if (!(co <= 0.0f) && !(fabsf(den) < 1.0e-6f)) {
      const float d = ggx_d(wm, m.spec_ax, m.spec_ay);
      const float g = ggx_g2(wo, wi, m.spec_ax, m.spec_ay);
      if (!(d <= 0.0f || g <= 0.0f)) {
        const float scale = importance ? 1.0f : 1.0f / (eta_rel * eta_rel);
        const float sc = d * g * fabsf(ci * co);
        const float denom = den * den * fabsf(wo.z) * fabsf(wi.z);
        if (!(denom <= 0.0f)) {
          const float scalar = sc * scale / denom;
          const V3 no_film = splat(spec_fresnel(m, s.face, co));
          const V3 fr = (m.flags & kOpbrFilm) ? filmed_dielectric(m, no_film, co, m.trans_eta) : no_film;
          // eval_dielectric_transmission_ms (open_pbr.rs:672-696)
          const float e_o = s.dec_eo[0];
          DevMsFace ft = fm;
          ft.eta_axis = fm.eta_rel_axis;
          const float e_i = dec_lookup_e(s.dec_e, ft, fabsf(wi.z));
          const float ms_scale = importance ? 1.0f : 1.0f / (fm.eta_rel * fm.eta_rel);
          const float ms = (1.0f - fm.ratio_r) * (1.0f - e_o) * (1.0f - e_i) * ms_scale /
                           (kPiF * fm.one_minus_e_avg_t);
          f = vmaxv(V3{1.0f, 1.0f, 1.0f} - fr, V3{0.0f, 0.0f, 0.0f}) * scalar + splat(ms);
        }
      }
      const float pdf_wm = pdf_wm_vndf(wo, wm, m.spec_ax, m.spec_ay);
      pdf_ss = pdf_wm <= 0.0f ? 0.0f : pdf_wm * fabsf(ci) / (den * den);
    }
  }
  pdf = (fm.trans_ss * pdf_ss + fm.trans_ms * cosine_pdf(-wi.z)) / fm.trans_total;
}

// OpenPbrBsdf::eval and ::pdf for one direction pair.  `lay` is the state of
// the direction the layer weights are taken at: the vertex itself in radiance
// transport, wi in importance transport (open_pbr.rs:228-233).  want_pdf =
// false leaves pdf_out at 0 (callers that need f only).  `importance` is the
// transport mode (the BTDF's eta^2 scaling depends on it).
static __device__ __noinline__ void eval_pdf(const OpbrVertex& s, const OpbrVertex& lay, V3 wi, V3& f_out,
                                             float& pdf_out, bool want_pdf = true, bool importance = false) {
  const DevOpenPbr& m = *s.m;
  const V3 wo = s.wo;
  V3 total = V3{0.0f, 0.0f, 0.0f};
  float pdf = 0.0f;
  f_out = total;
  pdf_out = 0.0f;
  if (!(wo.z > 0.0f)) return;  // is_upper_hemisphere(wo)
  if (wi.z < 0.0f) {
    // below the surface only the specular BTDF is non-zero (the reflection
    // lobes, fuzz and EON test wi.z > 0; the diffuse BTDF has zero weight);
    // the coat tint of a direction below the coat is one
    if (!(m.flags & kOpbrTrans)) return;
    const Below b = weights_below(lay, V3{1.0f, 1.0f, 1.0f});
    V3 fb, f_thin;
    float pb;
    btdf_eval_pdf(s, wi, importance, fb, pb, f_thin);
    if (length_sq(b.btdf) > 0.0f && (m.flags & kOpbrTransRough))
      f_out = (m.flags & kOpbrThinWalled) ? b.btdf * f_thin : b.btdf * fb;
    if (want_pdf && s.q_total > 0.0f && s.q_btdf > 0.0f && (m.flags & kOpbrTransRough))
      pdf_out = (s.q_btdf / s.q_total) * pb;
    return;
  }
  if (wi.z <= 0.0f) return;  // grazing (or NaN): every lobe is zero
  V3 wm;
  const bool has_wm = half_vector(wo, wi, wm);
  // layer weights with this wi (the coat tint depends on it)
  const V3 tint = m.coat > 0.0f ? coat_tint(m, lay.wo, wi) : V3{1.0f, 1.0f, 1.0f};
  const Below b = weights_below(lay, tint);
  const float coat_w = m.coat * lay.below_fuzz_s;
  const float inv4 = 4.0f * wo.z * wi.z;
  // specular GGX terms shared by the metal and dielectric lobes
  const bool need_spec = (m.flags & (kOpbrMetalRough | kOpbrSpecRough)) != 0;
  float d_s = 0.0f, g_s = 0.0f, pdf_ss_s = 0.0f;
  if (need_spec && has_wm) {
    d_s = ggx_d(wm, m.spec_ax, m.spec_ay);
    g_s = ggx_g2(wo, wi, m.spec_ax, m.spec_ay);
    const float pdf_wm = pdf_wm_bounded_vndf(wo, wm, m.spec_ax, m.spec_ay);
    const float denom = 4.0f * fabsf(dot(wo, wm));
    pdf_ss_s = denom <= 0.0f ? 0.0f : pdf_wm / denom;
  }
  const float pdf_cos = cosine_pdf(wi.z);
  // coat (eval_coat / pdf_coat)
  if (m.flags & kOpbrCoatRough) {
    if (coat_w > 0.0f && has_wm) {
      const float d = ggx_d(wm, m.coat_ax, m.coat_ay);
      const float g = ggx_g2(wo, wi, m.coat_ax, m.coat_ay);
      if (!(d <= 0.0f || g <= 0.0f)) {
        const float fr = fresnel_dielectric(fabsf(dot(wo, wm)), 1.0f, m.coat_eta);
        const float ss = d * g * fr / inv4;
        total = total + coat_w * splat(ss + refl_ms(s, 1, wi.z));
      }
    }
  }
  // metal (eval_metal)
  if (length_sq(b.metal) > 0.0f && (m.flags & kOpbrMetalRough) && has_wm && !(d_s <= 0.0f || g_s <= 0.0f)) {
    const V3 fr = metal_fresnel(m, fabsf(dot(wo, wm)));
    const V3 ss = fr * (d_s * g_s / inv4);
    const float e_i = cec_lookup_e(s.cec_e, m.cond_r, wi.z);
    const V3 ms = ld3(m.cond_f_ms) * ((1.0f - s.cec_eo) * (1.0f - e_i) / (kPiF * m.cond_one_minus_e_avg));
    total = total + b.metal * (ss + ms);
  }
  // dielectric specular reflection (eval_spec_brdf)
  if (length_sq(b.spec) > 0.0f && (m.flags & kOpbrSpecRough) && has_wm && !(d_s <= 0.0f || g_s <= 0.0f)) {
    if (m.flags & kOpbrThinWalled) {
      total = total + b.spec * (s.tw_r * (d_s * g_s / inv4));
    } else {
      const V3 ss = spec_fresnel3(m, s.face, fabsf(dot(wo, wm))) * (d_s * g_s / inv4);
      total = total + b.spec * (ss + splat(refl_ms(s, 0, wi.z)));
    }
  }
  float fz_f = 0.0f, fz_pdf = 0.0f;
  if (m.fuzz > 0.0f) fuzz_eval_pdf(m.fuzz_roughness, wo, wi, fz_f, fz_pdf);
  const V3 fuzz_w = m.fuzz * ld3(m.fuzz_color);
  if (length_sq(fuzz_w) > 0.0f) total = total + fuzz_w * splat(fz_f);
  float eon_f = 0.0f;
  if (length_sq(b.diff) > 0.0f) {
    eon_f = f_eon_white(m.eon_r, wo, wi);
    total = total + b.diff * splat(eon_f);
  }
  f_out = total;
  // pdf (open_pbr.rs:262-296)
  if (!want_pdf || s.q_total <= 0.0f) return;
  if (s.q_coat > 0.0f && (m.flags & kOpbrCoatRough)) {
    const DevMsFace& f = m.ms[1][s.face];
    float p;
    if (!has_wm) {
      p = f.lobe_ms * pdf_cos / f.lobe_total;
    } else {
      const float pdf_wm = pdf_wm_bounded_vndf(wo, wm, m.coat_ax, m.coat_ay);
      const float denom = 4.0f * fabsf(dot(wo, wm));
      p = denom <= 0.0f ? f.lobe_ms * pdf_cos / f.lobe_total
                        : (f.lobe_ss * (pdf_wm / denom) + f.lobe_ms * pdf_cos) / f.lobe_total;
    }
    pdf += (s.q_coat / s.q_total) * p;
  }
  if (s.q_metal > 0.0f && (m.flags & kOpbrMetalRough))
    pdf += (s.q_metal / s.q_total) * ((m.cond_ss * pdf_ss_s + m.cond_ms * pdf_cos) / m.cond_total);
  if (s.q_spec > 0.0f && (m.flags & kOpbrSpecRough)) {
    const DevMsFace& f = m.ms[0][s.face];
    pdf += (s.q_spec / s.q_total) * ((m.flags & kOpbrThinWalled) ? pdf_ss_s
                                                                   : (f.lobe_ss * pdf_ss_s + f.lobe_ms * pdf_cos) /
                                                                         f.lobe_total);
  }
  if (s.q_fuzz > 0.0f) pdf += (s.q_fuzz / s.q_total) * fz_pdf;
  if (s.q_diff > 0.0f) pdf += (s.q_diff / s.q_total) * eon_pdf(m.eon_r, m.eon_r_pow01, wo, wi);
  pdf_out = pdf;
}

struct Sample {
  V3 weight, wi;
  float pdf;
  float pdf_rev;  // pdf(wi -> wo), computed when requested (0 for delta samples)
  uint32_t flags;
  float lock;     // the wavelength this sample locks the path to (< 0: none)
};

// finalize_rough_sample_with_wavelength (open_pbr.rs:1997-2027).  `importance`
// selects the transport mode of the evaluation; `want_rev` computes pdf_rev.
__device__ __forceinline__ bool finalize(const OpbrVertex& s, V3 wi, uint32_t flags, bool importance, bool want_rev,
                                         Sample& out) {
  V3 f;
  float pdf;
  OpbrVertex at_wi;  // the same BSDF seen from wi
  if (importance || want_rev) {
    init_vertex(at_wi, s.m, s.cec_e, s.dec_e, wi, s.face == 0u, s.dk_cos);
    at_wi.thr = s.thr;
    at_wi.lock = s.lock;
  }
  eval_pdf(s, importance ? at_wi : s, wi, f, pdf, true, importance);
  if (pdf <= 0.0f) return false;
  if (length_sq(f) == 0.0f) return false;
  const float c = fabsf(wi.z);
  if (c <= 0.0f) return false;
  out.weight = f * (c / pdf);
  out.wi = wi;
  out.pdf = pdf;
  out.flags = flags;
  out.pdf_rev = 0.0f;
  if (want_rev) {
    V3 f_rev;
    eval_pdf(at_wi, at_wi, s.wo, f_rev, out.pdf_rev);
  }
  return true;
}

// sample_spec_btdf_camera_channels (open_pbr.rs:1838-1928): three per-channel
// wavelengths (u_rgb = ux[1..3]), one picked by the clamped throughput (ux[0]),
// the direction sampled at its eta, weighted by the three-channel BTDF over
// the channel-mixture pdf; the path locks to the picked wavelength.
static __device__ __noinline__ bool sample_btdf_channels(const OpbrVertex& s, float p_lobe, float u0, float u1,
                                                         const float* ux, Sample& out, bool importance) {
  const DevOpenPbr& m = *s.m;
  const V3 wo = s.wo;
  const V3 t = vmaxv(s.thr, V3{0.0f, 0.0f, 0.0f});
  const V3 w = max_element(t) > 0.0f ? t : V3{1.0f, 1.0f, 1.0f};
  const float sum = fmaxf(w.x + w.y + w.z, 1.0e-8f);
  const float prob[3] = {w.x / sum, w.y / sum, w.z / sum};
  float lam[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) lam[c] = disp::sample_channel_wavelength(c, ux[1 + c]);
  // pick_dispersion_channel
  float u = clampf(ux[0], 0.0f, 1.0f);
  int pick = 2;
  for (int c = 0; c < 3; ++c) {
    if (u <= prob[c]) {
      pick = c;
      break;
    }
    u -= prob[c];
  }
  if (prob[pick] <= 0.0f) return false;
  const float eta_u = disp::cauchy_ior(lam[pick], m.trans_eta, m.disp_abbe);
  const float eta_rel = s.face == 0u ? 1.0f / eta_u : eta_u;
  const TransMs tm = trans_ms_at(s, eta_u);
  const float ss_p = tm.ss / tm.total;
  V3 wi;
  if (u0 >= ss_p) {
    const float uu = ss_p < 1.0f ? (u0 - ss_p) / (1.0f - ss_p) : 0.0f;
    const V3 up = sample_cosine_hemisphere(uu, u1);
    wi = V3{up.x, up.y, -up.z};
  } else {
    const float uu = ss_p > 0.0f ? u0 / ss_p : 0.0f;
    V3 wm;
    if (!sample_wm_vndf(wo, m.spec_ax, m.spec_ay, uu, u1, wm)) return false;
    if (dot(wo, wm) <= 0.0f) return false;
    if (!refract_about(wo, wm, eta_rel, wi)) return false;
    if (wi.z >= 0.0f) return false;
  }
  if (wi.z >= 0.0f) return false;
  const V3 bw = weights_below(s, V3{1.0f, 1.0f, 1.0f}).btdf;
  float pdf_mix = 0.0f;
  V3 f = V3{0.0f, 0.0f, 0.0f};
  for (int c = 0; c < 3; ++c) {
    if (prob[c] <= 0.0f) continue;
    const BtdfEta b = btdf_at_eta(s, wi, importance, disp::cauchy_ior(lam[c], m.trans_eta, m.disp_abbe));
    pdf_mix += prob[c] * b.pdf;
    // eval_spec_btdf_sampled_channels: channel c's component of (1 - F) * scalar, plus ms
    const float ss = c == 0 ? b.ss.x : (c == 1 ? b.ss.y : b.ss.z);
    const float v = ss + b.ms;
    f = f + V3{c == 0 ? v : 0.0f, c == 1 ? v : 0.0f, c == 2 ? v : 0.0f};
  }
  const float pdf_total = p_lobe * pdf_mix;
  if (pdf_total <= 0.0f) return false;
  out.weight = bw * f * (fabsf(wi.z) / pdf_total);
  out.wi = wi;
  out.pdf = pdf_total;
  out.pdf_rev = 0.0f;  // pdf(wi, wo) with wi below the surface
  out.flags = kFlagGlossy | kFlagTransmission;
  out.lock = lam[pick];
  return true;
}

// sample_spec_btdf (open_pbr.rs:1670-1836): thin-walled (smooth pass-through
// or the mirrored thin-wall GGX lobe), smooth refraction, or the rough BTDF
// (VNDF single scattering / cosine multiple scattering); a dispersive one at
// the path's locked wavelength, at a wavelength drawn with ux[0] (smooth, front
// face: the path locks to it), or over sampled camera channels (rough, front
// face, unlocked).
static __device__ __noinline__ bool sample_btdf(const OpbrVertex& s, float p_lobe, float u0, float u1, Sample& out,
                                                bool importance, bool want_rev, const float* ux) {
  const DevOpenPbr& m = *s.m;
  const V3 wo = s.wo;
  const V3 one = V3{1.0f, 1.0f, 1.0f};
  const bool rough = (m.flags & kOpbrTransRough) != 0;
  out.pdf_rev = 0.0f;
  if (m.flags & kOpbrThinWalled) {
    if (!rough) {
      const V3 wi = -wo;
      out.weight = (weights_below(s, one).btdf * s.tw_t) / p_lobe;
      out.wi = wi;
      out.pdf = p_lobe;
      out.flags = kFlagDelta | kFlagTransmission;
      return true;
    }
    V3 wm;
    if (!sample_wm_bounded_vndf(wo, m.tw_ax, m.tw_ay, u0, u1, wm)) return false;
    const V3 wr = reflect_local(wo, wm);
    if (wr.z <= 0.0f) return false;
    const V3 wi = V3{wr.x, wr.y, -wr.z};
    const V3 bw = weights_below(s, one).btdf;
    V3 fb, f_thin;
    float pb;
    btdf_eval_pdf(s, wi, importance, fb, pb, f_thin);
    const float pdf_total = p_lobe * pb;
    if (pdf_total <= 0.0f) return false;
    out.weight = bw * f_thin * fabsf(wi.z) / pdf_total;
    out.wi = wi;
    out.pdf = pdf_total;
    out.flags = kFlagGlossy | kFlagTransmission;
    return true;  // pdf_rev = pdf(wi, wo) = 0: wi is below the surface
  }
  if (m.flags & kOpbrDisp) {
    if (camera_dispersion(s)) return sample_btdf_channels(s, p_lobe, u0, u1, ux, out, importance);
    if (s.lock >= 0.0f || s.face == 0u) {
      V3 basis = one;
      float eta_u;
      if (s.lock >= 0.0f) {
        eta_u = disp::cauchy_ior(s.lock, m.trans_eta, m.disp_abbe);
      } else {  // smooth, front face, unlocked: a fresh wavelength
        out.lock = disp::sample_wavelength_weighted(ux[0], s.thr, basis);
        eta_u = disp::cauchy_ior(out.lock, m.trans_eta, m.disp_abbe);
      }
      const float eta_rel = s.face == 0u ? 1.0f / eta_u : eta_u;
      if (!rough) {
        V3 wi;
        if (!refract_z(wo, eta_rel, wi)) return false;
        const float fr = dielectric_fresnel_eta(m, s.face, fabsf(wo.z), eta_u, eta_u);
        const float scale = importance ? 1.0f : 1.0f / (eta_rel * eta_rel);
        out.weight = (weights_below(s, one).btdf * basis * (1.0f - fr) * scale) / p_lobe;
        out.wi = wi;
        out.pdf = p_lobe;
        out.flags = kFlagDelta | kFlagTransmission;
        return true;
      }
      // rough and locked: the locked eta's lobe weights, evaluated at the lock
      const TransMs tm = trans_ms_at(s, eta_u);
      const float ss_p = tm.ss / tm.total;
      V3 wi;
      if (u0 >= ss_p) {
        const float uu = ss_p < 1.0f ? (u0 - ss_p) / (1.0f - ss_p) : 0.0f;
        const V3 up = sample_cosine_hemisphere(uu, u1);
        wi = V3{up.x, up.y, -up.z};
      } else {
        const float uu = ss_p > 0.0f ? u0 / ss_p : 0.0f;
        V3 wm;
        if (!sample_wm_vndf(wo, m.spec_ax, m.spec_ay, uu, u1, wm)) return false;
        const float co = dot(wo, wm);
        if (co <= 0.0f) return false;
        if (!refract_about(wo, wm, eta_rel, wi)) return false;
        if (wi.z >= 0.0f) return false;
        const float ci = dot(wi, wm);
        const float den = ci + eta_rel * co;
        if (fabsf(den) < 1.0e-6f) return false;
      }
      return finalize(s, wi, kFlagGlossy | kFlagTransmission, importance, want_rev, out);
    }
  }
  const float eta_rel = m.teta_rel[s.face];
  if (!rough) {
    V3 wi;
    if (!refract_z(wo, eta_rel, wi)) return false;
    const float fr = spec_fresnel(m, s.face, fabsf(wo.z));
    const float scale = importance ? 1.0f : 1.0f / (eta_rel * eta_rel);
    out.weight = (weights_below(s, one).btdf * one * (1.0f - fr) * scale) / p_lobe;
    out.wi = wi;
    out.pdf = p_lobe;
    out.flags = kFlagDelta | kFlagTransmission;
    return true;
  }
  const DevMsFace& fm = m.ms[0][s.face];
  const float ss_p = fm.trans_ss / fm.trans_total;
  V3 wi;
  if (u0 >= ss_p) {
    const float uu = ss_p < 1.0f ? (u0 - ss_p) / (1.0f - ss_p) : 0.0f;
    const V3 up = sample_cosine_hemisphere(uu, u1);
    wi = V3{up.x, up.y, -up.z};
  } else {
    const float uu = ss_p > 0.0f ? u0 / ss_p : 0.0f;
    V3 wm;
    if (!sample_wm_vndf(wo, m.spec_ax, m.spec_ay, uu, u1, wm)) return false;
    const float co = dot(wo, wm);
    if (co <= 0.0f) return false;
    if (!refract_about(wo, wm, eta_rel, wi)) return false;
    if (wi.z >= 0.0f) return false;
    const float ci = dot(wi, wm);
    const float den = ci + eta_rel * co;
    if (fabsf(den) < 1.0e-6f) return false;
  }
  return finalize(s, wi, kFlagGlossy | kFlagTransmission, importance, want_rev, out);
}

// OpenPbrBsdf::sample (open_pbr.rs:298-332) in the shading frame.
static __device__ __noinline__ bool sample(const OpbrVertex& s, float u_lobe, float u0, float u1, Sample& out,
                                           bool importance = false, bool want_rev = false,
                                           const float* ux = nullptr) {
  const DevOpenPbr& m = *s.m;
  const V3 wo = s.wo;
  out.lock = -1.0f;
  if (!(wo.z > 0.0f) || s.q_total <= 0.0f) return false;
  // pick_lobe over (coat, metal, spec_brdf, spec_btdf, fuzz, diff_brdf, diff_btdf = 0)
  float u = u_lobe * s.q_total;
  int lobe;
  float pl;
  if (u < s.q_coat) {
    lobe = 0;
    pl = s.q_coat;
  } else if ((u -= s.q_coat) < s.q_metal) {
    lobe = 1;
    pl = s.q_metal;
  } else if ((u -= s.q_metal) < s.q_spec) {
    lobe = 2;
    pl = s.q_spec;
  } else if ((u -= s.q_spec) < s.q_btdf) {
    lobe = 5;
    pl = s.q_btdf;
  } else if ((u -= s.q_btdf) < s.q_fuzz) {
    lobe = 3;
    pl = s.q_fuzz;
  } else if ((u -= s.q_fuzz) < s.q_diff) {
    lobe = 4;
    pl = s.q_diff;
  } else {
    return false;  // diffuse transmission: probability zero
  }
  const float p_lobe = pl / s.q_total;
  if (p_lobe <= 0.0f) return false;
  if (lobe == 5) {
    const float zeros[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    return sample_btdf(s, p_lobe, u0, u1, out, importance, want_rev, ux ? ux : zeros);
  }
  if (lobe == 3 || lobe == 4) {
    V3 wi;
    const bool ok = lobe == 3 ? fuzz_sample_dir(m.fuzz_roughness, wo, u0, u1, wi)
                              : eon_sample_dir(m.eon_r, m.eon_r_pow01, wo, u0, u1, wi);
    if (!ok) return false;
    return finalize(s, wi, lobe == 3 ? (kFlagGlossy | kFlagReflection) : (kFlagDiffuse | kFlagReflection),
                    importance, want_rev, out);
  }
  const bool rough = lobe == 0 ? (m.flags & kOpbrCoatRough) != 0
                               : (lobe == 1 ? (m.flags & kOpbrMetalRough) != 0 : (m.flags & kOpbrSpecRough) != 0);
  if (!rough) {
    // smooth lobe: mirror direction, delta sample
    const V3 wi = V3{-wo.x, -wo.y, wo.z};
    const V3 tint = m.coat > 0.0f ? coat_tint(m, wo, wi) : V3{1.0f, 1.0f, 1.0f};
    out.pdf_rev = 0.0f;
    if (lobe == 0) {
      const float fr = fresnel_dielectric(fabsf(wi.z), 1.0f, m.coat_eta);
      out.weight = splat(m.coat * s.below_fuzz_s * fr / p_lobe);
    } else {
      const Below b = weights_below(s, tint);
      // a thin-walled sheet reflects its slab reflectance (open_pbr.rs:1596-1602)
      const V3 fs = (m.flags & kOpbrThinWalled) ? s.tw_r : spec_fresnel3(m, s.face, fabsf(wi.z));
      out.weight = lobe == 1 ? (b.metal * metal_fresnel(m, fabsf(wi.z))) / p_lobe : (b.spec * fs) / p_lobe;
    }
    out.wi = wi;
    out.pdf = p_lobe;
    out.flags = kFlagDelta | kFlagReflection;
    return true;
  }
  // rough thin-walled specular: GGX single scattering only (open_pbr.rs:1615-1628)
  if (lobe == 2 && (m.flags & kOpbrThinWalled)) {
    V3 wm;
    if (!sample_wm_bounded_vndf(wo, m.spec_ax, m.spec_ay, u0, u1, wm)) return false;
    const V3 wi = reflect_local(wo, wm);
    if (wi.z <= 0.0f) return false;
    return finalize(s, wi, kFlagGlossy | kFlagReflection, importance, want_rev, out);
  }
  // rough: GGX single scattering or cosine multiple scattering
  float ss, tot, ax, ay;
  if (lobe == 1) {
    ss = m.cond_ss;
    tot = m.cond_total;
    ax = m.spec_ax;
    ay = m.spec_ay;
  } else {
    const DevMsFace& f = m.ms[lobe == 0 ? 1 : 0][s.face];
    ss = f.lobe_ss;
    tot = f.lobe_total;
    ax = lobe == 0 ? m.coat_ax : m.spec_ax;
    ay = lobe == 0 ? m.coat_ay : m.spec_ay;
  }
  const float ss_p = ss / tot;
  V3 wi;
  if (u0 >= ss_p) {
    const float uu = ss_p < 1.0f ? (u0 - ss_p) / (1.0f - ss_p) : 0.0f;
    wi = sample_cosine_hemisphere(uu, u1);
  } else {
    const float uu = ss_p > 0.0f ? u0 / ss_p : 0.0f;
    V3 wm;
    if (!sample_wm_bounded_vndf(wo, ax, ay, uu, u1, wm)) return false;
    wi = reflect_local(wo, wm);
    if (wi.z <= 0.0f) return false;
  }
  return finalize(s, wi, kFlagGlossy | kFlagReflection, importance, want_rev, out);
}

}  // namespace opbr
}  // namespace tpt
