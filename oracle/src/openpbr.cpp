// Oracle: OpenPBR BSDF and its lobes (bsdf/open_pbr.rs, bsdf/eon.rs) and the
// untextured material lowering (material/open_pbr.rs).
#include "openpbr.h"
#include "dispersion.h"

#include <cstring>

#include "render.h"

namespace orc {

namespace {
constexpr float kCos82 = 1.0f / 7.0f;
constexpr float kMsDenomEps = 1.0e-6f;
constexpr float kRcpPi = 1.0f / kPi;

float luminance(Vec3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
Vec3 vclamp01(Vec3 v) { return vmin(vmax(v, Vec3(0, 0, 0)), Vec3(1, 1, 1)); }
float lerp(float a, float b, float t) { return a + (b - a) * t; }
Vec3 lerp3(Vec3 a, Vec3 b, float t) { return a + (b - a) * t; }
Vec3 vpowf(Vec3 v, float e) {
  return Vec3(std::pow(fmax_num(v.x, 0.0f), e), std::pow(fmax_num(v.y, 0.0f), e), std::pow(fmax_num(v.z, 0.0f), e));
}
float cosine_pdf(float c) { return fmax_num(c, 0.0f) / kPi; }

// ---- bsdf/eon.rs -------------------------------------------------------------
constexpr float kC1Fon = 0.5f - 2.0f / (3.0f * kPi);
constexpr float kC2Fon = 2.0f / 3.0f - 28.0f / (15.0f * kPi);
constexpr float kEonEps = 1.0e-7f;

float e_fon_approx(float mu, float r) {
  float mc = 1.0f - mu;
  float g_over_pi = mc * (0.05710853f + mc * (0.49188188f + mc * (-0.33218145f + mc * 0.071443f)));
  return (1.0f + r * g_over_pi) / (1.0f + kC1Fon * r);
}
Vec3 f_eon(Vec3 rho, float r, Vec3 wo, Vec3 wi) {
  float mu_o = wo.z, mu_i = wi.z;
  float s = dot(wo, wi) - mu_i * mu_o;
  float s_over_t = s > 0.0f ? s / fmax_num(mu_o, mu_i) : s;
  float af = 1.0f / (1.0f + kC1Fon * r);
  Vec3 f_ss = rho * (kRcpPi * af * (1.0f + r * s_over_t));
  float e_fo = e_fon_approx(mu_o, r), e_fi = e_fon_approx(mu_i, r);
  float avg_ef = af * (1.0f + kC2Fon * r);
  float one_minus_avg = 1.0f - avg_ef;
  Vec3 denom = Vec3(1, 1, 1) - rho * one_minus_avg;
  Vec3 rho_ms = rho * rho * avg_ef / denom;
  float scale = kRcpPi * fmax_num(1.0f - e_fo, kEonEps) * fmax_num(1.0f - e_fi, kEonEps) / fmax_num(one_minus_avg, kEonEps);
  return f_ss + rho_ms * scale;
}
void ltc_coeffs(float mu, float r, float* a, float* b, float* c, float* d) {
  *a = 1.0f + r * (0.303392f + (-0.518982f + 0.111709f * mu) * mu + (-0.276266f + 0.335918f * mu) * r);
  *b = r * (-1.16407f + 1.15859f * mu + (0.150815f - 0.150105f * mu) * r) / (mu * mu * mu - 1.43545f);
  *c = 1.0f + r * (0.20013f + (-0.506373f + 0.261777f * mu) * mu);
  *d = r * (0.540852f + (-1.01625f + 0.475392f * mu) * mu) / (-1.0743f + (0.0725628f + mu) * mu);
}
Vec2 ltc_basis_x(Vec3 wo) {
  float len_sqr = wo.x * wo.x + wo.y * wo.y;
  if (len_sqr > 0.0f) {
    float inv = 1.0f / std::sqrt(len_sqr);
    return Vec2(wo.x * inv, wo.y * inv);
  }
  return Vec2(1.0f, 0.0f);
}
Vec3 ltc_apply_from(Vec3 wo, Vec3 v) {
  Vec2 x = ltc_basis_x(wo);
  Vec2 y(-x.y, x.x);
  return Vec3(x.x * v.x + y.x * v.y, x.y * v.x + y.y * v.y, v.z);
}
Vec3 ltc_apply_to(Vec3 wo, Vec3 v) {
  Vec2 x = ltc_basis_x(wo);
  Vec2 y(-x.y, x.x);
  return Vec3(x.x * v.x + x.y * v.y, y.x * v.x + y.y * v.y, v.z);
}
Vec3 cltc_sample(Vec3 wo, float r, float u1, float u2, float* pdf) {
  float a, b, c, d;
  ltc_coeffs(wo.z, r, &a, &b, &c, &d);
  float radius = std::sqrt(u1);
  float phi = 2.0f * kPi * u2;
  float x0 = radius * std::cos(phi), y0 = radius * std::sin(phi);
  float vz = 1.0f / std::sqrt(d * d + 1.0f);
  float s = 0.5f * (1.0f + vz);
  float edge = std::sqrt(fmax_num(1.0f - y0 * y0, 0.0f));
  float x = -((1.0f - s) * edge + s * x0);
  float y = y0;
  float wh_z = std::sqrt(fmax_num(1.0f - (x * x + y * y), 0.0f));
  Vec3 wh(x, y, wh_z);
  float pdf_wh = wh.z / (kPi * s);
  Vec3 wi_ltc(a * wh.x + b * wh.z, c * wh.y, d * wh.x + wh.z);
  float len = length(wi_ltc);
  float det_m = c * (a - b * d);
  *pdf = pdf_wh * (len * len * len) / det_m;
  return ltc_apply_from(wo, wi_ltc / len);
}
float cltc_pdf(Vec3 wo, Vec3 wi_local, float r) {
  Vec3 w = ltc_apply_to(wo, wi_local);
  float a, b, c, d;
  ltc_coeffs(wo.z, r, &a, &b, &c, &d);
  float det_m = c * (a - b * d);
  Vec3 wh(c * (w.x - b * w.z), (a - b * d) * w.y, -c * (d * w.x - a * w.z));
  float lensq = fmax_num(dot(wh, wh), 1.0e-30f);
  float vz = 1.0f / std::sqrt(d * d + 1.0f);
  float s = 0.5f * (1.0f + vz);
  float q = det_m / lensq;
  return q * q * fmax_num(wh.z, 0.0f) / (kPi * s);
}
float p_uniform(float mu, float r) {
  return std::pow(r, 0.1f) * (0.162925f + (-0.372058f + (0.538233f - 0.290822f * mu) * mu) * mu);
}
Vec3 sample_eon(Vec3 wo, float r, float u1, float u2, float* pdf) {
  float mu = wo.z;
  float p_u = p_uniform(mu, r);
  float p_c = 1.0f - p_u;
  Vec3 wi;
  float pdf_c;
  if (u1 < p_u) {
    float u1n = u1 / p_u;
    float st = std::sqrt(fmax_num(1.0f - u1n * u1n, 0.0f));
    float phi = 2.0f * kPi * u2;
    wi = Vec3(st * std::cos(phi), st * std::sin(phi), u1n);
    pdf_c = cltc_pdf(wo, wi, r);
  } else {
    float denom = fmax_num(p_c, 1.0e-30f);
    float u1n = (u1 - p_u) / denom;
    wi = cltc_sample(wo, r, u1n, u2, &pdf_c);
  }
  float pdf_u = 1.0f / (2.0f * kPi);
  *pdf = p_u * pdf_u + p_c * pdf_c;
  return wi;
}
float pdf_eon(Vec3 wo, Vec3 wi, float r) {
  float p_u = p_uniform(wo.z, r);
  float p_c = 1.0f - p_u;
  float pdf_c = cltc_pdf(wo, wi, r);
  return p_u * (1.0f / (2.0f * kPi)) + p_c * pdf_c;
}
// EonBsdf (eon.rs:18-58) with rho = ONE
struct Eon {
  float r;
  explicit Eon(float roughness) : r(clampf(roughness, 0.0f, 1.0f)) {}
  Vec3 eval(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return Vec3(0, 0, 0);
    return f_eon(Vec3(1, 1, 1), r, wo, wi);
  }
  float pdf(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
    return pdf_eon(wo, wi, r);
  }
  bool sample(Vec3 wo, Vec2 us, Vec3* wi) const {
    if (wo.z <= 0.0f) return false;
    float pdf;
    Vec3 w = sample_eon(wo, r, us.x, us.y, &pdf);
    if (pdf <= 0.0f || w.z <= 0.0f) return false;
    *wi = w;
    return true;
  }
};

// ---- fuzz (bsdf/open_pbr.rs:148-205, 2052-2123) ------------------------------
float zeltner_dir_albedo(float ndot_v, float roughness) {
  float x = clampf(ndot_v, 0.0f, 1.0f);
  float y = clampf(roughness, 0.01f, 1.0f);
  float s = y * (0.0206607f + 1.58491f * y) / (0.0379424f + y * (1.32227f + y));
  float m = y * (-0.193854f + y * (-1.14885f + y * (1.7932f - 0.95943f * y * y))) / (0.046391f + y);
  float o = y * (0.000654023f + (-0.0207818f + 0.119681f * y) * y) / (1.26264f + y * (-1.92021f + y));
  float q = (x - m) / s;
  return std::exp(-0.5f * (q * q)) / (s * std::sqrt(2.0f * kPi)) + o;
}
float zeltner_a_inv(float ndot_v, float roughness) {
  float x = clampf(ndot_v, 0.0f, 1.0f), y = clampf(roughness, 0.01f, 1.0f);
  return (2.58126f * x + 0.813703f * y) * y / (1.0f + 0.310327f * x * x + 2.60994f * x * y);
}
float zeltner_b_inv(float ndot_v, float roughness) {
  float x = clampf(ndot_v, 0.0f, 1.0f), y = clampf(roughness, 0.01f, 1.0f);
  return std::sqrt(1.0f - x) * (y - 1.0f) * y * y * y /
         (0.0000254053f + 1.71228f * x - 1.71506f * x * y + 1.34174f * y * y);
}
float eval_ltc(Vec3 wi, float a_inv, float b_inv) {
  Vec3 w(a_inv * wi.x + b_inv * wi.z, a_inv * wi.y, wi.z);
  float len = length(w);
  if (len <= 0.0f) return 0.0f;
  w /= len;
  if (w.z <= 0.0f) return 0.0f;
  float det = a_inv * a_inv;
  float jac = det / (len * len * len);
  return (w.z / kPi) * jac;
}
Vec3 sample_ltc(float a_inv, float b_inv, Vec2 u) {
  float phi = 2.0f * kPi * u.x;
  float ct = std::sqrt(u.y), st = std::sqrt(fmax_num(1.0f - u.y, 0.0f));
  Vec3 w(std::cos(phi) * st, std::sin(phi) * st, ct);
  Vec3 wi(w.x / a_inv - w.z * b_inv / a_inv, w.y / a_inv, w.z);
  return normalize_or_zero(wi);
}
float phi_of(Vec3 v) {
  float p = std::atan2(v.y, v.x);
  return p < 0.0f ? p + 2.0f * kPi : p;
}
Vec3 rotate_z(Vec3 v, float angle) {
  float s = std::sin(angle), c = std::cos(angle);
  return Vec3(c * v.x - s * v.y, s * v.x + c * v.y, v.z);
}
struct Fuzz {
  float r;
  explicit Fuzz(float roughness) : r(clampf(roughness, 0.01f, 1.0f)) {}
  Vec3 eval(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return Vec3(0, 0, 0);
    Vec3 w = rotate_z(wi, -phi_of(wo));
    float a = zeltner_a_inv(wo.z, r), b = zeltner_b_inv(wo.z, r);
    float alb = zeltner_dir_albedo(wo.z, r);
    float v = eval_ltc(w, a, b);
    float cos_i = fmax_num(wi.z, 1.0e-6f);
    return Vec3::splat(alb * v / cos_i);
  }
  float pdf(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
    Vec3 w = rotate_z(wi, -phi_of(wo));
    return eval_ltc(w, zeltner_a_inv(wo.z, r), zeltner_b_inv(wo.z, r));
  }
  bool sample(Vec3 wo, Vec2 us, Vec3* wi) const {
    if (wo.z <= 0.0f) return false;
    Vec3 w = sample_ltc(zeltner_a_inv(wo.z, r), zeltner_b_inv(wo.z, r), us);
    if (w.z <= 0.0f) return false;
    Vec3 v = rotate_z(w, phi_of(wo));
    if (v.z <= 0.0f) return false;
    *wi = v;
    return true;
  }
  float albedo(Vec3 wo) const { return zeltner_dir_albedo(clampf(wo.z, 0.0f, 1.0f), r); }
};

// ---- open_pbr.rs helpers -------------------------------------------------------
float f_avg_dielectric(float eta) {
  if (eta >= 1.0f) return clampf((eta - 1.0f) / (4.08567f + 1.00071f * eta), 0.0f, 1.0f);
  float e = fmax_num(eta, kMsDenomEps);
  float v = 0.997118f + 0.1014f * e - 0.965241f * e * e - 0.130607f * e * e * e;
  return clampf(v, 0.0f, 1.0f);
}
Vec3 conductor_f_ms(Vec3 f_avg, float e_avg) {
  float om = fmax_num(1.0f - e_avg, 0.0f);
  Vec3 denom = Vec3(1, 1, 1) - f_avg * om;
  Vec3 ds(fmax_num(denom.x, kMsDenomEps), fmax_num(denom.y, kMsDenomEps), fmax_num(denom.z, kMsDenomEps));
  return f_avg * f_avg * e_avg / ds;
}
Vec3 schlick3(Vec3 f0, float c) {
  float om = 1.0f - clampf(c, 0.0f, 1.0f);
  return f0 + (Vec3(1, 1, 1) - f0) * powi(om, 5);
}
// Constant-argument powi is folded at compile time through the host pow in
// double precision: (1 - 1/7)^5 and (1 - 1/7)^6 of the F82 terms.
float cos82_pow(int n) { return (float)std::pow((double)(1.0f - kCos82), (double)n); }
Vec3 schlick3_82(Vec3 f0) { return f0 + (Vec3(1, 1, 1) - f0) * cos82_pow(5); }
float weighted_fresnel_ratio(float c, float eta_ti, float eta_tp) {
  eta_ti = fmax_num(eta_ti, 1.0e-4f);
  eta_tp = fmax_num(eta_tp, 1.0e-4f);
  if (eta_tp >= 1.0f) return fresnel_dielectric(c, 1.0f, eta_tp);
  float cc = clampf(c, 0.0f, 1.0f);
  float mu2_t = 1.0f - (1.0f - cc * cc) / (eta_ti * eta_ti);
  if (mu2_t <= 0.0f) return 1.0f;
  return fresnel_dielectric(std::sqrt(mu2_t), 1.0f, 1.0f / eta_tp);
}
float refracted_cos(float mu, float eta) {
  float m = clampf(mu, 0.0f, 1.0f);
  float sin2_t = fmax_num(1.0f - m * m, 0.0f) / fmax_num(eta * eta, kMsDenomEps);
  return std::sqrt(fmax_num(1.0f - sin2_t, 0.0f));
}
float cos82_denom() { return kCos82 * cos82_pow(6); }

struct LayerWeights {
  float coat_amp;
  Vec3 metal, spec_brdf, spec_btdf, fuzz, diff_brdf, diff_btdf;
};
struct LobeProbs {
  float coat, metal, spec_brdf, spec_btdf, fuzz, diff_brdf, diff_btdf, total;
};
struct MsParams {
  float eta_o, eta_rel, roughness_eq, e_avg_o, ratio_r, one_minus_e_avg_o, one_minus_e_avg_t;
};
struct TwoLobe {
  float ss, ms, total;
};
enum Lobe { kCoat, kMetal, kSpecBrdf, kSpecBtdf, kFuzzLobe, kDiffBrdf, kDiffBtdf };

struct Impl {
  const OpenPbrParams& p;
  const OpenPbrLuts& L;

  bool coat_smooth() const { return p.coat <= 0.0f || fmax_num(p.coat_alpha_x, p.coat_alpha_y) < kSmoothAlpha; }
  bool metal_smooth() const {
    return p.metalness <= 0.0f || fmax_num(p.specular_alpha_x, p.specular_alpha_y) < kSmoothAlpha;
  }
  bool spec_smooth() const {
    return p.specular <= 0.0f || fmax_num(p.specular_alpha_x, p.specular_alpha_y) < kSmoothAlpha;
  }
  float coat_proxy() const { return clampf(std::sqrt(fmax_num(p.coat_alpha_x, p.coat_alpha_y)), 0.0f, 1.0f); }
  float spec_proxy() const { return clampf(std::sqrt(fmax_num(p.specular_alpha_x, p.specular_alpha_y)), 0.0f, 1.0f); }
  float conductor_req() const { return std::pow(p.specular_alpha_x * p.specular_alpha_y, 0.25f); }
  bool btdf_smooth() const {
    return p.transmission <= 0.0f || fmax_num(p.transmission_alpha_x, p.transmission_alpha_y) < kSmoothAlpha;
  }
  // TransportMode::transmission_scale (bsdf/mod.rs:102-107)
  static float trans_scale(TransportMode mode, float eta_rel) {
    return mode == kRadiance ? 1.0f / (eta_rel * eta_rel) : 1.0f;
  }
  // thin_wall_transmission_alpha_xy (open_pbr.rs:553-564)
  void thin_wall_alpha(float* ax, float* ay) const {
    float eta = fmax_num(p.transmission_eta, 1.0f);
    float scale = std::sqrt(fmax_num(3.7f * (eta - 1.0f) * powi(eta - 0.5f, 2) / powi(eta, 3), 0.0f));
    float s2 = scale * scale;
    *ax = clampf(p.transmission_alpha_x * s2, kMinAlpha, 1.0f);
    *ay = clampf(p.transmission_alpha_y * s2, kMinAlpha, 1.0f);
  }

  MsParams ms_params(float ax, float ay, float eta) const {
    MsParams m;
    m.eta_o = p.front_face ? fmax_num(eta, 1.0e-4f) : 1.0f / fmax_num(eta, 1.0e-4f);
    m.eta_rel = 1.0f / m.eta_o;
    m.roughness_eq = std::pow(ax * ay, 0.25f);
    m.e_avg_o = L.dielectric->lookup_e_avg(m.roughness_eq, m.eta_o);
    float e_avg_t = L.dielectric->lookup_e_avg(m.roughness_eq, m.eta_rel);
    m.one_minus_e_avg_o = fmax_num(1.0f - m.e_avg_o, kMsDenomEps);
    m.one_minus_e_avg_t = fmax_num(1.0f - e_avg_t, kMsDenomEps);
    float f_avg_o = f_avg_dielectric(m.eta_o), f_avg_t = f_avg_dielectric(m.eta_rel);
    float a = (1.0f - f_avg_o) / m.one_minus_e_avg_o;
    float b = (1.0f - f_avg_t) * m.eta_o * m.eta_o / m.one_minus_e_avg_t;
    float x = a + b > kMsDenomEps ? b / (a + b) : 0.5f;
    m.ratio_r = clampf(1.0f - x * (1.0f - f_avg_o), 0.0f, 1.0f);
    return m;
  }
  float ms_factor(const MsParams& m) const {
    float f_avg = clampf(f_avg_dielectric(m.eta_o), 0.0f, 1.0f);
    float denom = 1.0f - f_avg * fmax_num(1.0f - m.e_avg_o, 0.0f);
    return clampf(f_avg * f_avg * m.e_avg_o / fmax_num(denom, kMsDenomEps), 0.0f, 1.0f);
  }
  TwoLobe reflection_lobe_weights(const MsParams& m) const {
    float f_avg = clampf(f_avg_dielectric(m.eta_o), 0.0f, 1.0f);
    float ss = clampf(f_avg * m.e_avg_o, 0.0f, 1.0f);
    float ms = fmax_num(1.0f - m.e_avg_o, 0.0f) * ms_factor(m);
    return {ss, ms, fmax_num(ss + ms, 1.0e-8f)};
  }
  TwoLobe transmission_lobe_weights(const MsParams& m) const {  // open_pbr.rs:638-646
    float ss = clampf(m.e_avg_o, 0.0f, 1.0f);
    float ms = fmax_num(1.0f - m.e_avg_o, 0.0f) * clampf(1.0f - m.ratio_r, 0.0f, 1.0f);
    return {ss, ms, fmax_num(ss + ms, 1.0e-8f)};
  }
  TwoLobe conductor_lobe_weights() const {
    float e_avg = clampf(L.conductor->lookup_e_avg(conductor_req()), 0.0f, 1.0f);
    float ms = fmax_num(1.0f - e_avg, 0.0f);
    return {e_avg, ms, fmax_num(e_avg + ms, 1.0e-8f)};
  }
  float albedo_with_ms(Vec3 wo, float ax, float ay, float eta, float ss) const {
    if (wo.z <= 0.0f || fmax_num(ax, ay) < kSmoothAlpha) return clampf(ss, 0.0f, 1.0f);
    MsParams m = ms_params(ax, ay, eta);
    float e_o = L.dielectric->lookup_e(wo.z, m.roughness_eq, m.eta_o);
    return clampf(ss + ms_factor(m) * fmax_num(1.0f - e_o, 0.0f), 0.0f, 1.0f);
  }
  float coat_albedo(Vec3 wo) const {
    if (wo.z <= 0.0f) return 0.0f;
    float ss = L.coat->lookup(wo, coat_proxy(), 0.0f);
    return albedo_with_ms(wo, p.coat_alpha_x, p.coat_alpha_y, p.coat_eta, ss);
  }
  float spec_albedo(Vec3 wo) const {
    if (wo.z <= 0.0f) return 0.0f;
    float ss = L.spec->lookup(wo, spec_proxy(), 0.0f);
    if (p.thin_walled) return ss;
    return albedo_with_ms(wo, p.specular_alpha_x, p.specular_alpha_y, p.specular_eta, ss);
  }
  float fuzz_albedo(Vec3 wo) const {
    if (p.fuzz <= 0.0f) return 0.0f;
    return Fuzz(p.fuzz_roughness).albedo(wo);
  }
  Vec3 coat_absorb_tint(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return Vec3(1, 1, 1);
    float mu_o = refracted_cos(wo.z, p.coat_eta), mu_i = refracted_cos(wi.z, p.coat_eta);
    float e = 0.5f * (1.0f / fmax_num(mu_i, 1.0e-4f) + 1.0f / fmax_num(mu_o, 1.0e-4f));
    return vpowf(p.coat_color, e);
  }

  // open_pbr.rs:334-406
  LayerWeights layer_weights(Vec3 wo, const Vec3* wi) const {
    const Vec3 one(1, 1, 1);
    float e_fuzz = fuzz_albedo(wo);
    Vec3 fuzz_w = p.fuzz * p.fuzz_color;
    float below_fuzz_s = fmax_num(1.0f - p.fuzz * e_fuzz, 0.0f);
    Vec3 below_fuzz = Vec3::splat(below_fuzz_s);
    float coat_amp = p.coat;
    float e_coat = coat_amp > 0.0f ? coat_albedo(wo) : 0.0f;
    Vec3 under_coat = below_fuzz;
    if (coat_amp > 0.0f) {
      Vec3 tint = wi ? coat_absorb_tint(wo, *wi) : p.coat_color;
      Vec3 thr = p.coat_darkening * tint * Vec3::splat(fmax_num(1.0f - e_coat, 0.0f));
      under_coat = below_fuzz * (one * (1.0f - coat_amp) + thr * coat_amp);
    }
    Vec3 metal = p.metalness * under_coat;
    Vec3 below_metal = (1.0f - p.metalness) * under_coat;
    float e_spec = spec_albedo(wo);
    Vec3 spec_amp = p.specular_color;
    Vec3 spec_brdf_w = below_metal * spec_amp;
    Vec3 leakage = vmax(one - spec_amp * e_spec, Vec3(0, 0, 0));
    Vec3 below_spec = below_metal * leakage;
    float trans = p.transmission;
    Vec3 tint = p.thin_walled ? Vec3(1, 1, 1) : p.transmission_color;
    Vec3 spec_btdf_w = below_spec * trans * tint;
    Vec3 below_trans = below_spec * (1.0f - trans);
    float thin_factor = p.thin_walled ? 1.0f : 0.0f;
    Vec3 diff_brdf_w = below_trans * ((1.0f - p.subsurface) * p.base) * p.base_color;
    Vec3 diff_btdf_w = below_trans * (p.subsurface * thin_factor) * p.subsurface_color;
    return {coat_amp * below_fuzz_s, metal, spec_brdf_w, spec_btdf_w, fuzz_w, diff_brdf_w, diff_btdf_w};
  }

  // open_pbr.rs:408-437
  LobeProbs lobe_probabilities(Vec3 wo) const {
    LayerWeights w = layer_weights(wo, nullptr);
    LobeProbs q;
    q.coat = p.coat > 0.0f ? w.coat_amp : 0.0f;
    q.metal = luminance(w.metal * (Vec3::splat(0.5f) + 0.5f * p.base_color));
    q.spec_brdf = luminance(w.spec_brdf);
    q.spec_btdf = p.transmission > 0.0f ? fmax_num(luminance(w.spec_btdf), 0.0f) : 0.0f;
    q.fuzz = fmax_num(luminance(w.fuzz), 0.0f);
    q.diff_brdf = fmax_num(luminance(w.diff_brdf), 0.0f);
    q.diff_btdf = fmax_num(luminance(w.diff_btdf), 0.0f);
    q.total = q.coat + q.metal + q.spec_brdf + q.spec_btdf + q.fuzz + q.diff_brdf + q.diff_btdf;
    return q;
  }

  float eval_refl_ms(Vec3 wo, Vec3 wi, float ax, float ay, float eta) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
    MsParams m = ms_params(ax, ay, eta);
    float e_o = L.dielectric->lookup_e(wo.z, m.roughness_eq, m.eta_o);
    float e_i = L.dielectric->lookup_e(wi.z, m.roughness_eq, m.eta_o);
    return ms_factor(m) * (1.0f - e_o) * (1.0f - e_i) / (kPi * m.one_minus_e_avg_o);
  }
  Vec3 eval_coat(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return Vec3(0, 0, 0);
    Vec3 wm;
    if (!reflection_half_vector(wo, wi, &wm)) return Vec3(0, 0, 0);
    float d = ggx_d(wm, p.coat_alpha_x, p.coat_alpha_y);
    float g = ggx_g2(wo, wi, p.coat_alpha_x, p.coat_alpha_y);
    if (d <= 0.0f || g <= 0.0f) return Vec3(0, 0, 0);
    float f = fresnel_dielectric(std::fabs(dot(wo, wm)), 1.0f, p.coat_eta);
    float ss = d * g * f / (4.0f * wo.z * wi.z);
    float ms = eval_refl_ms(wo, wi, p.coat_alpha_x, p.coat_alpha_y, p.coat_eta);
    return Vec3::splat(ss + ms);
  }
  float pdf_coat(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
    MsParams m = ms_params(p.coat_alpha_x, p.coat_alpha_y, p.coat_eta);
    TwoLobe w = reflection_lobe_weights(m);
    float pdf_ms = cosine_pdf(wi.z);
    Vec3 wm;
    if (!reflection_half_vector(wo, wi, &wm)) return w.ms * pdf_ms / w.total;
    float pdf_wm = pdf_wm_bounded_vndf(wo, wm, p.coat_alpha_x, p.coat_alpha_y);
    float denom = 4.0f * std::fabs(dot(wo, wm));
    if (denom <= 0.0f) return w.ms * pdf_ms / w.total;
    return (w.ss * (pdf_wm / denom) + w.ms * pdf_ms) / w.total;
  }
  bool film() const { return p.thin_film_weight > 0.0f && p.thin_film_thickness > 0.0f; }
  // metal_fresnel (open_pbr.rs:761-790): F82 tint, blended with the filmed
  // conductor reflectance (over the coat's eta where there is a coat)
  Vec3 metal_fresnel(float c) const {
    Vec3 no_film = metal_f82(c);
    float w = clampf(p.thin_film_weight, 0.0f, 1.0f);
    if (!(w > 0.0f && p.thin_film_thickness > 0.0f)) return no_film;
    Vec3 unc = thin_film_conductor(c, 1.0f, p.thin_film_ior, p.metal_n, p.metal_k, p.thin_film_thickness);
    Vec3 f = unc;
    if (p.coat > 0.0f) {
      Vec3 coated = thin_film_conductor(c, p.coat_eta, p.thin_film_ior, p.metal_n, p.metal_k, p.thin_film_thickness);
      f = lerp3(unc, coated, clampf(p.coat, 0.0f, 1.0f));
    }
    return lerp3(no_film, f, w);
  }
  Vec3 metal_f82(float c) const {  // metal_f82_tint_fresnel (open_pbr.rs:792-802)
    Vec3 f0 = vmax(p.base * p.base_color, Vec3(0, 0, 0));
    Vec3 fs = schlick3(f0, c);
    Vec3 fs82 = schlick3_82(f0);
    Vec3 ft82 = vclamp01(p.specular_color) * fs82;
    float cc = clampf(c, 0.0f, 1.0f);
    float corr = cc * powi(1.0f - cc, 6) / fmax_num(cos82_denom(), 1.0e-8f);
    return vclamp01(p.specular * (fs - corr * (fs82 - ft82)));
  }
  // metal_fresnel_avg (open_pbr.rs:818-830): the closed form without film,
  // else a 16-point cosine-weighted average of the filmed Fresnel
  Vec3 metal_fresnel_avg() const {
    if (!film()) return metal_f82_avg();
    Vec3 sum(0, 0, 0);
    for (int i = 0; i < 16; ++i) {
      float mu = ((float)i + 0.5f) / 16.0f;
      sum += metal_fresnel(mu) * (2.0f * mu);
    }
    return sum / 16.0f;
  }
  Vec3 metal_f82_avg() const {
    Vec3 f0 = vmax(p.base * p.base_color, Vec3(0, 0, 0));
    Vec3 fs82 = schlick3_82(f0);
    Vec3 ft82 = vclamp01(p.specular_color) * fs82;
    Vec3 b = (fs82 - ft82) / fmax_num(cos82_denom(), 1.0e-8f);
    return vclamp01(p.specular * (f0 + (Vec3(1, 1, 1) - f0) / 21.0f - b / 126.0f));
  }
  Vec3 eval_metal_ms(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return Vec3(0, 0, 0);
    float req = conductor_req();
    float e_o = L.conductor->lookup_e(wo.z, req), e_i = L.conductor->lookup_e(wi.z, req);
    float e_avg = L.conductor->lookup_e_avg(req);
    float om = fmax_num(1.0f - e_avg, kMsDenomEps);
    Vec3 f_ms = conductor_f_ms(metal_fresnel_avg(), e_avg);
    return f_ms * ((1.0f - e_o) * (1.0f - e_i) / (kPi * om));
  }
  Vec3 eval_metal(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return Vec3(0, 0, 0);
    Vec3 wm;
    if (!reflection_half_vector(wo, wi, &wm)) return Vec3(0, 0, 0);
    float d = ggx_d(wm, p.specular_alpha_x, p.specular_alpha_y);
    float g = ggx_g2(wo, wi, p.specular_alpha_x, p.specular_alpha_y);
    if (d <= 0.0f || g <= 0.0f) return Vec3(0, 0, 0);
    Vec3 f = metal_fresnel(std::fabs(dot(wo, wm)));
    Vec3 ss = f * (d * g / (4.0f * wo.z * wi.z));
    return ss + eval_metal_ms(wo, wi);
  }
  float base_dielectric_fresnel(float c, float eta_ph, float eta_pr) const {
    float unc = p.front_face ? weighted_fresnel_ratio(c, eta_ph, eta_pr)
                             : weighted_fresnel_ratio(c, 1.0f / eta_ph, 1.0f / eta_pr);
    float coat = clampf(p.coat, 0.0f, 1.0f);
    if (coat <= 0.0f) return unc;
    float eta_bc = eta_ph / fmax_num(p.coat_eta, 1.0e-4f);
    float eta_bcp = eta_pr / fmax_num(p.coat_eta, 1.0e-4f);
    float a = eta_bc, b = eta_bcp;
    if (p.coat_eta > eta_ph) {
      a = 1.0f / fmax_num(eta_bc, 1.0e-4f);
      b = 1.0f / fmax_num(eta_bcp, 1.0e-4f);
    }
    float coated = p.front_face
                       ? weighted_fresnel_ratio(c, a, b)
                       : weighted_fresnel_ratio(c, 1.0f / fmax_num(a, 1.0e-4f), 1.0f / fmax_num(b, 1.0e-4f));
    return lerp(unc, coated, coat);
  }
  // spec_brdf_fresnel (open_pbr.rs:869-898) and spec_btdf_fresnel_with_eta
  // (1120-1152, film only off thin-walled surfaces): the dielectric Fresnel,
  // blended with the filmed reflectance (over the coat's eta where coated)
  Vec3 filmed_dielectric(Vec3 no_film, float c, float eta_base) const {
    float w = clampf(p.thin_film_weight, 0.0f, 1.0f);
    if (!(w > 0.0f && p.thin_film_thickness > 0.0f)) return no_film;
    Vec3 unc = thin_film_dielectric(c, 1.0f, p.thin_film_ior, eta_base, p.thin_film_thickness);
    Vec3 f = unc;
    if (p.coat > 0.0f) {
      Vec3 coated = thin_film_dielectric(c, p.coat_eta, p.thin_film_ior, eta_base, p.thin_film_thickness);
      f = lerp3(unc, coated, clampf(p.coat, 0.0f, 1.0f));
    }
    return lerp3(no_film, f, w);
  }
  Vec3 spec_fresnel(float c) const {
    return filmed_dielectric(Vec3::splat(base_dielectric_fresnel(c, p.transmission_eta, p.specular_eta)), c,
                             p.specular_eta);
  }
  Vec3 btdf_fresnel(float c, float eta_ph, float eta_pr) const {
    Vec3 no_film = Vec3::splat(base_dielectric_fresnel(c, eta_ph, eta_pr));
    return p.thin_walled ? no_film : filmed_dielectric(no_film, c, eta_pr);
  }
  Vec3 eval_spec_brdf(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return Vec3(0, 0, 0);
    Vec3 wm;
    if (!reflection_half_vector(wo, wi, &wm)) return Vec3(0, 0, 0);
    float d = ggx_d(wm, p.specular_alpha_x, p.specular_alpha_y);
    float g = ggx_g2(wo, wi, p.specular_alpha_x, p.specular_alpha_y);
    if (d <= 0.0f || g <= 0.0f) return Vec3(0, 0, 0);
    if (p.thin_walled) {
      Vec3 R, T;
      thin_wall_coeffs(std::fabs(wo.z), &R, &T);
      return R * (d * g / (4.0f * wo.z * wi.z));
    }
    Vec3 f = spec_fresnel(std::fabs(dot(wo, wm)));
    Vec3 ss = f * (d * g / (4.0f * wo.z * wi.z));
    Vec3 ms = Vec3::splat(eval_refl_ms(wo, wi, p.specular_alpha_x, p.specular_alpha_y, p.specular_eta));
    return ss + ms;
  }
  float pdf_spec_ss(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
    Vec3 wm;
    if (!reflection_half_vector(wo, wi, &wm)) return 0.0f;
    float pdf_wm = pdf_wm_bounded_vndf(wo, wm, p.specular_alpha_x, p.specular_alpha_y);
    float denom = 4.0f * std::fabs(dot(wo, wm));
    if (denom <= 0.0f) return 0.0f;
    return pdf_wm / denom;
  }
  float pdf_metal(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
    TwoLobe w = conductor_lobe_weights();
    return (w.ss * pdf_spec_ss(wo, wi) + w.ms * cosine_pdf(wi.z)) / w.total;
  }
  float pdf_spec_brdf(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
    if (p.thin_walled) return pdf_spec_ss(wo, wi);
    MsParams m = ms_params(p.specular_alpha_x, p.specular_alpha_y, p.specular_eta);
    TwoLobe w = reflection_lobe_weights(m);
    return (w.ss * pdf_spec_ss(wo, wi) + w.ms * cosine_pdf(wi.z)) / w.total;
  }

  // thin_wall_coefficients (open_pbr.rs:931-959) without thin film: the slab's
  // reflectance and transmittance with the absorption of its interior
  void thin_wall_coeffs(float cos_theta_o, Vec3* R, Vec3* T) const {
    const Vec3 one(1, 1, 1);
    float eta = fmax_num(p.transmission_eta, 1.0e-4f);
    float eta_prime = fmax_num(p.specular_eta, 1.0e-4f);
    float cos_o = clampf(cos_theta_o, 0.0f, 1.0f);
    float sin2_o = fmax_num(1.0f - cos_o * cos_o, 0.0f);
    float sin2_i = clampf(sin2_o / (eta * eta), 0.0f, 1.0f);
    float cos_i = fmax_num(std::sqrt(1.0f - sin2_i), 1.0e-4f);
    Vec3 f_o = vclamp01(spec_fresnel(cos_o));
    // thin_wall_internal_fresnel (open_pbr.rs:961-979)
    Vec3 f_i = Vec3::splat(
        weighted_fresnel_ratio(cos_i, 1.0f / fmax_num(eta, 1.0e-4f), 1.0f / fmax_num(eta_prime, 1.0e-4f)));
    float w = clampf(p.thin_film_weight, 0.0f, 1.0f);
    if (w > 0.0f && p.thin_film_thickness > 0.0f)
      f_i = lerp3(f_i, thin_film_dielectric(cos_i, fmax_num(eta, 1.0e-4f), p.thin_film_ior, 1.0f, p.thin_film_thickness),
                  w);
    f_i = vclamp01(f_i);
    Vec3 a = vpowf(vclamp01(p.transmission_color), 1.0f / cos_i);
    Vec3 a2 = a * a;
    Vec3 f_i2_a2 = a2 * f_i * f_i;
    Vec3 denom = vmax(one - f_i2_a2, Vec3::splat(1.0e-6f));
    Vec3 omfo = vmax(one - f_o, Vec3(0, 0, 0));
    Vec3 omfi = vmax(one - f_i, Vec3(0, 0, 0));
    Vec3 refl = f_o + omfo * omfi * f_i * a2 / denom;
    Vec3 trans = omfo * omfi * a * (one + f_i2_a2 / denom);
    *R = vclamp01(refl);
    *T = vclamp01(trans);
  }
  // eval_dielectric_transmission_ms (open_pbr.rs:672-696)
  float eval_trans_ms(Vec3 wo, Vec3 wi, float ax, float ay, float eta, TransportMode mode) const {
    if (wo.z <= 0.0f || wi.z >= 0.0f) return 0.0f;
    MsParams m = ms_params(ax, ay, eta);
    float cos_o = wo.z, cos_i = std::fabs(wi.z);
    float e_o = L.dielectric->lookup_e(cos_o, m.roughness_eq, m.eta_o);
    float e_i = L.dielectric->lookup_e(cos_i, m.roughness_eq, m.eta_rel);
    float scale = trans_scale(mode, m.eta_rel);
    return (1.0f - m.ratio_r) * (1.0f - e_o) * (1.0f - e_i) * scale / (kPi * m.one_minus_e_avg_t);
  }
  // dispersion (open_pbr.rs:1223-1253): the etas at the path's locked
  // wavelength, and whether an unlocked path integrates over the camera basis
  bool dispersive() const { return p.transmission_dispersion_abbe > 0.0f; }
  float eta_used() const {
    return p.has_lock && dispersive() ? cauchy_ior(p.wavelength_lock, p.transmission_eta, p.transmission_dispersion_abbe)
                                      : p.transmission_eta;
  }
  float fresnel_eta_used() const {
    return p.has_lock && dispersive() ? cauchy_ior(p.wavelength_lock, p.specular_eta, p.transmission_dispersion_abbe)
                                      : p.specular_eta;
  }
  float eta_rel_t() const {
    const float eta = eta_used();
    return p.front_face ? 1.0f / eta : eta;
  }
  bool camera_dispersion() const { return dispersive() && p.front_face && !btdf_smooth(); }
  struct Channel {
    float lambda;
    int color;
    float probability;
  };
  // sampled_dispersion_channels / pick_dispersion_channel (open_pbr.rs:1314-1354)
  void dispersion_channels(const float* u_rgb, Channel* ch) const {
    const Vec3 t = vmax(p.path_throughput, Vec3(0, 0, 0));
    const Vec3 w = max_element(t) > 0.0f ? t : Vec3(1, 1, 1);
    const float sum = fmax_num(w.x + w.y + w.z, 1.0e-8f);
    ch[0] = Channel{sample_camera_channel_wavelength(0, u_rgb[0]), 0, w.x / sum};
    ch[1] = Channel{sample_camera_channel_wavelength(1, u_rgb[1]), 1, w.y / sum};
    ch[2] = Channel{sample_camera_channel_wavelength(2, u_rgb[2]), 2, w.z / sum};
  }
  static Channel pick_channel(const Channel* ch, float u) {
    u = clampf(u, 0.0f, 1.0f);
    for (int k = 0; k < 3; ++k) {
      if (u <= ch[k].probability) return ch[k];
      u -= ch[k].probability;
    }
    return ch[2];
  }
  static Vec3 unit(int c) { return Vec3(c == 0 ? 1.0f : 0.0f, c == 1 ? 1.0f : 0.0f, c == 2 ? 1.0f : 0.0f); }
  // eval_spec_btdf_scalar_with_eta (open_pbr.rs:1074-1117): false for None
  bool btdf_scalar(Vec3 wo, Vec3 wi, float eta_rel, TransportMode mode, float* scalar, float* cos_wo_wm) const {
    Vec3 wmu = eta_rel * wo + wi;
    if (length_squared(wmu) < 1.0e-12f) return false;
    Vec3 wm = normalize(wmu);
    if (wm.z < 0.0f) wm = -wm;
    float co = dot(wo, wm);
    if (co <= 0.0f) return false;
    float ci = dot(wi, wm);
    float den = ci + eta_rel * co;
    if (std::fabs(den) < 1.0e-6f) return false;
    float d = ggx_d(wm, p.transmission_alpha_x, p.transmission_alpha_y);
    float g = ggx_g2(wo, wi, p.transmission_alpha_x, p.transmission_alpha_y);
    if (d <= 0.0f || g <= 0.0f) return false;
    float scale = trans_scale(mode, eta_rel);
    float s = d * g * std::fabs(ci * co);
    float denom = den * den * std::fabs(wo.z) * std::fabs(wi.z);
    if (denom <= 0.0f) return false;
    *scalar = s * scale / denom;
    *cos_wo_wm = co;
    return true;
  }
  // eval_thin_wall_spec_btdf (open_pbr.rs:1053-1072)
  Vec3 eval_thin_btdf(Vec3 wo, Vec3 wi) const {
    if (wo.z <= 0.0f || wi.z >= 0.0f) return Vec3(0, 0, 0);
    Vec3 R, T;
    thin_wall_coeffs(std::fabs(wo.z), &R, &T);
    if (btdf_smooth()) return Vec3(0, 0, 0);
    Vec3 wim(wi.x, wi.y, -wi.z);
    Vec3 wm;
    if (!reflection_half_vector(wo, wim, &wm)) return Vec3(0, 0, 0);
    float ax, ay;
    thin_wall_alpha(&ax, &ay);
    float d = ggx_d(wm, ax, ay);
    float g = ggx_g2(wo, wim, ax, ay);
    if (d <= 0.0f || g <= 0.0f) return Vec3(0, 0, 0);
    return T * (d * g / (4.0f * wo.z * std::fabs(wi.z)));
  }
  // eval_spec_btdf (open_pbr.rs:1024-1051), no dispersion
  Vec3 eval_spec_btdf(Vec3 wo, Vec3 wi, TransportMode mode) const {
    if (p.thin_walled) return eval_thin_btdf(wo, wi);
    if (wo.z <= 0.0f || wi.z >= 0.0f) return Vec3(0, 0, 0);
    float scalar, co;
    if (camera_dispersion() && !p.has_lock) return eval_btdf_camera(wo, wi, mode);
    if (!btdf_scalar(wo, wi, eta_rel_t(), mode, &scalar, &co)) return Vec3(0, 0, 0);
    const float eta_fr = fresnel_eta_used();
    Vec3 f = btdf_fresnel(co, eta_used(), eta_fr);
    Vec3 ss = vmax(Vec3(1, 1, 1) - f, Vec3(0, 0, 0)) * scalar;
    Vec3 ms = Vec3::splat(eval_trans_ms(wo, wi, p.transmission_alpha_x, p.transmission_alpha_y, eta_fr, mode));
    return ss + ms;
  }
  // eval_spec_btdf_camera_integrated (open_pbr.rs:1255-1289): the BTDF summed
  // over the 32 camera intervals at their midpoint wavelengths
  Vec3 eval_btdf_camera(Vec3 wo, Vec3 wi, TransportMode mode) const {
    Vec3 value(0, 0, 0);
    for (int i = 0; i < kSpectralIntervals; ++i) {
      const float lambda = camera_spectral_interval_midpoint_nm(i);
      const float eta = cauchy_ior(lambda, p.transmission_eta, p.transmission_dispersion_abbe);
      const float eta_fr = cauchy_ior(lambda, p.specular_eta, p.transmission_dispersion_abbe);
      const float eta_rel = p.front_face ? 1.0f / eta : eta;
      Vec3 ss(0, 0, 0);
      float scalar, co;
      if (btdf_scalar(wo, wi, eta_rel, mode, &scalar, &co))
        ss = vmax(Vec3(1, 1, 1) - btdf_fresnel(co, eta, eta_fr), Vec3(0, 0, 0)) * scalar;
      const Vec3 ms =
          Vec3::splat(eval_trans_ms(wo, wi, p.transmission_alpha_x, p.transmission_alpha_y, eta_fr, mode));
      value += camera_rgb_basis_at(lambda) * (ss + ms) * kLambdaStepNm;
    }
    return value;
  }
  // eval_spec_btdf_sampled_channels (open_pbr.rs:1356-1397)
  Vec3 eval_btdf_channels(Vec3 wo, Vec3 wi, const Channel* ch, TransportMode mode) const {
    Vec3 value(0, 0, 0);
    for (int k = 0; k < 3; ++k) {
      if (ch[k].probability <= 0.0f) continue;
      const float eta = cauchy_ior(ch[k].lambda, p.transmission_eta, p.transmission_dispersion_abbe);
      const float eta_fr = cauchy_ior(ch[k].lambda, p.specular_eta, p.transmission_dispersion_abbe);
      const float eta_rel = p.front_face ? 1.0f / eta : eta;
      const Vec3 color = unit(ch[k].color);
      float ss = 0.0f, scalar, co;
      if (btdf_scalar(wo, wi, eta_rel, mode, &scalar, &co))
        ss = fmax_num(1.0f - dot(btdf_fresnel(co, eta, eta_fr), color), 0.0f) * scalar;
      const float ms = eval_trans_ms(wo, wi, p.transmission_alpha_x, p.transmission_alpha_y, eta_fr, mode);
      value += color * (ss + ms);
    }
    return value;
  }
  // pdf_specular_btdf_ss_with_eta (open_pbr.rs:1193-1222)
  float pdf_btdf_ss(Vec3 wo, Vec3 wi, float eta_rel) const {
    Vec3 wmu = eta_rel * wo + wi;
    if (length_squared(wmu) < 1.0e-12f) return 0.0f;
    Vec3 wm = normalize(wmu);
    if (wm.z < 0.0f) wm = -wm;
    float co = dot(wo, wm);
    if (co <= 0.0f) return 0.0f;
    float ci = dot(wi, wm);
    float den = ci + eta_rel * co;
    if (std::fabs(den) < 1.0e-6f) return 0.0f;
    float pdf_wm = pdf_wm_vndf(wo, wm, p.transmission_alpha_x, p.transmission_alpha_y);
    if (pdf_wm <= 0.0f) return 0.0f;
    return pdf_wm * std::fabs(ci) / (den * den);
  }
  // pdf_specular_btdf and _with_eta (open_pbr.rs:1154-1191), no dispersion
  float pdf_spec_btdf(Vec3 wo, Vec3 wi) const {
    if (p.thin_walled) {
      if (btdf_smooth() || wo.z <= 0.0f || wi.z >= 0.0f) return 0.0f;
      Vec3 wim(wi.x, wi.y, -wi.z);
      Vec3 wm;
      if (!reflection_half_vector(wo, wim, &wm)) return 0.0f;
      float ax, ay;
      thin_wall_alpha(&ax, &ay);
      float pdf_wm = pdf_wm_bounded_vndf(wo, wm, ax, ay);
      float denom = 4.0f * std::fabs(dot(wo, wm));
      return denom > 0.0f ? pdf_wm / denom : 0.0f;
    }
    if (wo.z <= 0.0f || wi.z >= 0.0f) return 0.0f;
    if (camera_dispersion() && !p.has_lock) return pdf_btdf_camera(wo, wi);
    return pdf_btdf_with_eta(wo, wi, eta_rel_t(), eta_used());
  }
  float pdf_btdf_with_eta(Vec3 wo, Vec3 wi, float eta_rel, float eta) const {
    if (wo.z <= 0.0f || wi.z >= 0.0f) return 0.0f;
    MsParams m = ms_params(p.transmission_alpha_x, p.transmission_alpha_y, eta);
    TwoLobe w = transmission_lobe_weights(m);
    float pdf_ss = pdf_btdf_ss(wo, wi, eta_rel);
    float pdf_ms = cosine_pdf(-wi.z);
    return (w.ss * pdf_ss + w.ms * pdf_ms) / w.total;
  }
  // pdf_specular_btdf_camera_mixture (open_pbr.rs:1291-1312)
  float pdf_btdf_camera(Vec3 wo, Vec3 wi) const {
    float pdf = 0.0f;
    for (int i = 0; i < kSpectralIntervals; ++i) {
      const float lambda = camera_spectral_interval_midpoint_nm(i);
      const float eta = cauchy_ior(lambda, p.transmission_eta, p.transmission_dispersion_abbe);
      const float eta_fr = cauchy_ior(lambda, p.specular_eta, p.transmission_dispersion_abbe);
      const float eta_rel = p.front_face ? 1.0f / eta : eta;
      const float p_lambda = camera_wavelength_sampling_pdf(lambda, p.path_throughput);
      pdf += p_lambda * pdf_btdf_with_eta(wo, wi, eta_rel, eta_fr) * kLambdaStepNm;
    }
    return pdf;
  }
  // pdf_specular_btdf_sampled_channel_mixture (open_pbr.rs:1399-1427)
  float pdf_btdf_channels(Vec3 wo, Vec3 wi, const Channel* ch) const {
    float pdf = 0.0f;
    for (int k = 0; k < 3; ++k) {
      if (ch[k].probability <= 0.0f) continue;
      const float eta = cauchy_ior(ch[k].lambda, p.transmission_eta, p.transmission_dispersion_abbe);
      const float eta_fr = cauchy_ior(ch[k].lambda, p.specular_eta, p.transmission_dispersion_abbe);
      const float eta_rel = p.front_face ? 1.0f / eta : eta;
      pdf += ch[k].probability * pdf_btdf_with_eta(wo, wi, eta_rel, eta_fr);
    }
    return pdf;
  }
  // eval_diff_btdf / pdf_diff_btdf (open_pbr.rs:1445-1465): thin-walled only
  Vec3 eval_diff_btdf(Vec3 wo, Vec3 wi) const {
    if (!p.thin_walled || wo.z <= 0.0f || wi.z >= 0.0f) return Vec3(0, 0, 0);
    return Eon(p.diffuse_roughness).eval(wo, Vec3(wi.x, wi.y, -wi.z));
  }
  float pdf_diff_btdf(Vec3 wo, Vec3 wi) const {
    if (!p.thin_walled || wo.z <= 0.0f || wi.z >= 0.0f) return 0.0f;
    return Eon(p.diffuse_roughness).pdf(wo, Vec3(wi.x, wi.y, -wi.z));
  }

  // open_pbr.rs:224-296
  Vec3 eval(Vec3 wo, Vec3 wi, TransportMode mode) const {
    if (!(wo.z > 0.0f)) return Vec3(0, 0, 0);
    Vec3 layer_wo = mode == kImportance ? wi : wo;
    LayerWeights w = layer_weights(layer_wo, &wi);
    Vec3 total(0, 0, 0);
    if (w.coat_amp > 0.0f && !coat_smooth()) total += w.coat_amp * eval_coat(wo, wi);
    if (length_squared(w.metal) > 0.0f && !metal_smooth()) total += w.metal * eval_metal(wo, wi);
    if (length_squared(w.spec_brdf) > 0.0f && !spec_smooth()) total += w.spec_brdf * eval_spec_brdf(wo, wi);
    if (length_squared(w.spec_btdf) > 0.0f && !btdf_smooth()) total += w.spec_btdf * eval_spec_btdf(wo, wi, mode);
    if (length_squared(w.fuzz) > 0.0f) total += w.fuzz * Fuzz(p.fuzz_roughness).eval(wo, wi);
    if (length_squared(w.diff_brdf) > 0.0f) total += w.diff_brdf * Eon(p.diffuse_roughness).eval(wo, wi);
    if (length_squared(w.diff_btdf) > 0.0f) total += w.diff_btdf * eval_diff_btdf(wo, wi);
    return total;
  }
  float pdf(Vec3 wo, Vec3 wi) const {
    if (!(wo.z > 0.0f)) return 0.0f;
    LobeProbs q = lobe_probabilities(wo);
    if (q.total <= 0.0f) return 0.0f;
    float pdf = 0.0f;
    if (q.coat > 0.0f && !coat_smooth()) pdf += (q.coat / q.total) * pdf_coat(wo, wi);
    if (q.metal > 0.0f && !metal_smooth()) pdf += (q.metal / q.total) * pdf_metal(wo, wi);
    if (q.spec_brdf > 0.0f && !spec_smooth()) pdf += (q.spec_brdf / q.total) * pdf_spec_brdf(wo, wi);
    if (q.spec_btdf > 0.0f && !btdf_smooth()) pdf += (q.spec_btdf / q.total) * pdf_spec_btdf(wo, wi);
    if (q.fuzz > 0.0f) pdf += (q.fuzz / q.total) * Fuzz(p.fuzz_roughness).pdf(wo, wi);
    if (q.diff_brdf > 0.0f) pdf += (q.diff_brdf / q.total) * Eon(p.diffuse_roughness).pdf(wo, wi);
    if (q.diff_btdf > 0.0f) pdf += (q.diff_btdf / q.total) * pdf_diff_btdf(wo, wi);
    return pdf;
  }

  // finalize_rough_sample_with_wavelength (open_pbr.rs:1997-2027)
  bool finalize(Vec3 wo, Vec3 wi, uint32_t flags, TransportMode mode, BsdfSample* out, float eta = 1.0f) const {
    float pdf_v = pdf(wo, wi);
    if (pdf_v <= 0.0f) return false;
    Vec3 f = eval(wo, wi, mode);
    if (length_squared(f) == 0.0f) return false;
    float c = std::fabs(wi.z);
    if (c <= 0.0f) return false;
    out->weight = f * (c / pdf_v);
    out->wi = wi;
    out->pdf = pdf_v;
    out->pdf_rev = pdf(wi, wo);
    out->flags = flags;
    out->eta = eta;
    return true;
  }
  bool delta_out(Vec3 wi, Vec3 weight, float p_lobe, BsdfSample* out) const {
    out->weight = weight;
    out->wi = wi;
    out->pdf = p_lobe;
    out->pdf_rev = 0.0f;
    out->flags = kDelta | kReflection;
    out->eta = 1.0f;
    return true;
  }
  // Rough two-lobe sampling (GGX single scattering or cosine multiple
  // scattering) shared by sample_coat / sample_metal / sample_spec_brdf.
  bool sample_two_lobe(Vec3 wo, Vec2 us, TwoLobe w, float ax, float ay, TransportMode mode, BsdfSample* out) const {
    float ss_p = w.ss / w.total;
    if (us.x >= ss_p) {
      float u = ss_p < 1.0f ? (us.x - ss_p) / (1.0f - ss_p) : 0.0f;
      Vec3 wi = sample_cosine_hemisphere(Vec2(u, us.y));
      return finalize(wo, wi, kGlossy | kReflection, mode, out);
    }
    float u = ss_p > 0.0f ? us.x / ss_p : 0.0f;
    Vec3 wm;
    if (!sample_wm_bounded_vndf(wo, ax, ay, Vec2(u, us.y), &wm)) return false;
    Vec3 wi = reflect_local(wo, wm);
    if (wi.z <= 0.0f) return false;
    return finalize(wo, wi, kGlossy | kReflection, mode, out);
  }
  bool sample_coat(Vec3 wo, Vec2 us, float p_lobe, TransportMode mode, BsdfSample* out) const {
    if (wo.z <= 0.0f) return false;
    if (coat_smooth()) {
      Vec3 wi(-wo.x, -wo.y, wo.z);
      float f = fresnel_dielectric(std::fabs(wi.z), 1.0f, p.coat_eta);
      return delta_out(wi, Vec3::splat(layer_weights(wo, &wi).coat_amp * f / p_lobe), p_lobe, out);
    }
    MsParams m = ms_params(p.coat_alpha_x, p.coat_alpha_y, p.coat_eta);
    return sample_two_lobe(wo, us, reflection_lobe_weights(m), p.coat_alpha_x, p.coat_alpha_y, mode, out);
  }
  bool sample_metal(Vec3 wo, Vec2 us, float p_lobe, TransportMode mode, BsdfSample* out) const {
    if (metal_smooth()) {
      Vec3 wi(-wo.x, -wo.y, wo.z);
      Vec3 f = metal_fresnel(std::fabs(wi.z));
      return delta_out(wi, (layer_weights(wo, &wi).metal * f) / p_lobe, p_lobe, out);
    }
    return sample_two_lobe(wo, us, conductor_lobe_weights(), p.specular_alpha_x, p.specular_alpha_y, mode, out);
  }
  bool sample_spec(Vec3 wo, Vec2 us, float p_lobe, TransportMode mode, BsdfSample* out) const {
    if (spec_smooth()) {
      Vec3 wi(-wo.x, -wo.y, wo.z);
      Vec3 f;
      if (p.thin_walled) {
        Vec3 T;
        thin_wall_coeffs(std::fabs(wo.z), &f, &T);
      } else {
        f = spec_fresnel(std::fabs(wi.z));
      }
      return delta_out(wi, (layer_weights(wo, &wi).spec_brdf * f) / p_lobe, p_lobe, out);
    }
    if (p.thin_walled) {
      Vec3 wm;
      if (!sample_wm_bounded_vndf(wo, p.specular_alpha_x, p.specular_alpha_y, us, &wm)) return false;
      Vec3 wi = reflect_local(wo, wm);
      if (wi.z <= 0.0f) return false;
      return finalize(wo, wi, kGlossy | kReflection, mode, out);
    }
    MsParams m = ms_params(p.specular_alpha_x, p.specular_alpha_y, p.specular_eta);
    return sample_two_lobe(wo, us, reflection_lobe_weights(m), p.specular_alpha_x, p.specular_alpha_y, mode, out);
  }
  // math/mod.rs:83-100
  static bool refract_z(Vec3 wo, float eta, Vec3* out) {
    if (wo.z <= 0.0f) return false;
    float sin2_o = fmax_num(1.0f - wo.z * wo.z, 0.0f);
    float sin2_t = eta * eta * sin2_o;
    if (sin2_t >= 1.0f) return false;
    float cos_t = std::sqrt(fmax_num(1.0f - sin2_t, 0.0f));
    Vec3 wi = normalize_or_zero(Vec3(-eta * wo.x, -eta * wo.y, -cos_t));
    if (length_squared(wi) == 0.0f) return false;
    *out = wi;
    return true;
  }
  // refract_about (open_pbr.rs:2043-2058)
  static bool refract_about(Vec3 wo, Vec3 wm, float eta, Vec3* out) {
    float cos_o = dot(wo, wm);
    if (cos_o <= 0.0f) return false;
    float sin2_t = eta * eta * fmax_num(1.0f - cos_o * cos_o, 0.0f);
    if (sin2_t >= 1.0f) return false;
    float cos_t = std::sqrt(fmax_num(1.0f - sin2_t, 0.0f));
    Vec3 wi = normalize_or_zero(-eta * wo + (eta * cos_o - cos_t) * wm);
    if (length_squared(wi) == 0.0f) return false;
    *out = wi;
    return true;
  }
  // sample_spec_btdf_camera_channels (open_pbr.rs:1838-1928): one of three
  // per-channel wavelengths picked by throughput, the direction sampled at its
  // eta, weighted by the three-channel BTDF over the channel-mixture pdf
  bool sample_btdf_channels(Vec3 wo, Vec2 us, float p_lobe, float u_pick, const float* u_rgb, TransportMode mode,
                            BsdfSample* out) const {
    Channel ch[3];
    dispersion_channels(u_rgb, ch);
    const Channel c = pick_channel(ch, u_pick);
    if (c.probability <= 0.0f) return false;
    const float eta_u = cauchy_ior(c.lambda, p.transmission_eta, p.transmission_dispersion_abbe);
    const float eta_fr = cauchy_ior(c.lambda, p.specular_eta, p.transmission_dispersion_abbe);
    const float eta_rel = p.front_face ? 1.0f / eta_u : eta_u;
    MsParams m = ms_params(p.transmission_alpha_x, p.transmission_alpha_y, eta_fr);
    TwoLobe w = transmission_lobe_weights(m);
    float ss_p = w.ss / w.total;
    Vec3 wi;
    if (us.x >= ss_p) {
      float u = ss_p < 1.0f ? (us.x - ss_p) / (1.0f - ss_p) : 0.0f;
      Vec3 up = sample_cosine_hemisphere(Vec2(u, us.y));
      wi = Vec3(up.x, up.y, -up.z);
    } else {
      float u = ss_p > 0.0f ? us.x / ss_p : 0.0f;
      Vec3 wm;
      if (!sample_wm_vndf(wo, p.transmission_alpha_x, p.transmission_alpha_y, Vec2(u, us.y), &wm)) return false;
      if (dot(wo, wm) <= 0.0f) return false;
      if (!refract_about(wo, wm, eta_rel, &wi)) return false;
      if (wi.z >= 0.0f) return false;
    }
    if (wi.z >= 0.0f) return false;
    Vec3 bw = layer_weights(wo, &wi).spec_btdf;
    float pdf_total = p_lobe * pdf_btdf_channels(wo, wi, ch);
    if (pdf_total <= 0.0f) return false;
    Vec3 f = eval_btdf_channels(wo, wi, ch, mode);
    out->weight = bw * f * (std::fabs(wi.z) / pdf_total);
    out->wi = wi;
    out->pdf = pdf_total;
    out->pdf_rev = pdf(wi, wo);
    out->flags = kGlossy | kTransmission;
    out->eta = eta_rel;
    out->has_lock = true;
    out->wavelength_lock = c.lambda;
    return true;
  }
  // sample_spec_btdf (open_pbr.rs:1670-1836): u_aux draws the wavelength of a
  // smooth dispersive refraction, u_rgb the per-channel wavelengths of a rough one
  bool sample_spec_btdf(Vec3 wo, Vec2 us, float p_lobe, float u_aux, const float* u_rgb, TransportMode mode,
                        BsdfSample* out) const {
    if (p.thin_walled) {
      Vec3 R, T;
      thin_wall_coeffs(std::fabs(wo.z), &R, &T);
      if (btdf_smooth()) {
        Vec3 wi = -wo;
        Vec3 bw = layer_weights(wo, &wi).spec_btdf;
        out->weight = (bw * T) / p_lobe;
        out->wi = wi;
        out->pdf = p_lobe;
        out->pdf_rev = 0.0f;
        out->flags = kDelta | kTransmission;
        out->eta = 1.0f;
        return true;
      }
      float ax, ay;
      thin_wall_alpha(&ax, &ay);
      Vec3 wm;
      if (!sample_wm_bounded_vndf(wo, ax, ay, us, &wm)) return false;
      Vec3 wr = reflect_local(wo, wm);
      if (wr.z <= 0.0f) return false;
      Vec3 wi(wr.x, wr.y, -wr.z);
      Vec3 bw = layer_weights(wo, &wi).spec_btdf;
      float pdf_total = p_lobe * pdf_spec_btdf(wo, wi);
      if (pdf_total <= 0.0f) return false;
      Vec3 f = eval_thin_btdf(wo, wi);
      out->weight = bw * f * std::fabs(wi.z) / pdf_total;
      out->wi = wi;
      out->pdf = pdf_total;
      out->pdf_rev = pdf(wi, wo);
      out->flags = kGlossy | kTransmission;
      out->eta = 1.0f;
      return true;
    }
    if (camera_dispersion() && !p.has_lock) return sample_btdf_channels(wo, us, p_lobe, u_aux, u_rgb, mode, out);
    float eta_used = p.transmission_eta;
    Vec3 dispersion_basis(1, 1, 1);
    bool fresh = false;
    float fresh_lambda = 0.0f;
    if (dispersive()) {
      if (p.has_lock) {
        eta_used = cauchy_ior(p.wavelength_lock, p.transmission_eta, p.transmission_dispersion_abbe);
      } else if (p.front_face) {
        fresh_lambda = sample_dispersion_wavelength_weighted(u_aux, p.path_throughput, &dispersion_basis);
        eta_used = cauchy_ior(fresh_lambda, p.transmission_eta, p.transmission_dispersion_abbe);
        fresh = true;
      }
    }
    float eta_fresnel = p.specular_eta;
    if ((fresh || p.has_lock) && dispersive())
      eta_fresnel = cauchy_ior(fresh ? fresh_lambda : p.wavelength_lock, p.specular_eta, p.transmission_dispersion_abbe);
    const float eta_rel = p.front_face ? 1.0f / eta_used : eta_used;
    out->has_lock = fresh;
    out->wavelength_lock = fresh_lambda;
    if (btdf_smooth()) {
      Vec3 wi;
      if (!refract_z(wo, eta_rel, &wi)) return false;
      float f = base_dielectric_fresnel(std::fabs(wo.z), eta_used, eta_fresnel);
      float scale = trans_scale(mode, eta_rel);
      Vec3 bw = layer_weights(wo, &wi).spec_btdf;
      out->weight = (bw * dispersion_basis * (1.0f - f) * scale) / p_lobe;
      out->wi = wi;
      out->pdf = p_lobe;
      out->pdf_rev = 0.0f;
      out->flags = kDelta | kTransmission;
      out->eta = eta_rel;
      return true;
    }
    MsParams m = ms_params(p.transmission_alpha_x, p.transmission_alpha_y, eta_fresnel);
    TwoLobe w = transmission_lobe_weights(m);
    float ss_p = w.ss / w.total;
    if (us.x >= ss_p) {
      float u = ss_p < 1.0f ? (us.x - ss_p) / (1.0f - ss_p) : 0.0f;
      Vec3 up = sample_cosine_hemisphere(Vec2(u, us.y));
      return finalize(wo, Vec3(up.x, up.y, -up.z), kGlossy | kTransmission, mode, out, eta_rel);
    }
    float u = ss_p > 0.0f ? us.x / ss_p : 0.0f;
    Vec3 wm;
    if (!sample_wm_vndf(wo, p.transmission_alpha_x, p.transmission_alpha_y, Vec2(u, us.y), &wm)) return false;
    float co = dot(wo, wm);
    if (co <= 0.0f) return false;
    Vec3 wi;
    if (!refract_about(wo, wm, eta_rel, &wi)) return false;
    if (wi.z >= 0.0f) return false;
    float ci = dot(wi, wm);
    float den = ci + eta_rel * co;
    if (std::fabs(den) < 1.0e-6f) return false;
    return finalize(wo, wi, kGlossy | kTransmission, mode, out, eta_rel);
  }
  // open_pbr.rs:298-332 and pick_lobe (open_pbr.rs:2043-2070)
  bool sample(Vec3 wo, float u_lobe, Vec2 us, TransportMode mode, BsdfSample* out, const float* u_extra) const {
    if (!(wo.z > 0.0f)) return false;
    LobeProbs q = lobe_probabilities(wo);
    if (q.total <= 0.0f) return false;
    float u = u_lobe * q.total;
    Lobe lobe;
    float pl;
    if (u < q.coat) { lobe = kCoat; pl = q.coat; }
    else if ((u -= q.coat) < q.metal) { lobe = kMetal; pl = q.metal; }
    else if ((u -= q.metal) < q.spec_brdf) { lobe = kSpecBrdf; pl = q.spec_brdf; }
    else if ((u -= q.spec_brdf) < q.spec_btdf) { lobe = kSpecBtdf; pl = q.spec_btdf; }
    else if ((u -= q.spec_btdf) < q.fuzz) { lobe = kFuzzLobe; pl = q.fuzz; }
    else if ((u -= q.fuzz) < q.diff_brdf) { lobe = kDiffBrdf; pl = q.diff_brdf; }
    else { lobe = kDiffBtdf; pl = q.diff_btdf; }
    float p_lobe = pl / q.total;
    if (p_lobe <= 0.0f) return false;
    switch (lobe) {
      case kCoat: return sample_coat(wo, us, p_lobe, mode, out);
      case kMetal: return sample_metal(wo, us, p_lobe, mode, out);
      case kSpecBrdf: return sample_spec(wo, us, p_lobe, mode, out);
      case kFuzzLobe: {
        Vec3 wi;
        if (!Fuzz(p.fuzz_roughness).sample(wo, us, &wi)) return false;
        return finalize(wo, wi, kGlossy | kReflection, mode, out);
      }
      case kDiffBrdf: {
        Vec3 wi;
        if (!Eon(p.diffuse_roughness).sample(wo, us, &wi)) return false;
        return finalize(wo, wi, kDiffuse | kReflection, mode, out);
      }
      case kSpecBtdf: return sample_spec_btdf(wo, us, p_lobe, u_extra[0], u_extra + 1, mode, out);
      default: {  // kDiffBtdf: sample_diff_btdf (open_pbr.rs:1942-1957), thin-walled only
        if (!p.thin_walled) return false;
        Vec3 wi;
        if (!Eon(p.diffuse_roughness).sample(wo, us, &wi)) return false;
        return finalize(wo, Vec3(wi.x, wi.y, -wi.z), kDiffuse | kTransmission, mode, out);
      }
    }
  }
};

// material/open_pbr.rs:860-870
}  // namespace

// EonBsdf with an arbitrary rho (eon.rs:25-58), for the lobe's own unit tests.
Vec3 eon_eval(Vec3 rho, float roughness, Vec3 wo, Vec3 wi) {
  float r = clampf(roughness, 0.0f, 1.0f);
  if (wo.z <= 0.0f || wi.z <= 0.0f) return Vec3(0, 0, 0);
  return f_eon(rho, r, wo, wi);
}
float eon_pdf(float roughness, Vec3 wo, Vec3 wi) { return Eon(roughness).pdf(wo, wi); }
bool eon_sample(Vec3 rho, float roughness, Vec3 wo, Vec2 us, BsdfSample* s) {
  float r = clampf(roughness, 0.0f, 1.0f);
  if (wo.z <= 0.0f) return false;
  float pdf;
  Vec3 wi = sample_eon(wo, r, us.x, us.y, &pdf);
  if (pdf <= 0.0f || wi.z <= 0.0f) return false;
  s->weight = f_eon(rho, r, wo, wi) * (wi.z / pdf);
  s->wi = wi;
  s->pdf = pdf;
  s->pdf_rev = eon_pdf(roughness, wi, wo);
  s->flags = kDiffuse | kReflection;
  s->eta = 1.0f;
  return true;
}

namespace {
void alpha_xy(float roughness, float anisotropy, float* ax, float* ay) {
  float r = clampf(roughness, 0.0f, 1.0f);
  float a = clampf(anisotropy, 0.0f, 1.0f);
  float alpha = r * r;
  float oma = 1.0f - a;
  float x = alpha * std::sqrt(2.0f / (1.0f + oma * oma));
  float y = oma * x;
  *ax = clampf(x, kMinAlpha, 1.0f);
  *ay = clampf(y, kMinAlpha, 1.0f);
}
float modulated_eta(float eta, float w) {  // material/open_pbr.rs:872-879
  if (std::fabs(w - 1.0f) < 1.0e-6f) return eta;
  float f0 = powi((eta - 1.0f) / (eta + 1.0f), 2);
  float eps = std::sqrt(clampf(w * f0, 0.0f, 0.99999f)) * std::copysign(1.0f, eta - 1.0f);
  return fmax_num((1.0f + eps) / fmax_num(1.0f - eps, 1.0e-6f), 1.0e-4f);
}
float dielectric_fresnel_avg(float eta) {  // material/open_pbr.rs:881-887
  eta = clampf(eta, 1.0f, 3.0f);
  return clampf(std::log(fmax_num((10893.0f * eta - 1438.2f) / (-774.4f * eta * eta + 10212.0f * eta + 1.0f), 1.0e-6f)),
                0.0f, 1.0f);
}
}  // namespace

Vec3 OpenPbrBsdf::eval(Vec3 wo, Vec3 wi, TransportMode mode) const { return Impl{p, L}.eval(wo, wi, mode); }
float OpenPbrBsdf::pdf(Vec3 wo, Vec3 wi) const { return Impl{p, L}.pdf(wo, wi); }
bool OpenPbrBsdf::sample(Vec3 wo, float u_lobe, Vec2 u_dir, TransportMode mode, BsdfSample* out,
                         const float* u_extra) const {
  static const float kZeros[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  return Impl{p, L}.sample(wo, u_lobe, u_dir, mode, out, u_extra ? u_extra : kZeros);
}

float openpbr_fuzz_albedo(float ndot_v, float roughness) { return zeltner_dir_albedo(ndot_v, roughness); }

float openpbr_specular_eta(const OpenPbrDesc& m) {
  return modulated_eta(fmax_num(m.specular_ior, 1.0e-4f), fmax_num(m.specular_weight, 0.0f));
}

// OpenPbrMaterial::make_bsdf (material/open_pbr.rs:393-487) and its helpers
// (effective roughness 749-783, coat darkening 823-858) without textures.
OpenPbrParams make_openpbr_params(const OpenPbrDesc& m, bool front_face, Vec3 wo_local) {
  const Vec3 base_color(m.base_color[0], m.base_color[1], m.base_color[2]);
  const float metalness = clampf(m.base_metalness, 0.0f, 1.0f);
  const float fuzz_w = clampf(m.fuzz_weight, 0.0f, 1.0f);
  const float fuzz_r = clampf(m.fuzz_roughness, 0.0f, 1.0f);
  auto fuzz_roughen = [&](float r) {
    if (fuzz_w <= 0.0f) return r;
    Vec3 fc = vclamp01(Vec3(m.fuzz_color[0], m.fuzz_color[1], m.fuzz_color[2]));
    float e_fuzz = zeltner_dir_albedo(1.0f, fuzz_r);
    float r_f = clampf(luminance(fc * e_fuzz), 0.0f, 1.0f);
    float rough = std::pow(fmin_num(powi(r, 4) + 2.0f * powi(r_f, 4), 1.0f), 0.25f);
    return lerp(r, rough, fuzz_w);
  };
  const float coat_rough = fuzz_roughen(clampf(m.coat_roughness, 0.0f, 1.0f));
  const float r_base = clampf(m.specular_roughness, 0.0f, 1.0f);
  const float coat_roughened = std::pow(fmin_num(powi(r_base, 4) + 2.0f * powi(coat_rough, 4), 1.0f), 0.25f);
  const float spec_rough = fuzz_roughen(lerp(r_base, coat_roughened, clampf(m.coat_weight, 0.0f, 1.0f)));

  OpenPbrParams p;
  alpha_xy(spec_rough, m.specular_roughness_anisotropy, &p.specular_alpha_x, &p.specular_alpha_y);
  alpha_xy(coat_rough, m.coat_roughness_anisotropy, &p.coat_alpha_x, &p.coat_alpha_y);
  const float coat_w = clampf(m.coat_weight, 0.0f, 1.0f);
  const Vec3 coat_color = vclamp01(Vec3(m.coat_color[0], m.coat_color[1], m.coat_color[2]));
  // coat_darkening_factor (material/open_pbr.rs:823-858)
  Vec3 darkening(1, 1, 1);
  const float delta = clampf(m.coat_darkening, 0.0f, 1.0f);
  if (!(coat_w <= 0.0f || delta <= 0.0f)) {
    float eta_coat = fmax_num(m.coat_ior, 1.0f);
    float ef = dielectric_fresnel_avg(eta_coat);
    float kr = 1.0f - (1.0f - ef) / (eta_coat * eta_coat);
    float ks = fresnel_dielectric(clampf(std::fabs(wo_local.z), 0.0f, 1.0f), 1.0f, eta_coat);
    float ior = fmax_num(m.specular_ior, 1.0e-4f);
    float eta_s = lerp(ior, ior / eta_coat, coat_w);
    float f0 = powi((eta_s - 1.0f) / (eta_s + 1.0f), 2);
    float fs = clampf(fmax_num(m.specular_weight, 0.0f) * f0, 0.0f, 1.0f);
    float rd = lerp(1.0f, r_base, fs);
    float rb = lerp(rd, r_base, metalness);
    float k = clampf(lerp(ks, kr, rb), 0.0f, 1.0f);
    Vec3 base_weighted = base_color * clampf(m.base_weight, 0.0f, 1.0f);
    Vec3 subsurface = vclamp01(Vec3(m.subsurface_color[0], m.subsurface_color[1], m.subsurface_color[2]));
    // subsurface_weight is forced to 0 when the reference adds the material
    // (OpenPbrMaterial::validate_and_warn, material/open_pbr.rs:301-317).
    Vec3 e_dielec = lerp3(lerp3(base_weighted, subsurface, 0.0f),
                          Vec3::splat(1.0f - f0), clampf(m.transmission_weight, 0.0f, 1.0f));
    Vec3 e_metal = vclamp01(base_weighted * fmax_num(m.specular_weight, 0.0f));
    Vec3 e_base = vclamp01(lerp3(e_dielec, e_metal, metalness));
    Vec3 denom = vmax(Vec3(1, 1, 1) - e_base * (k * coat_color), Vec3::splat(1.0e-4f));
    Vec3 delta_factor = Vec3::splat(fmax_num(1.0f - k, 0.0f)) / denom;
    darkening = vclamp01(lerp3(Vec3(1, 1, 1), delta_factor, coat_w * delta));
  }
  const Vec3 spec_color = vclamp01(Vec3(m.specular_color[0], m.specular_color[1], m.specular_color[2]));
  p.base_color = base_color;
  p.base = clampf(m.base_weight, 0.0f, 1.0f);
  p.specular = fmax_num(m.specular_weight, 0.0f);
  p.specular_color = spec_color;
  p.specular_eta = openpbr_specular_eta(m);
  p.transmission_eta = p.specular_eta;
  p.metalness = metalness;
  p.coat = coat_w;
  p.coat_color = coat_color;
  p.coat_darkening = darkening;
  p.coat_eta = fmax_num(m.coat_ior, 1.0e-4f);
  p.fuzz = fuzz_w;
  p.fuzz_color = vclamp01(Vec3(m.fuzz_color[0], m.fuzz_color[1], m.fuzz_color[2]));
  p.fuzz_roughness = fuzz_r;
  p.transmission = clampf(m.transmission_weight, 0.0f, 1.0f);
  p.transmission_color = vclamp01(Vec3(m.transmission_color[0], m.transmission_color[1], m.transmission_color[2]));
  p.transmission_alpha_x = p.specular_alpha_x;
  p.transmission_alpha_y = p.specular_alpha_y;
  p.thin_walled = m.geometry_thin_walled != 0;
  // thin film (make_bsdf, thin_film_thickness_nm_at: micrometres to nm)
  p.thin_film_weight = clampf(m.thin_film_weight, 0.0f, 1.0f);
  p.thin_film_thickness = m.thin_film_weight <= 0.0f ? 0.0f : fmax_num(m.thin_film_thickness, 0.0f) * 1000.0f;
  p.thin_film_ior = fmax_num(m.thin_film_ior, 1.0e-4f);
  artist_friendly_complex_ior(vclamp01(base_color), vclamp01(spec_color), &p.metal_n, &p.metal_k);
  p.diffuse_roughness = clampf(m.base_diffuse_roughness, 0.0f, 1.0f);
  p.subsurface = 0.0f;
  p.subsurface_color = vclamp01(Vec3(m.subsurface_color[0], m.subsurface_color[1], m.subsurface_color[2]));
  p.front_face = front_face;
  // transmission_dispersion_abbe (material/open_pbr.rs:783-790)
  const float scale = fmax_num(m.transmission_dispersion_scale, 0.0f);
  p.transmission_dispersion_abbe = scale <= 0.0f ? 0.0f : fmax_num(m.transmission_dispersion_abbe_number, 1.0e-6f) / scale;
  return p;
}

}  // namespace orc

// ---- scene-level table cache -------------------------------------------------
#include <map>
#include <memory>
#include <mutex>

namespace orc {
namespace {
std::mutex g_lut_mu;
std::map<uint32_t, std::unique_ptr<DielectricAlbedoLut>> g_da;
std::unique_ptr<ConductorEcLut> g_cec;
std::unique_ptr<DielectricEcLut> g_dec;

const DielectricAlbedoLut* da_for(float eta, int nthreads) {
  eta = sanitize_dielectric_eta(eta);
  uint32_t key;
  std::memcpy(&key, &eta, 4);
  auto& slot = g_da[key];
  if (!slot) {
    slot.reset(new DielectricAlbedoLut());
    slot->build(eta, nthreads);
  }
  return slot.get();
}
}  // namespace

OpenPbrLuts openpbr_luts_for(const OpenPbrDesc& m, int nthreads) {
  std::lock_guard<std::mutex> g(g_lut_mu);
  if (!g_cec) {
    g_cec.reset(new ConductorEcLut());
    g_cec->build(nthreads);
  }
  if (!g_dec) {
    g_dec.reset(new DielectricEcLut());
    g_dec->build(nthreads);
  }
  OpenPbrLuts L;
  L.spec = da_for(openpbr_specular_eta(m), nthreads);
  L.coat = da_for(m.coat_ior, nthreads);
  L.conductor = g_cec.get();
  L.dielectric = g_dec.get();
  return L;
}

}  // namespace orc
