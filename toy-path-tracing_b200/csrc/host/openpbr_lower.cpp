// Host lowering of OpenPBR materials (material/open_pbr.rs make_bsdf and its
// helpers; the material-only terms of bsdf/open_pbr.rs) and the host halves of
// the table construction (bsdf/directional_albedo.rs).  Compiled with
// -ffp-contract=off so every f32 operation rounds as in the reference.
#include "openpbr_lower.h"

#include "../device/thin_film.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace tpt {

namespace {
constexpr float kPi = 3.14159274101257324f;
constexpr float kTau = 6.28318548202514648f;
constexpr float kFracPi2 = 1.57079637050628662f;
constexpr float kMinAlpha = 1.0e-4f;
constexpr float kSmoothAlpha = 1.0e-3f;
constexpr float kMsEps = 1.0e-6f;
constexpr float kCos82 = 1.0f / 7.0f;

struct F3 {
  float x, y, z;
};
F3 f3(const float* p) { return F3{p[0], p[1], p[2]}; }
F3 splat(float s) { return F3{s, s, s}; }
F3 operator+(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
F3 operator-(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
F3 operator*(F3 a, F3 b) { return F3{a.x * b.x, a.y * b.y, a.z * b.z}; }
F3 operator*(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
F3 operator*(float s, F3 a) { return F3{s * a.x, s * a.y, s * a.z}; }
F3 operator/(F3 a, float s) { return F3{a.x / s, a.y / s, a.z / s}; }
F3 operator/(F3 a, F3 b) { return F3{a.x / b.x, a.y / b.y, a.z / b.z}; }
float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
F3 vmax(F3 a, F3 b) { return F3{std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
F3 clamp01(F3 v) {
  return F3{std::fmin(std::fmax(v.x, 0.0f), 1.0f), std::fmin(std::fmax(v.y, 0.0f), 1.0f),
            std::fmin(std::fmax(v.z, 0.0f), 1.0f)};
}
void put(float* o, F3 v) {
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
}
float lerp(float a, float b, float t) { return a + (b - a) * t; }
F3 lerp3(F3 a, F3 b, float t) { return a + (b - a) * t; }
float lum(F3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
float sq(float x) { return x * x; }
float pow4(float x) {  // llvm.powi(x, 4)
  float x2 = x * x;
  return x2 * x2;
}
// Constant-argument powi, folded at compile time through the host pow in
// double precision: (1 - 1/7)^n of the F82 terms.
float cos82_pow(int n) { return (float)std::pow((double)(1.0f - kCos82), (double)n); }

float fresnel_dielectric(float cos_i, float eta_i, float eta_t) {  // math/mod.rs:50-71
  cos_i = clampf(cos_i, -1.0f, 1.0f);
  if (cos_i < 0.0f) {
    std::swap(eta_i, eta_t);
    cos_i = -cos_i;
  }
  float sin_i = std::sqrt(std::fmax(1.0f - cos_i * cos_i, 0.0f));
  float sin_t = (eta_i / eta_t) * sin_i;
  if (sin_t >= 1.0f) return 1.0f;
  float cos_t = std::sqrt(std::fmax(1.0f - sin_t * sin_t, 0.0f));
  float r_par = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t);
  float r_perp = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t);
  return 0.5f * (r_par * r_par + r_perp * r_perp);
}

DevLerpAxis axis_lerp(float value, int resolution) {  // directional_albedo.rs:388-408
  float position = clampf(value, 0.0f, 1.0f) * (float)resolution - 0.5f;
  if (position <= 0.0f) return DevLerpAxis{0u, 0u, 0.0f};
  int max_index = resolution - 1;
  if (position >= (float)max_index) return DevLerpAxis{(uint32_t)max_index, (uint32_t)max_index, 0.0f};
  int lower = (int)std::floor(position);
  return DevLerpAxis{(uint32_t)lower, (uint32_t)lower + 1u, position - (float)lower};
}

float dec_eta_to_axis(float eta) {  // directional_albedo.rs:845-853
  const float kMinInv = 1.0f / 3.0f, kMax = 3.0f;
  eta = clampf(eta, kMinInv, kMax);
  if (eta >= 1.0f) return 0.5f + 0.5f * ((eta - 1.0f) / (kMax - 1.0f));
  float inv = 1.0f / eta;
  return 0.5f - 0.5f * ((inv - 1.0f) / (kMax - 1.0f));
}
float dec_axis_to_eta(float t) {  // directional_albedo.rs:855-863
  const float kMax = 3.0f;
  t = clampf(t, 0.0f, 1.0f);
  if (t >= 0.5f) return 1.0f + (t - 0.5f) * 2.0f * (kMax - 1.0f);
  float inv = 1.0f + (0.5f - t) * 2.0f * (kMax - 1.0f);
  return 1.0f / inv;
}
float cec_lookup_e_avg(const float* e_avg, float roughness) {  // directional_albedo.rs:771-777
  roughness = clampf(roughness, 0.0f, 1.0f);
  DevLerpAxis r = axis_lerp(roughness, 64);
  float v = (1.0f - r.t) * e_avg[r.lo] + r.t * e_avg[r.hi];
  return clampf(v, 0.0f, 1.0f);
}
float dec_lookup_e_avg(const float* e_avg, float roughness, float eta) {  // directional_albedo.rs:955-969
  roughness = clampf(roughness, 0.0f, 1.0f);
  DevLerpAxis r = axis_lerp(roughness, 32), h = axis_lerp(dec_eta_to_axis(eta), 32);
  const uint32_t ri[2] = {r.lo, r.hi}, hi[2] = {h.lo, h.hi};
  const float rw[2] = {1.0f - r.t, r.t}, hw[2] = {1.0f - h.t, h.t};
  float value = 0.0f;
  for (int x = 0; x < 2; ++x)
    for (int y = 0; y < 2; ++y) value += hw[x] * rw[y] * e_avg[hi[x] * 32u + ri[y]];
  return clampf(value, 0.0f, 1.0f);
}

float f_avg_dielectric(float eta) {  // bsdf/open_pbr.rs:2183-2191
  if (eta >= 1.0f) return clampf((eta - 1.0f) / (4.08567f + 1.00071f * eta), 0.0f, 1.0f);
  float e = std::fmax(eta, kMsEps);
  float v = 0.997118f + 0.1014f * e - 0.965241f * e * e - 0.130607f * e * e * e;
  return clampf(v, 0.0f, 1.0f);
}

// dielectric_ms_params + ms factor + reflection lobe weights (open_pbr.rs:583-652)
DevMsFace ms_face(float ax, float ay, float eta, bool front, const float* dec_e_avg) {
  DevMsFace f;
  float eta_o = front ? std::fmax(eta, 1.0e-4f) : 1.0f / std::fmax(eta, 1.0e-4f);
  float eta_rel = 1.0f / eta_o;
  float req = std::pow(ax * ay, 0.25f);
  float e_avg_o = dec_lookup_e_avg(dec_e_avg, req, eta_o);
  float om_o = std::fmax(1.0f - e_avg_o, kMsEps);
  float f_avg = clampf(f_avg_dielectric(eta_o), 0.0f, 1.0f);
  float denom = 1.0f - f_avg * std::fmax(1.0f - e_avg_o, 0.0f);
  float factor = clampf(f_avg * f_avg * e_avg_o / std::fmax(denom, kMsEps), 0.0f, 1.0f);
  float ss = clampf(f_avg * e_avg_o, 0.0f, 1.0f);
  float ms = std::fmax(1.0f - e_avg_o, 0.0f) * factor;
  // transmission terms (open_pbr.rs:621-636, 638-646)
  float e_avg_t = dec_lookup_e_avg(dec_e_avg, req, eta_rel);
  float om_t = std::fmax(1.0f - e_avg_t, kMsEps);
  float f_avg_o = f_avg_dielectric(eta_o), f_avg_t = f_avg_dielectric(eta_rel);
  float a = (1.0f - f_avg_o) / om_o;
  float b = (1.0f - f_avg_t) * eta_o * eta_o / om_t;
  float x = a + b > kMsEps ? b / (a + b) : 0.5f;
  f.eta_rel = eta_rel;
  f.one_minus_e_avg_t = om_t;
  f.ratio_r = clampf(1.0f - x * (1.0f - f_avg_o), 0.0f, 1.0f);
  f.trans_ss = clampf(e_avg_o, 0.0f, 1.0f);
  f.trans_ms = std::fmax(1.0f - e_avg_o, 0.0f) * clampf(1.0f - f.ratio_r, 0.0f, 1.0f);
  f.trans_total = std::fmax(f.trans_ss + f.trans_ms, 1.0e-8f);
  f.eta_rel_axis = axis_lerp(dec_eta_to_axis(eta_rel), 32);
  f.eta_o = eta_o;
  f.one_minus_e_avg_o = om_o;
  f.ms_factor = factor;
  f.lobe_ss = ss;
  f.lobe_ms = ms;
  f.lobe_total = std::fmax(ss + ms, 1.0e-8f);
  f.r_axis = axis_lerp(clampf(req, 0.0f, 1.0f), 32);
  f.eta_axis = axis_lerp(dec_eta_to_axis(eta_o), 32);
  return f;
}

void alpha_xy(float roughness, float anisotropy, float* ax, float* ay) {  // material/open_pbr.rs:860-870
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
  float f0 = sq((eta - 1.0f) / (eta + 1.0f));
  float eps = std::sqrt(clampf(w * f0, 0.0f, 0.99999f)) * std::copysign(1.0f, eta - 1.0f);
  return std::fmax((1.0f + eps) / std::fmax(1.0f - eps, 1.0e-6f), 1.0e-4f);
}
float dielectric_fresnel_avg(float eta) {  // material/open_pbr.rs:881-887
  eta = clampf(eta, 1.0f, 3.0f);
  return clampf(
      std::log(std::fmax((10893.0f * eta - 1438.2f) / (-774.4f * eta * eta + 10212.0f * eta + 1.0f), 1.0e-6f)), 0.0f,
      1.0f);
}
float zeltner_albedo(float ndot_v, float roughness) {  // bsdf/open_pbr.rs:2098-2107
  float x = clampf(ndot_v, 0.0f, 1.0f), y = clampf(roughness, 0.01f, 1.0f);
  float s = y * (0.0206607f + 1.58491f * y) / (0.0379424f + y * (1.32227f + y));
  float m = y * (-0.193854f + y * (-1.14885f + y * (1.7932f - 0.95943f * y * y))) / (0.046391f + y);
  float o = y * (0.000654023f + (-0.0207818f + 0.119681f * y) * y) / (1.26264f + y * (-1.92021f + y));
  float q = (x - m) / s;
  return std::exp(-0.5f * (q * q)) / (s * std::sqrt(2.0f * kPi)) + o;
}
float sanitize_eta(float eta) { return (std::isfinite(eta) && eta > 0.0f) ? eta : 1.5f; }

uint32_t reverse_bits(uint32_t v) {
  uint32_t r = 0;
  for (int i = 0; i < 32; ++i) r |= ((v >> i) & 1u) << (31 - i);
  return r;
}
float radical_inverse_vdc(uint32_t bits) { return (float)reverse_bits(bits) * 2.3283064e-10f; }
float radical_inverse_base3(uint32_t n) {
  float q = 0.0f, bk = 1.0f / 3.0f;
  while (n > 0) {
    q += (float)(n % 3u) * bk;
    n /= 3u;
    bk /= 3.0f;
  }
  return q;
}
}  // namespace

float openpbr_spec_table_eta(const tpt_openpbr_desc& m) {
  return sanitize_eta(modulated_eta(std::fmax(m.specular_ior, 1.0e-4f), std::fmax(m.specular_weight, 0.0f)));
}
float openpbr_coat_table_eta(const tpt_openpbr_desc& m) { return sanitize_eta(m.coat_ior); }

void lower_openpbr(const tpt_openpbr_desc& m, const float* spec_da, const float* coat_da, const float* cec_e_avg,
                   const float* dec_e_avg, DevOpenPbr* out) {
  DevOpenPbr d;
  std::memset(&d, 0, sizeof d);
  const F3 base_color = f3(m.base_color);
  const float metalness = clampf(m.base_metalness, 0.0f, 1.0f);
  const float fuzz_w = clampf(m.fuzz_weight, 0.0f, 1.0f);
  const float fuzz_r = clampf(m.fuzz_roughness, 0.0f, 1.0f);
  const F3 fuzz_color = clamp01(f3(m.fuzz_color));
  // effective roughness (material/open_pbr.rs:749-783)
  auto fuzz_roughen = [&](float r) {
    if (fuzz_w <= 0.0f) return r;
    float e_fuzz = zeltner_albedo(1.0f, fuzz_r);
    float r_f = clampf(lum(fuzz_color * e_fuzz), 0.0f, 1.0f);
    float rough = std::pow(std::fmin(pow4(r) + 2.0f * pow4(r_f), 1.0f), 0.25f);
    return lerp(r, rough, fuzz_w);
  };
  const float coat_rough = fuzz_roughen(clampf(m.coat_roughness, 0.0f, 1.0f));
  const float r_base = clampf(m.specular_roughness, 0.0f, 1.0f);
  const float coat_roughened = std::pow(std::fmin(pow4(r_base) + 2.0f * pow4(coat_rough), 1.0f), 0.25f);
  const float coat_w = clampf(m.coat_weight, 0.0f, 1.0f);
  const float spec_rough = fuzz_roughen(lerp(r_base, coat_roughened, coat_w));
  float sax, say, cax, cay;
  alpha_xy(spec_rough, m.specular_roughness_anisotropy, &sax, &say);
  alpha_xy(coat_rough, m.coat_roughness_anisotropy, &cax, &cay);
  const F3 coat_color = clamp01(f3(m.coat_color));
  const F3 spec_color = clamp01(f3(m.specular_color));
  const float specular = std::fmax(m.specular_weight, 0.0f);
  const float spec_eta = modulated_eta(std::fmax(m.specular_ior, 1.0e-4f), specular);
  const float coat_eta = std::fmax(m.coat_ior, 1.0e-4f);
  const float base = clampf(m.base_weight, 0.0f, 1.0f);

  put(d.base_color, base_color);
  d.base = base;
  d.specular = specular;
  put(d.specular_color, spec_color);
  d.spec_ax = sax;
  d.spec_ay = say;
  d.metalness = metalness;
  d.coat = coat_w;
  put(d.coat_color, coat_color);
  d.coat_ax = cax;
  d.coat_ay = cay;
  d.coat_eta = coat_eta;
  d.fuzz = fuzz_w;
  d.fuzz_roughness = clampf(fuzz_r, 0.01f, 1.0f);  // OpenPbrFuzzBsdf::new
  put(d.fuzz_color, fuzz_color);
  d.eon_r = clampf(clampf(m.base_diffuse_roughness, 0.0f, 1.0f), 0.0f, 1.0f);
  d.eon_r_pow01 = std::pow(d.eon_r, 0.1f);

  const bool spec_alpha_smooth = std::fmax(sax, say) < kSmoothAlpha;
  const bool coat_alpha_smooth = std::fmax(cax, cay) < kSmoothAlpha;
  uint32_t flags = 0;
  if (!(coat_w <= 0.0f || coat_alpha_smooth)) flags |= kOpbrCoatRough;
  if (!(metalness <= 0.0f || spec_alpha_smooth)) flags |= kOpbrMetalRough;
  if (!(specular <= 0.0f || spec_alpha_smooth)) flags |= kOpbrSpecRough;

  // albedo tables: roughness proxy and its axis (open_pbr.rs:468-476)
  d.spec_da = spec_da;
  d.coat_da = coat_da;
  d.spec_da_eta = openpbr_spec_table_eta(m);
  d.coat_da_eta = openpbr_coat_table_eta(m);
  const float spec_proxy = clampf(std::sqrt(std::fmax(sax, say)), 0.0f, 1.0f);
  const float coat_proxy = clampf(std::sqrt(std::fmax(cax, cay)), 0.0f, 1.0f);
  auto proxy_smooth = [](float r) {  // alpha_xy_from_roughness(r, 0) < EFFECTIVELY_SMOOTH_ALPHA
    float a = clampf(clampf(r, 0.0f, 1.0f) * clampf(r, 0.0f, 1.0f), kMinAlpha, 1.0f);
    return a < kSmoothAlpha;
  };
  if (proxy_smooth(spec_proxy)) flags |= kOpbrSpecDaSmooth;
  if (proxy_smooth(coat_proxy)) flags |= kOpbrCoatDaSmooth;
  d.spec_da_r = axis_lerp(clampf(spec_proxy, 0.0f, 1.0f), 64);
  d.coat_da_r = axis_lerp(clampf(coat_proxy, 0.0f, 1.0f), 64);

  // metal: F82-tint terms (open_pbr.rs:744-786) and conductor MS (560-582, 788-800)
  const F3 f0 = vmax(base * base_color, splat(0.0f));
  const F3 fs82 = f0 + (splat(1.0f) - f0) * cos82_pow(5);
  const F3 ft82 = spec_color * fs82;
  const float f82_denom = std::fmax(kCos82 * cos82_pow(6), 1.0e-8f);
  put(d.f0, f0);
  put(d.f82_delta, fs82 - ft82);
  d.f82_denom = f82_denom;
  const float cond_req = std::pow(sax * say, 0.25f);
  const float e_avg = clampf(cec_lookup_e_avg(cec_e_avg, cond_req), 0.0f, 1.0f);
  d.cond_ss = e_avg;
  d.cond_ms = std::fmax(1.0f - e_avg, 0.0f);
  d.cond_total = std::fmax(d.cond_ss + d.cond_ms, 1.0e-8f);
  const float e_avg_ms = cec_lookup_e_avg(cec_e_avg, cond_req);  // eval_metal_ms reads it unclamped
  d.cond_one_minus_e_avg = std::fmax(1.0f - e_avg_ms, kMsEps);
  const F3 b = (fs82 - ft82) / f82_denom;
  F3 f_avg = clamp01(specular * (f0 + (splat(1.0f) - f0) / 21.0f - b / 126.0f));
  // thin film (make_bsdf: thickness in nm; artist_friendly_complex_ior of the
  // clamped base and specular colours for the filmed metal)
  const float film_w = clampf(m.thin_film_weight, 0.0f, 1.0f);
  const float film_thick = m.thin_film_weight <= 0.0f ? 0.0f : std::fmax(m.thin_film_thickness, 0.0f) * 1000.0f;
  const float film_ior = std::fmax(m.thin_film_ior, 1.0e-4f);
  film::F3 mn, mk;
  film::complex_ior(film::F3{clamp01(base_color).x, clamp01(base_color).y, clamp01(base_color).z},
                    film::F3{spec_color.x, spec_color.y, spec_color.z}, &mn, &mk);
  const bool has_film = film_w > 0.0f && film_thick > 0.0f;
  if (has_film) {
    // metal_fresnel_avg (open_pbr.rs:818-830): a 16-point average of the
    // filmed metal Fresnel (metal_fresnel, 761-790)
    auto filmed_metal = [&](float c) {
      const float om = 1.0f - clampf(c, 0.0f, 1.0f);
      const float om2 = om * om;
      const F3 fs = f0 + (splat(1.0f) - f0) * (om * (om2 * om2));
      const float cc = clampf(c, 0.0f, 1.0f);
      const float omc = 1.0f - cc, omc2 = omc * omc;
      const float corr = cc * (omc2 * (omc2 * omc2)) / f82_denom;
      const F3 no_film = clamp01(specular * (fs - corr * (fs82 - ft82)));
      film::F3 fl = film::film_conductor(c, 1.0f, film_ior, mn, mk, film_thick);
      if (coat_w > 0.0f)
        fl = film::lerp3(fl, film::film_conductor(c, coat_eta, film_ior, mn, mk, film_thick), clampf(coat_w, 0.0f, 1.0f));
      const F3 f = F3{fl.x, fl.y, fl.z};
      return no_film + (f - no_film) * film_w;
    };
    F3 sum = splat(0.0f);
    for (int i = 0; i < 16; ++i) {
      const float mu = ((float)i + 0.5f) / 16.0f;
      sum = sum + filmed_metal(mu) * (2.0f * mu);
    }
    f_avg = sum / 16.0f;
  }
  {  // compute_conductor_f_ms (open_pbr.rs:2193-2203)
    float om = std::fmax(1.0f - e_avg_ms, 0.0f);
    F3 denom = splat(1.0f) - f_avg * om;
    F3 ds = F3{std::fmax(denom.x, kMsEps), std::fmax(denom.y, kMsEps), std::fmax(denom.z, kMsEps)};
    put(d.cond_f_ms, f_avg * f_avg * e_avg_ms / ds);
  }
  d.cond_r = axis_lerp(clampf(cond_req, 0.0f, 1.0f), 64);

  // dielectric multiple scattering per lobe and face
  for (int face = 0; face < 2; ++face) {
    d.ms[0][face] = ms_face(sax, say, spec_eta, face == 0, dec_e_avg);
    d.ms[1][face] = ms_face(cax, cay, coat_eta, face == 0, dec_e_avg);
  }
  // base_dielectric_fresnel arguments per face (open_pbr.rs:903-931)
  {
    const float eta_ph = spec_eta, eta_pr = spec_eta;
    const float eta_bc = eta_ph / std::fmax(coat_eta, 1.0e-4f);
    const float eta_bcp = eta_pr / std::fmax(coat_eta, 1.0e-4f);
    float a = eta_bc, bb = eta_bcp;
    if (coat_eta > eta_ph) {
      a = 1.0f / std::fmax(eta_bc, 1.0e-4f);
      bb = 1.0f / std::fmax(eta_bcp, 1.0e-4f);
    }
    d.fres[0] = DevFresnelFace{eta_ph, eta_pr, a, bb};
    d.fres[1] = DevFresnelFace{1.0f / eta_ph, 1.0f / eta_pr, 1.0f / std::fmax(a, 1.0e-4f), 1.0f / std::fmax(bb, 1.0e-4f)};
  }
  d.coat_clamped = clampf(coat_w, 0.0f, 1.0f);

  // specular transmission (make_bsdf: transmission alphas = specular alphas,
  // transmission_eta = specular_eta; open_pbr.rs:553-564 thin-wall alphas)
  const float trans = clampf(m.transmission_weight, 0.0f, 1.0f);
  d.transmission = trans;
  put(d.trans_color, clamp01(f3(m.transmission_color)));
  d.trans_eta = spec_eta;
  d.teta_rel[0] = 1.0f / spec_eta;
  d.teta_rel[1] = spec_eta;
  {
    const float eta = std::fmax(spec_eta, 1.0f);
    // powi(eta, 3) expands as eta * (eta * eta), as the oracle's powi does
    const float scale = std::sqrt(std::fmax(3.7f * (eta - 1.0f) * sq(eta - 0.5f) / (eta * (eta * eta)), 0.0f));
    const float s2 = scale * scale;
    d.tw_ax = clampf(sax * s2, kMinAlpha, 1.0f);
    d.tw_ay = clampf(say * s2, kMinAlpha, 1.0f);
  }
  if (trans > 0.0f) flags |= kOpbrTrans;
  if (!(trans <= 0.0f || spec_alpha_smooth)) flags |= kOpbrTransRough;
  if (m.geometry_thin_walled) flags |= kOpbrThinWalled;
  if (has_film) flags |= kOpbrFilm;
  // transmission_dispersion_abbe (material/open_pbr.rs:783-790)
  const float disp_scale = std::fmax(m.transmission_dispersion_scale, 0.0f);
  d.disp_abbe = disp_scale <= 0.0f ? 0.0f : std::fmax(m.transmission_dispersion_abbe_number, 1.0e-6f) / disp_scale;
  if (d.disp_abbe > 0.0f) flags |= kOpbrDisp;
  d.film_w = film_w;
  d.film_thick = film_thick;
  d.film_ior = film_ior;
  d.metal_n[0] = mn.x; d.metal_n[1] = mn.y; d.metal_n[2] = mn.z;
  d.metal_k[0] = mk.x; d.metal_k[1] = mk.y; d.metal_k[2] = mk.z;

  // coat darkening without the view term (material/open_pbr.rs:823-858)
  const float delta = clampf(m.coat_darkening, 0.0f, 1.0f);
  if (!(coat_w <= 0.0f || delta <= 0.0f)) {
    flags |= kOpbrDarkening;
    const float eta_c = std::fmax(m.coat_ior, 1.0f);
    const float ef = dielectric_fresnel_avg(eta_c);
    d.dk_kr = 1.0f - (1.0f - ef) / (eta_c * eta_c);
    const float ior = std::fmax(m.specular_ior, 1.0e-4f);
    const float eta_s = lerp(ior, ior / eta_c, coat_w);
    const float f0s = sq((eta_s - 1.0f) / (eta_s + 1.0f));
    const float fs = clampf(std::fmax(m.specular_weight, 0.0f) * f0s, 0.0f, 1.0f);
    const float rd = lerp(1.0f, r_base, fs);
    d.dk_rb = lerp(rd, r_base, metalness);
    const F3 base_weighted = base_color * base;
    const F3 subsurface = clamp01(f3(m.subsurface_color));
    // subsurface_weight is 0 after OpenPbrMaterial::validate_and_warn
    const F3 e_dielec = lerp3(lerp3(base_weighted, subsurface, 0.0f), splat(1.0f - f0s),
                              clampf(m.transmission_weight, 0.0f, 1.0f));
    const F3 e_metal = clamp01(base_weighted * std::fmax(m.specular_weight, 0.0f));
    put(d.dk_e_base, clamp01(lerp3(e_dielec, e_metal, metalness)));
    d.dk_wd = coat_w * delta;
    d.dk_eta = eta_c;
  }
  d.flags = flags;
  *out = d;
}

void lut_sample_tables(LutSampleTables* t) {
  t->da_dirs.resize(64 * 3);
  for (int i = 0; i < 64; ++i) {  // generate_uniform_hemisphere_samples
    float u = ((float)i + 0.5f) / 64.0f;
    float v = radical_inverse_vdc((uint32_t)i);
    float z = clampf(u, 0.0f, 1.0f);
    float r = std::sqrt(std::fmax(1.0f - z * z, 0.0f));
    float phi = kTau * v;
    t->da_dirs[3 * i] = r * std::cos(phi);
    t->da_dirs[3 * i + 1] = r * std::sin(phi);
    t->da_dirs[3 * i + 2] = z;
  }
  t->da_phi_cs.resize(16 * 2);
  for (int i = 0; i < 16; ++i) {
    float phi = (((float)i + 0.5f) / 16.0f) * kFracPi2;
    t->da_phi_cs[2 * i] = std::cos(phi);
    t->da_phi_cs[2 * i + 1] = std::sin(phi);
  }
  t->cec_u.resize(256);
  t->cec_cs.resize(256 * 2);
  for (uint32_t i = 0; i < 256; ++i) {  // generate_stratified_unit_square_samples_ec
    t->cec_u[i] = ((float)i + 0.5f) / 256.0f;
    float phi = kTau * radical_inverse_vdc(i);
    t->cec_cs[2 * i] = std::cos(phi);
    t->cec_cs[2 * i + 1] = std::sin(phi);
  }
  t->dec_uc.resize(4096);
  t->dec_ux.resize(4096);
  t->dec_cs.resize(4096 * 2);
  for (uint32_t i = 0; i < 4096; ++i) {
    t->dec_uc[i] = ((float)i + 0.5f) / 4096.0f;
    t->dec_ux[i] = radical_inverse_vdc(i + 1);
    float phi = kTau * radical_inverse_base3(i + 1);
    t->dec_cs[2 * i] = std::cos(phi);
    t->dec_cs[2 * i + 1] = std::sin(phi);
  }
}

void conductor_e_avg(const float* e, float* e_avg) {  // directional_albedo.rs:731-742
  for (int ir = 0; ir < 64; ++ir) {
    float weighted = 0.0f;
    for (int ic = 0; ic < 64; ++ic) {
      float sqrt_cos = ((float)ic + 0.5f) / 64.0f;
      float cos_theta = sqrt_cos * sqrt_cos;
      weighted += e[ir * 64 + ic] * cos_theta * sqrt_cos;
    }
    e_avg[ir] = clampf(4.0f / 64.0f * weighted, 0.0f, 1.0f);
  }
}

void dielectric_e_avg(const float* e, float* e_avg) {  // directional_albedo.rs:900-920
  for (int ie = 0; ie < 32; ++ie)
    for (int ir = 0; ir < 32; ++ir) {
      float weighted = 0.0f;
      for (int ic = 0; ic < 32; ++ic) {
        float sqrt_cos = ((float)ic + 0.5f) / 32.0f;
        float cos_theta = sqrt_cos * sqrt_cos;
        weighted += e[(ie * 32 + ir) * 32 + ic] * cos_theta * sqrt_cos;
      }
      e_avg[ie * 32 + ir] = clampf(4.0f / 32.0f * weighted, 0.0f, 1.0f);
    }
}

}  // namespace tpt

extern "C" void tpt_openpbr_defaults(tpt_openpbr_desc* d) {
  if (!d) return;
  std::memset(d, 0, sizeof *d);
  d->base_weight = 1.0f;
  d->base_color[0] = d->base_color[1] = d->base_color[2] = 0.8f;
  d->specular_weight = 1.0f;
  d->specular_color[0] = d->specular_color[1] = d->specular_color[2] = 1.0f;
  d->specular_roughness = 0.3f;
  d->specular_ior = 1.5f;
  d->transmission_color[0] = d->transmission_color[1] = d->transmission_color[2] = 1.0f;
  d->subsurface_color[0] = d->subsurface_color[1] = d->subsurface_color[2] = 0.8f;
  d->fuzz_color[0] = d->fuzz_color[1] = d->fuzz_color[2] = 1.0f;
  d->fuzz_roughness = 0.5f;
  d->coat_color[0] = d->coat_color[1] = d->coat_color[2] = 1.0f;
  d->coat_ior = 1.6f;
  d->coat_darkening = 1.0f;
  d->thin_film_thickness = 0.5f;
  d->thin_film_ior = 1.4f;
  d->emission_color[0] = d->emission_color[1] = d->emission_color[2] = 1.0f;
  d->geometry_opacity = 1.0f;
  d->transmission_dispersion_abbe_number = 20.0f;
}
