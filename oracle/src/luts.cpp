// Oracle: GGX microfacet math (bsdf/smith_ggx.rs), the dielectric GGX
// reflection/transmission used to build the tables (bsdf/dielectric_ggx.rs,
// no energy-compensation table attached) and the three lookup tables of
// bsdf/directional_albedo.rs with their builders and lookups.
#include <atomic>
#include <thread>

#include "openpbr.h"
#include "render.h"

namespace orc {

namespace {
constexpr float kFracPi2 = 1.57079637050628662f;
constexpr float kUniformHemispherePdf = 1.0f / (2.0f * kPi);

template <class F>
void par_rows(int n, int nthreads, F&& f) {
  if (nthreads <= 1) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> ts;
  for (int t = 0; t < nthreads; ++t)
    ts.emplace_back([&]() {
      for (;;) {
        int i = next.fetch_add(1);
        if (i >= n) break;
        f(i);
      }
    });
  for (auto& t : ts) t.join();
}

uint32_t reverse_bits(uint32_t v) {
  uint32_t r = 0;
  for (int i = 0; i < 32; ++i) r |= ((v >> i) & 1u) << (31 - i);
  return r;
}
// directional_albedo.rs:343-356
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
// directional_albedo.rs:410-412
float cell_center(int index, int resolution) { return ((float)index + 0.5f) / (float)resolution; }

// directional_albedo.rs:388-408
struct AxisLerp {
  int lo, hi;
  float t;
};
AxisLerp axis_lerp(float value, int resolution) {
  if (resolution == 1) return {0, 0, 0.0f};
  float position = clampf(value, 0.0f, 1.0f) * (float)resolution - 0.5f;
  if (position <= 0.0f) return {0, 0, 0.0f};
  int max_index = resolution - 1;
  if (position >= (float)max_index) return {max_index, max_index, 0.0f};
  int lower = (int)std::floor(position);
  return {lower, lower + 1, position - (float)lower};
}

// directional_albedo.rs:358-370
void alpha_xy_from_roughness(float roughness, float anisotropy, float* ax, float* ay) {
  roughness = clampf(roughness, 0.0f, 1.0f);
  anisotropy = clampf(anisotropy, -1.0f, 1.0f);
  float alpha = roughness * roughness;
  float aspect = std::sqrt(1.0f - 0.9f * std::fabs(anisotropy));
  float x, y;
  if (anisotropy >= 0.0f) {
    x = alpha / aspect;
    y = alpha * aspect;
  } else {
    x = alpha * aspect;
    y = alpha / aspect;
  }
  *ax = clampf(x, kMinAlpha, 1.0f);
  *ay = clampf(y, kMinAlpha, 1.0f);
}

// directional_albedo.rs:380-386
float fold_phi(Vec3 w) {
  if (w.x == 0.0f && w.y == 0.0f) return 0.0f;
  return std::atan2(std::fabs(w.y), std::fabs(w.x));
}

// DielectricGgxBsdf (dielectric_ggx.rs) with alpha clamped to MIN_ALPHA and no
// energy-compensation table: the single-scattering reflection eval
// (dielectric_ggx.rs:133-163) and sample_rough (dielectric_ggx.rs:509-588).
float dielectric_reflection_eval(float eta, float ax, float ay, Vec3 wo, Vec3 wi) {
  if (!(wo.z > 0.0f) || eta <= 0.0f) return 0.0f;
  if (!(wo.z * wi.z > 0.0f)) return 0.0f;
  Vec3 wm;
  if (!reflection_half_vector(wo, wi, &wm)) return 0.0f;
  float cos_wo_wm = dot(wo, wm);
  if (cos_wo_wm <= 0.0f) return 0.0f;
  float cos_o = std::fabs(wo.z), cos_i = std::fabs(wi.z);
  if (cos_o <= 0.0f || cos_i <= 0.0f) return 0.0f;
  float d = ggx_d(wm, ax, ay);
  if (d <= 0.0f) return 0.0f;
  float g = ggx_g2(wo, wi, ax, ay);
  if (g <= 0.0f) return 0.0f;
  float f = fresnel_dielectric(cos_wo_wm, 1.0f, eta);
  return d * g * f / (4.0f * cos_o * cos_i);
}

Vec3 refract_about_wm(Vec3 wo, Vec3 wm, float eta, bool* ok) {
  *ok = false;
  float cos_o = dot(wo, wm);
  if (cos_o <= 0.0f) return Vec3();
  float sin2_t = eta * eta * fmax_num(1.0f - cos_o * cos_o, 0.0f);
  if (sin2_t >= 1.0f) return Vec3();
  float cos_t = std::sqrt(fmax_num(1.0f - sin2_t, 0.0f));
  Vec3 wi = normalize_or_zero(-eta * wo + (eta * cos_o - cos_t) * wm);
  if (length_squared(wi) == 0.0f) return Vec3();
  *ok = true;
  return wi;
}

// Returns false for None; *transmitted says which branch was taken.
bool dielectric_sample_rough(float eta, float ax, float ay, Vec3 wo, float uc, Vec2 us, float* weight_x,
                             bool* transmitted) {
  const float eta_rel = 1.0f / eta;  // front face
  Vec3 wm;
  if (!sample_wm_vndf(wo, ax, ay, us, &wm)) return false;
  float cos_wo_wm = dot(wo, wm);
  if (cos_wo_wm <= 0.0f) return false;
  float f = fresnel_dielectric(cos_wo_wm, 1.0f, eta);
  float g1 = ggx_g1(wo, ax, ay);
  if (g1 <= 0.0f) return false;
  float pr = fmax_num(f, 0.0f), pt = fmax_num(1.0f - f, 0.0f);
  float sum = pr + pt;
  if (sum <= 0.0f) return false;
  pr /= sum;
  pt /= sum;
  if (uc < pr) {
    Vec3 wi = reflect_local(wo, wm);
    if (!(wi.z > 0.0f)) return false;
    float g2 = ggx_g2(wo, wi, ax, ay);
    float pdf_wm = pdf_wm_vndf(wo, wm, ax, ay);
    if (pdf_wm <= 0.0f) return false;
    float pdf = pr * pdf_wm / (4.0f * cos_wo_wm);
    if (pdf <= 0.0f) return false;
    *weight_x = f * g2 / (pr * g1);
    *transmitted = false;
    return true;
  }
  bool ok;
  Vec3 wi = refract_about_wm(wo, wm, eta_rel, &ok);
  if (!ok) return false;
  if (wi.z >= 0.0f) return false;
  float cos_wi_wm = dot(wi, wm);
  float den = cos_wi_wm + eta_rel * cos_wo_wm;
  if (std::fabs(den) < 1.0e-6f) return false;
  float g2 = ggx_g2(wo, wi, ax, ay);
  float pdf_wm = pdf_wm_vndf(wo, wm, ax, ay);
  if (pdf_wm <= 0.0f) return false;
  float pdf = pt * pdf_wm * std::fabs(cos_wi_wm) / (den * den);
  if (pdf <= 0.0f) return false;
  float radiance_scale = 1.0f / (eta_rel * eta_rel);
  *weight_x = radiance_scale * (1.0f - f) * g2 / (pt * g1);
  *transmitted = true;
  return true;
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
}  // namespace

// ---- smith_ggx.rs ----------------------------------------------------------
float powi(float x, int n) {
  // llvm.powi with a constant exponent: n == 2 is x * x; otherwise binary
  // exponentiation, multiplying the running result by the running square.
  if (n == 2) return x * x;
  float res = 0.0f, sq = x;
  bool have = false;
  for (unsigned v = (unsigned)n; v; v >>= 1) {
    if (v & 1u) {
      res = have ? res * sq : sq;
      have = true;
    }
    if (v >> 1) sq = sq * sq;
  }
  return have ? res : 1.0f;
}

// math/mod.rs:50-71
float fresnel_dielectric(float cos_i, float eta_i, float eta_t) {
  cos_i = clampf(cos_i, -1.0f, 1.0f);
  if (cos_i < 0.0f) {
    std::swap(eta_i, eta_t);
    cos_i = -cos_i;
  }
  float sin_i = std::sqrt(fmax_num(1.0f - cos_i * cos_i, 0.0f));
  float sin_t = (eta_i / eta_t) * sin_i;
  if (sin_t >= 1.0f) return 1.0f;
  float cos_t = std::sqrt(fmax_num(1.0f - sin_t * sin_t, 0.0f));
  float r_par = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t);
  float r_perp = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t);
  return 0.5f * (r_par * r_par + r_perp * r_perp);
}

Vec3 reflect_local(Vec3 wo, Vec3 wm) { return normalize_or_zero(-wo + 2.0f * dot(wo, wm) * wm); }

bool reflection_half_vector(Vec3 wo, Vec3 wi, Vec3* wm) {
  Vec3 m = normalize_or_zero(wo + wi);
  if (length_squared(m) == 0.0f) return false;
  *wm = m.z < 0.0f ? -m : m;
  return true;
}

float ggx_d(Vec3 wm, float ax, float ay) {
  if (wm.z <= 0.0f) return 0.0f;
  float term = wm.x * wm.x / (ax * ax) + wm.y * wm.y / (ay * ay) + wm.z * wm.z;
  float denom = kPi * ax * ay * term * term;
  return denom <= 0.0f ? 0.0f : 1.0f / denom;
}

float ggx_lambda(Vec3 w, float ax, float ay) {
  float c = std::fabs(w.z);
  if (c <= 0.0f) return kInf;
  float term = 1.0f + (ax * ax * w.x * w.x + ay * ay * w.y * w.y) / (c * c);
  return 0.5f * (-1.0f + std::sqrt(term));
}

float ggx_g1(Vec3 w, float ax, float ay) {
  float l = ggx_lambda(w, ax, ay);
  if (!std::isfinite(l)) return 0.0f;
  return 1.0f / (1.0f + l);
}

float ggx_g2(Vec3 wo, Vec3 wi, float ax, float ay) {
  float lo = ggx_lambda(wo, ax, ay), li = ggx_lambda(wi, ax, ay);
  if (!std::isfinite(lo) || !std::isfinite(li)) return 0.0f;
  return 1.0f / (1.0f + lo + li);
}

float pdf_wm_vndf(Vec3 wo, Vec3 wm, float ax, float ay) {
  if (!(wo.z > 0.0f) || wm.z <= 0.0f) return 0.0f;
  float d = ggx_d(wm, ax, ay);
  float g1 = ggx_g1(wo, ax, ay);
  float c = fmax_num(dot(wo, wm), 0.0f);
  if (d <= 0.0f || g1 <= 0.0f || c <= 0.0f) return 0.0f;
  return d * g1 * c / wo.z;
}

bool sample_wm_vndf(Vec3 wo, float ax, float ay, Vec2 us, Vec3* out) {
  if (wo.z <= 0.0f) return false;
  ax = fmax_num(ax, kMinAlpha);
  ay = fmax_num(ay, kMinAlpha);
  Vec3 wo_std = normalize_or_zero(Vec3(ax * wo.x, ay * wo.y, wo.z));
  if (length_squared(wo_std) == 0.0f) return false;
  float lensq = wo_std.x * wo_std.x + wo_std.y * wo_std.y;
  Vec3 t1 = lensq > 0.0f ? Vec3(-wo_std.y, wo_std.x, 0.0f) / std::sqrt(lensq) : Vec3(1, 0, 0);
  Vec3 t2 = cross(wo_std, t1);
  float r = std::sqrt(clampf(us.x, 0.0f, 1.0f));
  float phi = kTau * us.y;
  float p1 = r * std::cos(phi);
  float p2 = r * std::sin(phi);
  float s = 0.5f * (1.0f + wo_std.z);
  p2 = (1.0f - s) * std::sqrt(fmax_num(1.0f - p1 * p1, 0.0f)) + s * p2;
  Vec3 nh = p1 * t1 + p2 * t2 + std::sqrt(fmax_num(1.0f - p1 * p1 - p2 * p2, 0.0f)) * wo_std;
  Vec3 wm = normalize_or_zero(Vec3(ax * nh.x, ay * nh.y, fmax_num(nh.z, 0.0f)));
  if (length_squared(wm) == 0.0f || wm.z <= 0.0f) return false;
  *out = wm;
  return true;
}

bool sample_wm_bounded_vndf(Vec3 wo, float ax, float ay, Vec2 us, Vec3* out) {
  if (wo.z <= 0.0f) return false;
  ax = fmax_num(ax, kMinAlpha);
  ay = fmax_num(ay, kMinAlpha);
  Vec3 wo_std = normalize_or_zero(Vec3(ax * wo.x, ay * wo.y, wo.z));
  if (length_squared(wo_std) == 0.0f) return false;
  float phi = kTau * us.x;
  float a = clampf(fmin_num(ax, ay), 0.0f, 1.0f);
  float s = 1.0f + std::sqrt(wo.x * wo.x + wo.y * wo.y);
  float a2 = a * a, s2 = s * s;
  float k = (1.0f - a2) * s2 / (s2 + a2 * wo.z * wo.z);
  float lower = wo.z > 0.0f ? -k * wo_std.z : -wo_std.z;
  float z = std::fma(lower, us.y, 1.0f - us.y);
  float sin_theta = std::sqrt(clampf(1.0f - z * z, 0.0f, 1.0f));
  Vec3 o_std(sin_theta * std::cos(phi), sin_theta * std::sin(phi), z);
  Vec3 wm_std = wo_std + o_std;
  Vec3 wm = normalize_or_zero(Vec3(ax * wm_std.x, ay * wm_std.y, wm_std.z));
  if (length_squared(wm) == 0.0f || wm.z <= 0.0f) return false;
  *out = wm;
  return true;
}

float pdf_wm_bounded_vndf(Vec3 wo, Vec3 wm, float ax, float ay) {
  if (wo.z <= 0.0f || wm.z <= 0.0f) return 0.0f;
  ax = fmax_num(ax, kMinAlpha);
  ay = fmax_num(ay, kMinAlpha);
  float a = clampf(fmin_num(ax, ay), 0.0f, 1.0f);
  float s = 1.0f + std::sqrt(wo.x * wo.x + wo.y * wo.y);
  float a2 = a * a, s2 = s * s;
  float k = (1.0f - a2) * s2 / (s2 + a2 * wo.z * wo.z);
  float t = std::sqrt(ax * ax * wo.x * wo.x + ay * ay * wo.y * wo.y + wo.z * wo.z);
  float denom = k * wo.z + t;
  if (denom <= 0.0f) return 0.0f;
  return 2.0f * ggx_d(wm, ax, ay) * fmax_num(dot(wo, wm), 0.0f) / denom;
}

// math/mod.rs:26-36
Vec3 sample_cosine_hemisphere(Vec2 us) {
  float r = std::sqrt(clampf(us.x, 0.0f, 1.0f));
  float phi = kTau * us.y;
  float dx = r * std::cos(phi), dy = r * std::sin(phi);
  float z = std::sqrt(fmax_num(1.0f - (dx * dx + dy * dy), 0.0f));
  return Vec3(dx, dy, z);
}

float sanitize_dielectric_eta(float eta) { return (std::isfinite(eta) && eta > 0.0f) ? eta : 1.5f; }

// ---- DielectricGgxDirectionalAlbedoLut (directional_albedo.rs:134-257, 292-341)
void DielectricAlbedoLut::build(float eta_in, int nthreads) {
  eta = sanitize_dielectric_eta(eta_in);
  Vec3 dirs[64];
  for (int i = 0; i < 64; ++i) {
    float u = ((float)i + 0.5f) / 64.0f;
    float v = radical_inverse_vdc((uint32_t)i);
    float z = clampf(u, 0.0f, 1.0f);
    float r = std::sqrt(fmax_num(1.0f - z * z, 0.0f));
    float phi = kTau * v;
    dirs[i] = Vec3(r * std::cos(phi), r * std::sin(phi), z);
  }
  values.assign(kDaLen, 0.0f);
  const float e = eta;
  par_rows(kDaCos * kDaPhi, nthreads, [&](int row) {
    const int ic = row / kDaPhi, ip = row % kDaPhi;
    float sqrt_cos = cell_center(ic, kDaCos);
    float cos_theta = sqrt_cos * sqrt_cos;
    float sin_theta = std::sqrt(fmax_num(1.0f - cos_theta * cos_theta, 0.0f));
    float phi = cell_center(ip, kDaPhi) * kFracPi2;
    Vec3 wo(sin_theta * std::cos(phi), sin_theta * std::sin(phi), cos_theta);
    for (int ir = 0; ir < kDaRough; ++ir)
      for (int ia = 0; ia < kDaAniso; ++ia) {
        float roughness = cell_center(ir, kDaRough);
        float anisotropy = 2.0f * cell_center(ia, kDaAniso) - 1.0f;
        float ax, ay;
        alpha_xy_from_roughness(roughness, anisotropy, &ax, &ay);
        float val;
        if (!(wo.z > 0.0f)) {
          val = 0.0f;
        } else if (fmax_num(ax, ay) < kSmoothAlpha) {
          val = fresnel_dielectric(clampf(wo.z, 0.0f, 1.0f), 1.0f, e);
        } else {
          ax = fmax_num(ax, kMinAlpha);
          ay = fmax_num(ay, kMinAlpha);
          float sum = 0.0f;
          for (int k = 0; k < 64; ++k)
            sum += dielectric_reflection_eval(e, ax, ay, wo, dirs[k]) * fmax_num(dirs[k].z, 0.0f) /
                   kUniformHemispherePdf;
          val = clampf(sum / 64.0f, 0.0f, 1.0f);
        }
        values[((size_t)(ic * kDaPhi + ip) * kDaRough + ir) * kDaAniso + ia] = val;
      }
  });
}

float DielectricAlbedoLut::lookup(Vec3 w, float roughness, float anisotropy) const {
  if (w.z <= 0.0f) return 0.0f;
  roughness = clampf(roughness, 0.0f, 1.0f);
  anisotropy = clampf(anisotropy, -1.0f, 1.0f);
  float ax, ay;
  alpha_xy_from_roughness(roughness, anisotropy, &ax, &ay);
  if (fmax_num(ax, ay) < kSmoothAlpha) return fresnel_dielectric(clampf(w.z, 0.0f, 1.0f), 1.0f, eta);
  float sqrt_cos = std::sqrt(clampf(w.z, 0.0f, 1.0f));
  float phi = fold_phi(w) / kFracPi2;
  roughness = clampf(roughness, 0.0f, 1.0f);
  float aniso = 0.5f * (anisotropy + 1.0f);
  AxisLerp c = axis_lerp(sqrt_cos, kDaCos), p = axis_lerp(phi, kDaPhi), r = axis_lerp(roughness, kDaRough),
           a = axis_lerp(aniso, kDaAniso);
  const int ci[2] = {c.lo, c.hi}, pi[2] = {p.lo, p.hi}, ri[2] = {r.lo, r.hi}, ai[2] = {a.lo, a.hi};
  const float cw[2] = {1.0f - c.t, c.t}, pw[2] = {1.0f - p.t, p.t}, rw[2] = {1.0f - r.t, r.t},
              aw[2] = {1.0f - a.t, a.t};
  float value = 0.0f;
  for (int x = 0; x < 2; ++x)
    for (int y = 0; y < 2; ++y)
      for (int z = 0; z < 2; ++z)
        for (int q = 0; q < 2; ++q)
          value += cw[x] * pw[y] * rw[z] * aw[q] *
                   values[((size_t)(ci[x] * kDaPhi + pi[y]) * kDaRough + ri[z]) * kDaAniso + ai[q]];
  return clampf(value, 0.0f, 1.0f);
}

// ---- ConductorGgxEnergyCompensationLut (directional_albedo.rs:700-830) -------
void ConductorEcLut::build(int nthreads) {
  Vec2 strata[256];
  for (int i = 0; i < 256; ++i) strata[i] = Vec2(((float)i + 0.5f) / 256.0f, radical_inverse_vdc((uint32_t)i));
  e.assign(kCecCos * kCecRough, 0.0f);
  par_rows(kCecCos * kCecRough, nthreads, [&](int index) {
    int ic = index % kCecCos, ir = index / kCecCos;
    float sqrt_cos = cell_center(ic, kCecCos);
    float cos_theta = sqrt_cos * sqrt_cos;
    float roughness = cell_center(ir, kCecRough);
    float val;
    float alpha = clampf(roughness * roughness, kMinAlpha, 1.0f);
    if (cos_theta <= 0.0f) {
      val = 0.0f;
    } else if (alpha < kSmoothAlpha) {
      val = 1.0f;
    } else {
      float sin_theta = std::sqrt(fmax_num(1.0f - cos_theta * cos_theta, 0.0f));
      Vec3 wo(sin_theta, 0.0f, cos_theta);
      float g1 = ggx_g1(wo, alpha, alpha);
      if (g1 <= 0.0f) {
        val = 0.0f;
      } else {
        float sum = 0.0f;
        for (int k = 0; k < 256; ++k) {
          float term = 0.0f;
          Vec3 wm;
          if (sample_wm_vndf(wo, alpha, alpha, strata[k], &wm)) {
            float c = dot(wo, wm);
            if (!(c <= 0.0f)) {
              Vec3 wi = reflect_local(wo, wm);
              if (!(wi.z <= 0.0f)) term = ggx_g2(wo, wi, alpha, alpha) / g1;
            }
          }
          sum += term;
        }
        val = clampf(sum / 256.0f, 0.0f, 1.0f);
      }
    }
    e[index] = val;
  });
  e_avg.assign(kCecRough, 0.0f);
  for (int ir = 0; ir < kCecRough; ++ir) {
    float weighted = 0.0f;
    for (int ic = 0; ic < kCecCos; ++ic) {
      float sqrt_cos = cell_center(ic, kCecCos);
      float cos_theta = sqrt_cos * sqrt_cos;
      weighted += e[ir * kCecCos + ic] * cos_theta * sqrt_cos;
    }
    e_avg[ir] = clampf(4.0f / (float)kCecCos * weighted, 0.0f, 1.0f);
  }
}

float ConductorEcLut::lookup_e(float cos_theta, float roughness) const {
  cos_theta = clampf(cos_theta, 0.0f, 1.0f);
  roughness = clampf(roughness, 0.0f, 1.0f);
  float sqrt_cos = std::sqrt(cos_theta);
  AxisLerp c = axis_lerp(sqrt_cos, kCecCos), r = axis_lerp(roughness, kCecRough);
  const int ci[2] = {c.lo, c.hi}, ri[2] = {r.lo, r.hi};
  const float cw[2] = {1.0f - c.t, c.t}, rw[2] = {1.0f - r.t, r.t};
  float value = 0.0f;
  for (int x = 0; x < 2; ++x)
    for (int y = 0; y < 2; ++y) value += cw[x] * rw[y] * e[ri[y] * kCecCos + ci[x]];
  return clampf(value, 0.0f, 1.0f);
}

float ConductorEcLut::lookup_e_avg(float roughness) const {
  roughness = clampf(roughness, 0.0f, 1.0f);
  AxisLerp r = axis_lerp(roughness, kCecRough);
  float v = (1.0f - r.t) * e_avg[r.lo] + r.t * e_avg[r.hi];
  return clampf(v, 0.0f, 1.0f);
}

// ---- DielectricGgxEnergyCompensationLut (directional_albedo.rs:871-1023) -----
void DielectricEcLut::build(int nthreads) {
  struct S {
    float uc;
    Vec2 us;
  };
  std::vector<S> smp(4096);
  for (uint32_t i = 0; i < 4096; ++i)
    smp[i] = S{((float)i + 0.5f) / 4096.0f, Vec2(radical_inverse_vdc(i + 1), radical_inverse_base3(i + 1))};
  e.assign(kDecCos * kDecRough * kDecEta, 0.0f);
  par_rows(kDecCos * kDecRough * kDecEta, nthreads, [&](int index) {
    int ic = index % kDecCos, rest = index / kDecCos;
    int ir = rest % kDecRough, ie = rest / kDecRough;
    float sqrt_cos = cell_center(ic, kDecCos);
    float cos_theta = sqrt_cos * sqrt_cos;
    float roughness = cell_center(ir, kDecRough);
    float eta = dec_axis_to_eta(cell_center(ie, kDecEta));
    float val;
    float alpha = clampf(roughness * roughness, kMinAlpha, 1.0f);
    if (cos_theta <= 0.0f || eta <= 0.0f) {
      val = 0.0f;
    } else if (alpha < kSmoothAlpha) {
      val = 1.0f;
    } else {
      float sin_theta = std::sqrt(fmax_num(1.0f - cos_theta * cos_theta, 0.0f));
      Vec3 wo(sin_theta, 0.0f, cos_theta);
      float inv_eta_sq = 1.0f / (eta * eta);
      float a = fmax_num(alpha, kMinAlpha);
      float sum = 0.0f;
      for (int k = 0; k < 4096; ++k) {
        float wx;
        bool tr;
        if (!dielectric_sample_rough(eta, a, a, wo, smp[k].uc, smp[k].us, &wx, &tr)) continue;
        if (!std::isfinite(wx)) continue;
        sum += wx * (tr ? inv_eta_sq : 1.0f);
      }
      val = clampf(sum / 4096.0f, 0.0f, 1.0f);
    }
    e[index] = val;
  });
  e_avg.assign(kDecRough * kDecEta, 0.0f);
  for (int ie = 0; ie < kDecEta; ++ie)
    for (int ir = 0; ir < kDecRough; ++ir) {
      float weighted = 0.0f;
      for (int ic = 0; ic < kDecCos; ++ic) {
        float sqrt_cos = cell_center(ic, kDecCos);
        float cos_theta = sqrt_cos * sqrt_cos;
        weighted += e[(ie * kDecRough + ir) * kDecCos + ic] * cos_theta * sqrt_cos;
      }
      e_avg[ie * kDecRough + ir] = clampf(4.0f / (float)kDecCos * weighted, 0.0f, 1.0f);
    }
}

float DielectricEcLut::lookup_e(float cos_theta, float roughness, float eta) const {
  cos_theta = clampf(cos_theta, 0.0f, 1.0f);
  roughness = clampf(roughness, 0.0f, 1.0f);
  float sqrt_cos = std::sqrt(cos_theta);
  float eta_axis = dec_eta_to_axis(eta);
  AxisLerp c = axis_lerp(sqrt_cos, kDecCos), r = axis_lerp(roughness, kDecRough), h = axis_lerp(eta_axis, kDecEta);
  const int ci[2] = {c.lo, c.hi}, ri[2] = {r.lo, r.hi}, hi[2] = {h.lo, h.hi};
  const float cw[2] = {1.0f - c.t, c.t}, rw[2] = {1.0f - r.t, r.t}, hw[2] = {1.0f - h.t, h.t};
  float value = 0.0f;
  for (int x = 0; x < 2; ++x)
    for (int y = 0; y < 2; ++y)
      for (int z = 0; z < 2; ++z) value += hw[x] * rw[y] * cw[z] * e[(hi[x] * kDecRough + ri[y]) * kDecCos + ci[z]];
  return clampf(value, 0.0f, 1.0f);
}

float DielectricEcLut::lookup_e_avg(float roughness, float eta) const {
  roughness = clampf(roughness, 0.0f, 1.0f);
  float eta_axis = dec_eta_to_axis(eta);
  AxisLerp r = axis_lerp(roughness, kDecRough), h = axis_lerp(eta_axis, kDecEta);
  const int ri[2] = {r.lo, r.hi}, hi[2] = {h.lo, h.hi};
  const float rw[2] = {1.0f - r.t, r.t}, hw[2] = {1.0f - h.t, h.t};
  float value = 0.0f;
  for (int x = 0; x < 2; ++x)
    for (int y = 0; y < 2; ++y) value += hw[x] * rw[y] * e_avg[hi[x] * kDecRough + ri[y]];
  return clampf(value, 0.0f, 1.0f);
}

}  // namespace orc
