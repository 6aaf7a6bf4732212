// Oracle: thin-film interference (crates/renderer/src/bsdf/thin_film.rs) and
// the artist-friendly complex IOR (bsdf/conductor_complex.rs:132-147).  Test
// infrastructure: the checker of the device's thin-film Fresnel terms.
#include "openpbr.h"

namespace orc {

namespace {

constexpr float kPiF = 3.14159274101257324f;

Vec3 vsqrt0(Vec3 v) {  // thin_film.rs:256-262
  return Vec3(std::sqrt(fmax_num(v.x, 0.0f)), std::sqrt(fmax_num(v.y, 0.0f)), std::sqrt(fmax_num(v.z, 0.0f)));
}

// thin_film.rs:170-183
void fresnel_dielectric_polarized(float cos_i, float eta_i, float eta_t, float r[2], float phi[2]) {
  cos_i = clampf(cos_i, 0.0f, 1.0f);
  float sin_i_sq = fmax_num(1.0f - cos_i * cos_i, 0.0f);
  float sin_t_sq = powi(eta_i / eta_t, 2) * sin_i_sq;
  if (sin_t_sq >= 1.0f) {
    r[0] = r[1] = 1.0f;
    phi[0] = phi[1] = 0.0f;
    return;
  }
  float cos_t = std::sqrt(fmax_num(1.0f - sin_t_sq, 0.0f));
  float r_s = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t);
  float r_p = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t);
  phi[0] = r_s < 0.0f ? kPiF : 0.0f;
  phi[1] = r_p < 0.0f ? kPiF : 0.0f;
  r[0] = std::fabs(r_s);
  r[1] = std::fabs(r_p);
}

// thin_film.rs:196-254 (the p-phase estimate it computes and discards is left out)
void fresnel_complex_polarized(float cos_i, float eta_i, float eta_t, float kappa_t, float out[4]) {
  cos_i = clampf(cos_i, 0.0f, 1.0f);
  float cos_i2 = cos_i * cos_i;
  float sin_i2 = fmax_num(1.0f - cos_i2, 0.0f);
  float eta_r = eta_t / fmax_num(eta_i, 1.0e-6f);
  float kappa_r = kappa_t / fmax_num(eta_i, 1.0e-6f);
  float eta_r2 = eta_r * eta_r, kappa_r2 = kappa_r * kappa_r;
  float inner = eta_r2 - kappa_r2 - sin_i2;
  float radicand = fmax_num(inner * inner + 4.0f * eta_r2 * kappa_r2, 0.0f);
  float a2_plus_b2 = std::sqrt(radicand);
  float a2 = fmax_num(0.5f * (a2_plus_b2 + inner), 0.0f);
  float b2 = fmax_num(0.5f * (a2_plus_b2 - inner), 0.0f);
  float a = std::sqrt(a2);
  float t1 = a2_plus_b2 + cos_i2;
  float t2 = 2.0f * a * cos_i;
  float r_s2 = (t1 - t2) / fmax_num(t1 + t2, 1.0e-12f);
  float t3 = a2_plus_b2 * cos_i2 + sin_i2 * sin_i2;
  float t4 = t2 * sin_i2;
  float r_p2 = r_s2 * (t3 - t4) / fmax_num(t3 + t4, 1.0e-12f);
  out[0] = std::sqrt(fmax_num(r_s2, 0.0f));
  out[1] = std::sqrt(fmax_num(r_p2, 0.0f));
  out[2] = std::atan2(2.0f * std::sqrt(b2) * cos_i, cos_i2 - a2 - b2);
  if (r_p2 > 0.0f) {
    float p_num = 2.0f * cos_i * (std::sqrt(b2) * (eta_r2 + kappa_r2) - 2.0f * a * eta_r * kappa_r);
    float p_den = (eta_r2 + kappa_r2) * (eta_r2 + kappa_r2) * cos_i2 - (a2 + b2);
    out[3] = std::atan2(p_num, p_den);
  } else {
    out[3] = 0.0f;
  }
}

// thin_film.rs:126-168
Vec3 eval_sensitivity(float opd, Vec3 shift) {
  float phase = 2.0f * kPiF * opd * 1.0e-9f;
  Vec3 val(5.4856e-13f, 4.4201e-13f, 5.2481e-13f);
  Vec3 pos(1.6810e+06f, 1.7953e+06f, 2.2084e+06f);
  Vec3 var(4.3278e+09f, 9.3046e+09f, 6.6121e+09f);
  float two_pi = 2.0f * kPiF;
  Vec3 amp = vsqrt0(var * two_pi);
  Vec3 cosines(std::cos(pos.x * phase + shift.x), std::cos(pos.y * phase + shift.y), std::cos(pos.z * phase + shift.z));
  Vec3 exps(std::exp(-phase * phase * var.x), std::exp(-phase * phase * var.y), std::exp(-phase * phase * var.z));
  Vec3 xyz = val * amp * cosines * exps;
  float extra_var = 4.5282e+09f;
  float extra_amp = std::sqrt(two_pi * extra_var);
  float extra_cos = std::cos(2.2399e+06f * phase + shift.x);
  float extra_exp = std::exp(-extra_var * phase * phase);
  xyz.x += 9.7470e-14f * extra_amp * extra_cos * extra_exp;
  xyz = Vec3(xyz.x / 1.0685e-7f, xyz.y / 1.0685e-7f, xyz.z / 1.0685e-7f);
  // XYZ_TO_REC709 (glam Mat3 columns) * xyz
  Vec3 c0(3.2404542f, -0.969266f, 0.0556434f), c1(-1.5371385f, 1.8750108f, -0.2040259f),
      c2(-0.4985314f, 0.041556f, 1.0572252f);
  Vec3 res = c0 * xyz.x;
  res = res + c1 * xyz.y;
  res = res + c2 * xyz.z;
  return res;
}

// thin_film.rs:47-124
Vec3 thin_film_inner(float cos_theta_i, float eta_outside, float eta_film, Vec3 n_base, Vec3 k_base,
                     float thickness_nm) {
  float cos1 = clampf(cos_theta_i, 0.0f, 1.0f);
  eta_outside = fmax_num(eta_outside, 1.0e-3f);
  eta_film = fmax_num(eta_film, 1.0e-3f);
  float eta_ratio = eta_outside / eta_film;
  float sin1_sq = fmax_num(1.0f - cos1 * cos1, 0.0f);
  float sin2_sq = eta_ratio * eta_ratio * sin1_sq;
  if (sin2_sq >= 1.0f) return Vec3(1, 1, 1);
  float cos2 = std::sqrt(fmax_num(1.0f - sin2_sq, 0.0f));
  float r12[2], phi12[2];
  fresnel_dielectric_polarized(cos1, eta_outside, eta_film, r12, phi12);
  float phi21[2] = {kPiF - phi12[0], kPiF - phi12[1]};
  float r12_sq[2] = {r12[0] * r12[0], r12[1] * r12[1]};
  float t121_sq[2] = {fmax_num(1.0f - r12_sq[0], 0.0f), fmax_num(1.0f - r12_sq[1], 0.0f)};
  float o[3][4];
  fresnel_complex_polarized(cos2, eta_film, n_base.x, k_base.x, o[0]);
  fresnel_complex_polarized(cos2, eta_film, n_base.y, k_base.y, o[1]);
  fresnel_complex_polarized(cos2, eta_film, n_base.z, k_base.z, o[2]);
  Vec3 r23_s(o[0][0], o[1][0], o[2][0]), r23_p(o[0][1], o[1][1], o[2][1]);
  Vec3 phi23_s(o[0][2], o[1][2], o[2][2]), phi23_p(o[0][3], o[1][3], o[2][3]);
  Vec3 r23_s_sq = r23_s * r23_s, r23_p_sq = r23_p * r23_p;
  float opd = 2.0f * eta_film * thickness_nm * cos2;
  Vec3 phi2_s = Vec3::splat(phi21[0]) + phi23_s, phi2_p = Vec3::splat(phi21[1]) + phi23_p;
  Vec3 i_s = Vec3::splat(r12_sq[0]), i_p = Vec3::splat(r12_sq[1]);
  Vec3 r_geo_s = vsqrt0(vmax(Vec3::splat(r12_sq[0]) * r23_s_sq, Vec3(0, 0, 0)));
  Vec3 r_geo_p = vsqrt0(vmax(Vec3::splat(r12_sq[1]) * r23_p_sq, Vec3(0, 0, 0)));
  Vec3 cm_s = Vec3::splat(t121_sq[0]) * r23_s_sq /
              vmax(Vec3(1, 1, 1) - Vec3::splat(r12_sq[0]) * r23_s_sq, Vec3::splat(1.0e-6f));
  Vec3 cm_p = Vec3::splat(t121_sq[1]) * r23_p_sq /
              vmax(Vec3(1, 1, 1) - Vec3::splat(r12_sq[1]) * r23_p_sq, Vec3::splat(1.0e-6f));
  i_s += cm_s;
  i_p += cm_p;
  cm_s = Vec3::splat(t121_sq[0]) * r23_s_sq;
  cm_p = Vec3::splat(t121_sq[1]) * r23_p_sq;
  for (int m = 1; m <= 2; ++m) {
    Vec3 s_s = eval_sensitivity((float)m * opd, (float)m * phi2_s);
    Vec3 s_p = eval_sensitivity((float)m * opd, (float)m * phi2_p);
    i_s += 2.0f * cm_s * s_s;
    i_p += 2.0f * cm_p * s_p;
    cm_s = cm_s * r_geo_s;
    cm_p = cm_p * r_geo_p;
  }
  Vec3 r = 0.5f * (i_s + i_p);
  return Vec3(clampf(r.x, 0.0f, 1.0f), clampf(r.y, 0.0f, 1.0f), clampf(r.z, 0.0f, 1.0f));
}

}  // namespace

Vec3 thin_film_dielectric(float cos_i, float eta_outside, float eta_film, float eta_base, float thickness_nm) {
  return thin_film_inner(cos_i, eta_outside, eta_film, Vec3::splat(eta_base), Vec3(0, 0, 0), thickness_nm);
}
Vec3 thin_film_conductor(float cos_i, float eta_outside, float eta_film, Vec3 n, Vec3 k, float thickness_nm) {
  return thin_film_inner(cos_i, eta_outside, eta_film, n, k, thickness_nm);
}

void artist_friendly_complex_ior(Vec3 face, Vec3 edge, Vec3* n_out, Vec3* k_out) {
  Vec3 r(clampf(face.x, 0.0f, 0.999f), clampf(face.y, 0.0f, 0.999f), clampf(face.z, 0.0f, 0.999f));
  Vec3 g = vmin(vmax(edge, Vec3(0, 0, 0)), Vec3(1, 1, 1));
  Vec3 r_sqrt = vsqrt0(r);
  Vec3 one(1, 1, 1);
  Vec3 n_max = (one + r_sqrt) / vmax(one - r_sqrt, Vec3::splat(1.0e-6f));
  Vec3 n_min = (one - r) / (one + r);
  Vec3 n = g * n_min + (one - g) * n_max;
  Vec3 np1 = n + one, nm1 = n - one;
  Vec3 k2 = vmax((np1 * np1 * r - nm1 * nm1) / vmax(one - r, Vec3::splat(1.0e-6f)), Vec3(0, 0, 0));
  *n_out = n;
  *k_out = vsqrt0(k2);
}

}  // namespace orc

extern "C" void orc_thin_film(float cos_i, float eta_outside, float eta_film, const float* n, const float* k,
                              float thickness_nm, float* out3) {
  orc::Vec3 r = orc::thin_film_conductor(cos_i, eta_outside, eta_film, orc::Vec3(n[0], n[1], n[2]),
                                         orc::Vec3(k[0], k[1], k[2]), thickness_nm);
  out3[0] = r.x;
  out3[1] = r.y;
  out3[2] = r.z;
}
