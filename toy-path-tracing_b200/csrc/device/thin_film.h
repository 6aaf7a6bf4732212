// Thin-film interference on the specular and metal Fresnel terms of OpenPBR
// (crates/renderer/src/bsdf/thin_film.rs): the Airy summation of a film over a
// dielectric or conductor base, two interference orders folded with the
// spectral sensitivity of the camera's CIE XYZ matching (Gaussian fit) and
// converted to linear Rec.709, and the artist-friendly complex IOR of the
// metal base (bsdf/conductor_complex.rs:132-147).
//
// Compiled for the device (the per-vertex Fresnel terms) and for the host (the
// material lowering's 16-sample hemispherical average of the filmed metal
// Fresnel), so one restatement serves both; the arithmetic order is the
// reference's, and the host build does not contract multiply-adds.
#pragma once
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define TPT_HD __host__ __device__ __forceinline__
#else
#define TPT_HD inline
#endif

namespace tpt {
namespace film {

struct F3 {
  float x, y, z;
};
TPT_HD F3 mk(float x, float y, float z) { return F3{x, y, z}; }
TPT_HD F3 spl(float s) { return F3{s, s, s}; }
TPT_HD F3 add(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
TPT_HD F3 sub(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
TPT_HD F3 mul(F3 a, F3 b) { return F3{a.x * b.x, a.y * b.y, a.z * b.z}; }
TPT_HD F3 muls(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
TPT_HD F3 smul(float s, F3 a) { return F3{s * a.x, s * a.y, s * a.z}; }
TPT_HD F3 divv(F3 a, F3 b) { return F3{a.x / b.x, a.y / b.y, a.z / b.z}; }
TPT_HD float fmx(float a, float b) { return a > b ? a : (b > a ? b : (a == a ? a : b)); }
TPT_HD F3 vmx(F3 a, F3 b) { return F3{fmx(a.x, b.x), fmx(a.y, b.y), fmx(a.z, b.z)}; }
TPT_HD float clmp(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
TPT_HD float sqrt0(float v) { return sqrtf(fmx(v, 0.0f)); }  // vec3_sqrt's lane
TPT_HD F3 vsqrt(F3 v) { return F3{sqrt0(v.x), sqrt0(v.y), sqrt0(v.z)}; }
TPT_HD F3 lerp3(F3 a, F3 b, float t) { return add(a, muls(sub(b, a), t)); }

constexpr float kPi = 3.14159274101257324f;

// fresnel_dielectric_polarized (thin_film.rs:170-183): |r_s|, |r_p| and their
// phase shifts (pi where the amplitude is negative)
TPT_HD void dielectric_polarized(float cos_i, float eta_i, float eta_t, float* r, float* phi) {
  cos_i = clmp(cos_i, 0.0f, 1.0f);
  const float sin_i_sq = fmx(1.0f - cos_i * cos_i, 0.0f);
  const float q = eta_i / eta_t;
  const float sin_t_sq = q * q * sin_i_sq;
  if (sin_t_sq >= 1.0f) {
    r[0] = r[1] = 1.0f;
    phi[0] = phi[1] = 0.0f;
    return;
  }
  const float cos_t = sqrtf(fmx(1.0f - sin_t_sq, 0.0f));
  const float r_s = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t);
  const float r_p = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t);
  phi[0] = r_s < 0.0f ? kPi : 0.0f;
  phi[1] = r_p < 0.0f ? kPi : 0.0f;
  r[0] = fabsf(r_s);
  r[1] = fabsf(r_p);
}

// fresnel_complex_polarized (thin_film.rs:196-254): amplitudes and phases of a
// film -> conductor (or dielectric, kappa 0) interface
TPT_HD void complex_polarized(float cos_i, float eta_i, float eta_t, float kappa_t, float* rs_o, float* rp_o,
                              float* ps_o, float* pp_o) {
  cos_i = clmp(cos_i, 0.0f, 1.0f);
  const float cos_i2 = cos_i * cos_i;
  const float sin_i2 = fmx(1.0f - cos_i2, 0.0f);
  const float eta_r = eta_t / fmx(eta_i, 1.0e-6f);
  const float kappa_r = kappa_t / fmx(eta_i, 1.0e-6f);
  const float eta_r2 = eta_r * eta_r;
  const float kappa_r2 = kappa_r * kappa_r;
  const float inner = eta_r2 - kappa_r2 - sin_i2;
  const float radicand = fmx(inner * inner + 4.0f * eta_r2 * kappa_r2, 0.0f);
  const float a2_plus_b2 = sqrtf(radicand);
  const float a2 = fmx(0.5f * (a2_plus_b2 + inner), 0.0f);
  const float b2 = fmx(0.5f * (a2_plus_b2 - inner), 0.0f);
  const float a = sqrtf(a2);
  const float t1 = a2_plus_b2 + cos_i2;
  const float t2 = 2.0f * a * cos_i;
  const float denom_s = fmx(t1 + t2, 1.0e-12f);
  const float r_s2 = (t1 - t2) / denom_s;
  const float t3 = a2_plus_b2 * cos_i2 + sin_i2 * sin_i2;
  const float t4 = t2 * sin_i2;
  const float denom_p = fmx(t3 + t4, 1.0e-12f);
  const float r_p2 = r_s2 * (t3 - t4) / denom_p;
  *rs_o = sqrtf(fmx(r_s2, 0.0f));
  *rp_o = sqrtf(fmx(r_p2, 0.0f));
  const float phi_s_num = 2.0f * sqrtf(b2) * cos_i;
  const float phi_s_den = cos_i2 - a2 - b2;
  *ps_o = atan2f(phi_s_num, phi_s_den);
  if (r_p2 > 0.0f) {
    const float p_num = 2.0f * cos_i * (sqrtf(b2) * (eta_r2 + kappa_r2) - 2.0f * a * eta_r * kappa_r);
    const float p_den = (eta_r2 + kappa_r2) * (eta_r2 + kappa_r2) * cos_i2 - (a2 + b2);
    *pp_o = atan2f(p_num, p_den);
  } else {
    *pp_o = 0.0f;
  }
}

// eval_sensitivity (thin_film.rs:126-168): the XYZ response of one
// interference order with optical path difference `opd` (nm) and phase shifts
// `shift` per channel, in linear Rec.709
TPT_HD F3 sensitivity(float opd, F3 shift) {
  const float phase = 2.0f * kPi * opd * 1.0e-9f;
  const F3 val = mk(5.4856e-13f, 4.4201e-13f, 5.2481e-13f);
  const F3 pos = mk(1.6810e+06f, 1.7953e+06f, 2.2084e+06f);
  const F3 var = mk(4.3278e+09f, 9.3046e+09f, 6.6121e+09f);
  const float two_pi = 2.0f * kPi;
  const F3 amp = vsqrt(muls(var, two_pi));
  const F3 cosines = mk(cosf(pos.x * phase + shift.x), cosf(pos.y * phase + shift.y), cosf(pos.z * phase + shift.z));
  const F3 exps = mk(expf(-phase * phase * var.x), expf(-phase * phase * var.y), expf(-phase * phase * var.z));
  F3 xyz = mul(mul(mul(val, amp), cosines), exps);
  const float extra_var = 4.5282e+09f;
  const float extra_amp = sqrtf(two_pi * extra_var);
  const float extra_cos = cosf(2.2399e+06f * phase + shift.x);
  const float extra_exp = expf(-extra_var * phase * phase);
  xyz.x = xyz.x + 9.7470e-14f * extra_amp * extra_cos * extra_exp;
  xyz = mk(xyz.x / 1.0685e-7f, xyz.y / 1.0685e-7f, xyz.z / 1.0685e-7f);
  // XYZ_TO_REC709 (columns) times xyz, glam's Mat3 * Vec3 order
  F3 res = smul(xyz.x, mk(3.2404542f, -0.969266f, 0.0556434f));
  res = add(smul(xyz.y, mk(-1.5371385f, 1.8750108f, -0.2040259f)), res);
  res = add(smul(xyz.z, mk(-0.4985314f, 0.041556f, 1.0572252f)), res);
  return res;
}

// eval_thin_film_inner (thin_film.rs:47-124)
TPT_HD F3 film_inner(float cos_theta_i, float eta_outside, float eta_film, F3 n_base, F3 k_base, float thickness_nm) {
  const float cos1 = clmp(cos_theta_i, 0.0f, 1.0f);
  eta_outside = fmx(eta_outside, 1.0e-3f);
  eta_film = fmx(eta_film, 1.0e-3f);
  const float eta_ratio = eta_outside / eta_film;
  const float sin1_sq = fmx(1.0f - cos1 * cos1, 0.0f);
  const float sin2_sq = eta_ratio * eta_ratio * sin1_sq;
  if (sin2_sq >= 1.0f) return spl(1.0f);
  const float cos2 = sqrtf(fmx(1.0f - sin2_sq, 0.0f));
  float r12[2], phi12[2];
  dielectric_polarized(cos1, eta_outside, eta_film, r12, phi12);
  const float phi21_s = kPi - phi12[0], phi21_p = kPi - phi12[1];
  const float r12_sq_s = r12[0] * r12[0], r12_sq_p = r12[1] * r12[1];
  const float t121_sq_s = fmx(1.0f - r12_sq_s, 0.0f), t121_sq_p = fmx(1.0f - r12_sq_p, 0.0f);
  float rs[3], rp[3], ps[3], pp[3];
  const float nb[3] = {n_base.x, n_base.y, n_base.z}, kb[3] = {k_base.x, k_base.y, k_base.z};
  for (int c = 0; c < 3; ++c) complex_polarized(cos2, eta_film, nb[c], kb[c], &rs[c], &rp[c], &ps[c], &pp[c]);
  const F3 r23_s = mk(rs[0], rs[1], rs[2]), r23_p = mk(rp[0], rp[1], rp[2]);
  const F3 phi23_s = mk(ps[0], ps[1], ps[2]), phi23_p = mk(pp[0], pp[1], pp[2]);
  const F3 r23_s_sq = mul(r23_s, r23_s), r23_p_sq = mul(r23_p, r23_p);
  const float opd = 2.0f * eta_film * thickness_nm * cos2;
  const F3 phi2_s = add(spl(phi21_s), phi23_s), phi2_p = add(spl(phi21_p), phi23_p);
  F3 i_s = spl(r12_sq_s), i_p = spl(r12_sq_p);
  const F3 r_geo_s = vsqrt(vmx(mul(spl(r12_sq_s), r23_s_sq), spl(0.0f)));
  const F3 r_geo_p = vsqrt(vmx(mul(spl(r12_sq_p), r23_p_sq), spl(0.0f)));
  F3 cm_s = divv(mul(spl(t121_sq_s), r23_s_sq), vmx(sub(spl(1.0f), mul(spl(r12_sq_s), r23_s_sq)), spl(1.0e-6f)));
  F3 cm_p = divv(mul(spl(t121_sq_p), r23_p_sq), vmx(sub(spl(1.0f), mul(spl(r12_sq_p), r23_p_sq)), spl(1.0e-6f)));
  i_s = add(i_s, cm_s);
  i_p = add(i_p, cm_p);
  cm_s = mul(spl(t121_sq_s), r23_s_sq);
  cm_p = mul(spl(t121_sq_p), r23_p_sq);
  for (int m = 1; m <= 2; ++m) {
    const float mf = (float)m;
    const F3 s_s = sensitivity(mf * opd, smul(mf, phi2_s));
    const F3 s_p = sensitivity(mf * opd, smul(mf, phi2_p));
    i_s = add(i_s, mul(smul(2.0f, cm_s), s_s));
    i_p = add(i_p, mul(smul(2.0f, cm_p), s_p));
    cm_s = mul(cm_s, r_geo_s);
    cm_p = mul(cm_p, r_geo_p);
  }
  const F3 result = smul(0.5f, add(i_s, i_p));
  return mk(clmp(result.x, 0.0f, 1.0f), clmp(result.y, 0.0f, 1.0f), clmp(result.z, 0.0f, 1.0f));
}

// eval_thin_film_dielectric / _conductor (thin_film.rs:11-45)
TPT_HD F3 film_dielectric(float cos_i, float eta_out, float eta_film, float eta_base, float thickness_nm) {
  return film_inner(cos_i, eta_out, eta_film, spl(eta_base), spl(0.0f), thickness_nm);
}
TPT_HD F3 film_conductor(float cos_i, float eta_out, float eta_film, F3 n, F3 k, float thickness_nm) {
  return film_inner(cos_i, eta_out, eta_film, n, k, thickness_nm);
}

// artist_friendly_complex_ior (conductor_complex.rs:132-147)
TPT_HD void complex_ior(F3 face_color, F3 edge_color, F3* n_out, F3* k_out) {
  const F3 r = mk(clmp(face_color.x, 0.0f, 0.999f), clmp(face_color.y, 0.0f, 0.999f), clmp(face_color.z, 0.0f, 0.999f));
  const F3 g = mk(clmp(edge_color.x, 0.0f, 1.0f), clmp(edge_color.y, 0.0f, 1.0f), clmp(edge_color.z, 0.0f, 1.0f));
  const F3 r_sqrt = vsqrt(r);
  const F3 one = spl(1.0f);
  const F3 n_max = divv(add(one, r_sqrt), vmx(sub(one, r_sqrt), spl(1.0e-6f)));
  const F3 n_min = divv(sub(one, r), add(one, r));
  const F3 n = add(mul(g, n_min), mul(sub(one, g), n_max));
  const F3 np1 = add(n, one), nm1 = sub(n, one);
  F3 k2 = divv(sub(mul(mul(np1, np1), r), mul(nm1, nm1)), vmx(sub(one, r), spl(1.0e-6f)));
  k2 = vmx(k2, spl(0.0f));
  *n_out = n;
  *k_out = vsqrt(k2);
}

}  // namespace film
}  // namespace tpt
