// Oracle: the material interface with transport modes for the kinds in scope
// (material/mod.rs:33-79 modified_bsdf_eval / _sample_weight,
// material/normalized_lambert.rs:115-190, material/open_pbr.rs:489-603,
// material/emissive.rs:48-94).
#include "render.h"

namespace orc {

namespace {
constexpr float kGeomCosEps = 1.0e-6f;

// material/mod.rs:33-53
Vec3 modified_eval(const Vertex& v, Vec3 wi, Vec3 f, TransportMode mode) {
  if (length_squared(f) == 0.0f) return Vec3(0, 0, 0);
  Vec3 dir = mode == kRadiance ? wi : v.wo;
  float cos_geom = std::fabs(dot(dir, v.ng));
  if (cos_geom <= kGeomCosEps) return Vec3(0, 0, 0);
  return f * (std::fabs(dot(dir, v.ns)) / cos_geom);
}
// material/mod.rs:55-79
Vec3 modified_weight(const Vertex& v, Vec3 wi, Vec3 w, bool delta, TransportMode mode) {
  if (mode == kRadiance || delta || length_squared(w) == 0.0f) return w;
  float cos_wo_geom = std::fabs(dot(v.wo, v.ng));
  float cos_wo_sh = std::fabs(dot(v.wo, v.ns));
  float cos_wi_geom = std::fabs(dot(wi, v.ng));
  float cos_wi_sh = std::fabs(dot(wi, v.ns));
  if (cos_wo_geom <= kGeomCosEps || cos_wi_sh <= kGeomCosEps) return Vec3(0, 0, 0);
  return w * (cos_wo_sh / cos_wo_geom) * (cos_wi_geom / cos_wi_sh);
}
float lambert_bsdf_pdf(Vec3 wo, Vec3 wi) {  // bsdf/normalized_lambert.rs:27-33
  if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
  return fmax_num(wi.z, 0.0f) / kPi;
}
OpenPbrBsdf make_bsdf(const Material& m, const Vertex& v, Vec3 wo_l) {
  OpenPbrBsdf b{make_openpbr_params(m.openpbr, v.front_face, wo_l), m.luts};
  b.p.path_throughput = v.path_throughput;
  b.p.has_lock = v.has_lock;
  b.p.wavelength_lock = v.wavelength_lock;
  return b;
}
}  // namespace

Vec3 material_eval(const Material& m, const Vertex& v, Vec3 wi, TransportMode mode) {
  if (m.kind == kLambert) {
    if (dot(v.wo, v.ng) <= 0.0f || dot(wi, v.ng) <= 0.0f) return Vec3(0, 0, 0);
    Vec3 wo_l = normalize_or_zero(v.frame.to_local(v.wo));
    Vec3 wi_l = normalize_or_zero(v.frame.to_local(wi));
    Vec3 f(0, 0, 0);
    if (!(wo_l.z <= 0.0f || wi_l.z <= 0.0f)) f = m.rho / kPi;
    return modified_eval(v, wi, f, mode);
  }
  if (m.kind == kOpenPbr) {
    if (dot(v.wo, v.ng) <= 0.0f) return Vec3(0, 0, 0);
    Vec3 wo_l = normalize_or_zero(v.frame.to_local(v.wo));
    Vec3 wi_l = normalize_or_zero(v.frame.to_local(wi));
    if (wo_l.z <= 0.0f) return Vec3(0, 0, 0);
    return modified_eval(v, wi, make_bsdf(m, v, wo_l).eval(wo_l, wi_l, mode), mode);
  }
  return Vec3(0, 0, 0);
}

float material_pdf(const Material& m, const Vertex& v, Vec3 wi) {
  if (m.kind == kLambert) {
    if (dot(v.wo, v.ng) <= 0.0f || dot(wi, v.ng) <= 0.0f) return 0.0f;
    return lambert_bsdf_pdf(normalize_or_zero(v.frame.to_local(v.wo)), normalize_or_zero(v.frame.to_local(wi)));
  }
  if (m.kind == kOpenPbr) {
    if (dot(v.wo, v.ng) <= 0.0f) return 0.0f;
    Vec3 wo_l = normalize_or_zero(v.frame.to_local(v.wo));
    Vec3 wi_l = normalize_or_zero(v.frame.to_local(wi));
    if (wo_l.z <= 0.0f) return 0.0f;
    return make_bsdf(m, v, wo_l).pdf(wo_l, wi_l);
  }
  return 0.0f;
}

bool material_sample(const Material& m, const Vertex& v, const MaterialRandoms& r, TransportMode mode,
                     MatSampleOut* s) {
  if (m.kind == kLambert) {
    Vec3 wo_l = normalize_or_zero(v.frame.to_local(v.wo));
    if (wo_l.z <= 0.0f) return false;
    Vec3 wi_l = sample_cosine_hemisphere(r.u_dir);
    float pdf = lambert_bsdf_pdf(wo_l, wi_l);
    if (pdf <= 0.0f) return false;
    Vec3 wi = v.frame.to_world(wi_l);
    s->weight = modified_weight(v, wi, m.rho, false, mode);
    s->wi = wi;
    s->pdf = pdf;
    s->pdf_rev = lambert_bsdf_pdf(wi_l, wo_l);
    s->delta = false;
    return dot(wi, v.ng) > kGeomCosEps;
  }
  if (m.kind == kOpenPbr) {
    if (dot(v.wo, v.ng) <= 0.0f) return false;
    Vec3 wo_l = normalize_or_zero(v.frame.to_local(v.wo));
    if (wo_l.z <= 0.0f) return false;
    BsdfSample bs;
    const float u_extra[4] = {r.u_extra0, r.u_extra1, r.u_extra2, r.u_extra3};
    if (!make_bsdf(m, v, wo_l).sample(wo_l, r.u_lobe, r.u_dir, mode, &bs, u_extra)) return false;
    Vec3 wi = v.frame.to_world(bs.wi);
    // material/open_pbr.rs:523-531: transmission must leave below the geometric
    // surface (delta transmission is kept either way), reflection above it
    if (bs.flags & kTransmission) {
      if (dot(wi, v.ng) >= -kGeomCosEps && !(bs.flags & kDelta)) return false;
    } else if (dot(wi, v.ng) <= kGeomCosEps) {
      return false;
    }
    s->delta = (bs.flags & kDelta) != 0;
    s->weight = modified_weight(v, wi, bs.weight, s->delta, mode);
    s->wi = wi;
    s->pdf = bs.pdf;
    s->pdf_rev = bs.pdf_rev;
    s->has_lock = bs.has_lock;
    s->wavelength_lock = bs.wavelength_lock;
    return true;
  }
  return false;  // Emissive: pure emitter
}

bool may_emit(const Material& m) {
  if (m.kind == kEmissive) return true;
  return m.kind == kOpenPbr && m.openpbr.emission_luminance > 0.0f;
}

float max_emission(const Material& m) {
  if (m.kind == kEmissive) {
    Vec3 e = m.color * m.strength;
    return fmax_num(fmax_num(fmax_num(e.x, e.y), e.z), 0.0f);
  }
  if (m.kind == kOpenPbr && m.openpbr.emission_luminance > 0.0f) {  // material/open_pbr.rs:381-391
    const float* c = m.openpbr.emission_color;
    return fmax_num(fmax_num(c[0], fmax_num(c[1], c[2])) * m.openpbr.emission_luminance * 1.0f, 0.0f);
  }
  return 0.0f;
}

namespace {
// OpenPbrMaterial::emission_exit_tint (material/open_pbr.rs:608-638): the
// emission leaves through the coat (its colour over the refracted path) and
// under the fuzz (what the fuzz does not reflect)
Vec3 openpbr_exit_tint(const OpenPbrDesc& d, const Vertex& v) {
  Vec3 wo_l = normalize_or_zero(v.frame.to_local(v.wo));
  float cos_o = clampf(std::fabs(wo_l.z), 0.0f, 1.0f);
  if (cos_o <= 0.0f) return Vec3(0, 0, 0);
  Vec3 tint(1, 1, 1);
  float cw = clampf(d.coat_weight, 0.0f, 1.0f);
  if (cw > 0.0f) {
    float eta = fmax_num(d.coat_ior, 1.0e-4f);
    float mu_t = fmax_num(std::sqrt(fmax_num(1.0f - (1.0f - cos_o * cos_o) / (eta * eta), 0.0f)), 1.0e-4f);
    Vec3 cc = vmin(vmax(Vec3(d.coat_color[0], d.coat_color[1], d.coat_color[2]), Vec3(0, 0, 0)), Vec3(1, 1, 1));
    float e = 1.0f / mu_t;
    Vec3 trans(std::pow(cc.x, e), std::pow(cc.y, e), std::pow(cc.z, e));
    tint *= Vec3(1, 1, 1) + (trans - Vec3(1, 1, 1)) * cw;
  }
  float fw = clampf(d.fuzz_weight * 1.0f, 0.0f, 1.0f);
  if (fw > 0.0f) {
    float e_fuzz = openpbr_fuzz_albedo(cos_o, clampf(d.fuzz_roughness * 1.0f, 0.0f, 1.0f));
    tint *= Vec3::splat(1.0f + (fmax_num(1.0f - e_fuzz, 0.0f) - 1.0f) * fw);
  }
  return tint;
}
}  // namespace

bool material_le(const Material& m, const Vertex& v, Vec3* le) {
  if (m.kind == kEmissive) {
    *le = m.color * m.strength;
    return true;
  }
  if (m.kind != kOpenPbr) return false;
  const OpenPbrDesc& d = m.openpbr;
  if (d.emission_luminance <= 0.0f) return false;
  if (!d.geometry_thin_walled && !v.front_face) return false;
  Vec3 c(d.emission_color[0], d.emission_color[1], d.emission_color[2]);
  *le = c * Vec3(1, 1, 1) * fmax_num(d.emission_luminance, 0.0f) * openpbr_exit_tint(d, v);
  return true;
}

}  // namespace orc
