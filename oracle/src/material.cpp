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
  return OpenPbrBsdf{make_openpbr_params(m.openpbr, v.front_face, wo_l), m.luts};
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
    if (!make_bsdf(m, v, wo_l).sample(wo_l, r.u_lobe, r.u_dir, mode, &bs)) return false;
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
    return true;
  }
  return false;  // Emissive: pure emitter
}

bool material_le(const Material& m, Vec3* le) {
  if (m.kind != kEmissive) return false;
  *le = m.color * m.strength;
  return true;
}

}  // namespace orc
