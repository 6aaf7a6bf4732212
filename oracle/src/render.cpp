// Oracle: per-sample rendering.  See render.h for the reference files restated.
#include <cstdio>
#include <cstdlib>
#include "render.h"

#include <atomic>
#include <thread>

namespace orc {

namespace {
constexpr float kSgMax = 2.1990233e12f;
constexpr float kMinPos = 1.17549435e-38f;
constexpr float kEps = 1.1920929e-7f;
constexpr float kGeomCosEps = 1.0e-6f;

template <class F>
void par_for(uint64_t n, int nthreads, F&& f) {
  if (nthreads <= 1 || n < 64) {
    for (uint64_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<uint64_t> next{0};
  std::vector<std::thread> ts;
  for (int t = 0; t < nthreads; ++t)
    ts.emplace_back([&]() {
      for (;;) {
        uint64_t i = next.fetch_add(1);
        if (i >= n) break;
        f(i);
      }
    });
  for (auto& t : ts) t.join();
}

Vec3 face_forward(Vec3 n, Vec3 r) { return dot(n, r) < 0.0f ? -n : n; }
Vec3 interp(Vec3 b, Vec3 a0, Vec3 a1, Vec3 a2) { return b.x * a0 + b.y * a1 + b.z * a2; }
float balance(float a, float b) {
  float s = a + b;
  if (a <= 0.0f || s <= 0.0f) return 0.0f;
  return a / s;
}
float luminance(Vec3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

// ---- math/sg.rs -------------------------------------------------------------
float expm1_over_x(float x) {
  float u = std::exp(x);
  if (u == 1.0f) return 1.0f;
  float y = u - 1.0f;
  return std::fabs(x) < 1.0f ? y / std::log(u) : y / x;
}
float sg_erf(float x) {
  if (std::fabs(x) >= 4.0f) return std::copysign(1.0f, x);
  if (std::fabs(x) > 1.0f) {
    const float A1 = 1.6284595f, A2 = 9.156747e-1f, A3 = 1.5432939e-1f, A4 = -3.5175983e-2f, A5 = 5.6679556e-3f,
                A6 = -5.648746e-4f, A7 = 2.5890768e-5f;
    float a = std::fabs(x);
    float y = 1.0f - std::exp2(-((((((((A7 * a + A6) * a + A5) * a + A4) * a + A3) * a + A2) * a + A1) * a)));
    return std::copysign(y, x);
  }
  const float A1 = 1.12837916709551257390f, A2 = -3.76123e-1f, A3 = 1.1279922e-1f, A4 = -2.6703065e-2f,
              A5 = 4.9073556e-3f, A6 = -5.5885315e-4f;
  float x2 = x * x;
  return (((((A6 * x2 + A5) * x2 + A4) * x2 + A3) * x2 + A2) * x2 + A1) * x;
}
float sg_integral(float k) { return 4.0f * kPi * expm1_over_x(-2.0f * k); }
struct SgLobe {
  Vec3 axis;
  float sharpness, log_amplitude;
};
SgLobe sg_product(Vec3 a1, float k1, Vec3 a2, float k2) {
  Vec3 axis = a1 * k1 + a2 * k2;
  float sharp = length(axis);
  Vec3 d = a1 - a2;
  float len2 = dot(d, d);
  float denom = fmax_num(sharp + k1 + k2, kMinPos);
  SgLobe l;
  l.log_amplitude = -k1 * k2 * len2 / denom;
  l.axis = sharp > kMinPos ? axis / sharp : Vec3(0, 0, 1);
  l.sharpness = sharp;
  return l;
}
float upper_cc(float s) {
  if (s <= 0.5f)
    return (((((((-1.0f / 362880.0f) * s + 1.0f / 40320.0f) * s - 1.0f / 5040.0f) * s + 1.0f / 720.0f) * s -
              1.0f / 120.0f) * s + 1.0f / 24.0f) * s - 1.0f / 6.0f) * s + 0.5f;
  return (std::expm1(-s) + s) / (s * s);
}
float lower_cc(float s) {
  float e = std::exp(-s);
  if (s <= 0.5f)
    return e * (((((((((1.0f / 403200.0f) * s - 1.0f / 45360.0f) * s + 1.0f / 5760.0f) * s - 1.0f / 840.0f) * s +
                     1.0f / 144.0f) * s - 1.0f / 30.0f) * s + 1.0f / 8.0f) * s - 1.0f / 3.0f) * s + 0.5f);
  return e * (-std::expm1(-s) - s * e) / (s * s);
}
float sg_cc_product_over_pi(float z, float s) {
  float t = s * std::sqrt(0.5f * ((s + 2.736083f) * s + 17.021297f) / (((s + 4.0100827f) * s + 15.219156f) * s + 76.0879f));
  float tz = t * z;
  const float isp = 0.5641896f;
  float lerp = 0.5f * (z * (1.0f - sg_erf(-tz)) + (1.0f - sg_erf(t))) -
               0.5f * isp * std::exp(-tz * tz) * std::expm1(t * t * (z * z - 1.0f)) / fmax_num(t, kMinPos);
  lerp = clampf(lerp, 0.5f * kEps, 1.0f);
  float lo = lower_cc(s), up = upper_cc(s);
  return 2.0f * (lo + (up - lo) * lerp);
}

// ---- light_tree/lobe.rs:233-283 ---------------------------------------------
bool sg_light_for_node(Vec3 p, Vec3 n, const LightNode& node, float* w, SgLobe* lobe) {
  if (node.flux <= 0.0f) return false;
  Vec3 d = Vec3(node.mu[0], node.mu[1], node.mu[2]) - p;
  float r2 = dot(d, d);
  if (r2 <= 0.0f) return false;
  float inv_r = 1.0f / std::sqrt(r2);
  float cos_below = fmax_num(-(dot(n, d)) * inv_r, 0.0f);
  float bound_var = 0.5f * node.radius * node.radius;
  float sigma2 = node.sigma_s2 * (1.0f - cos_below) + bound_var * cos_below;
  float min_sigma2 = r2 / kSgMax;
  if (sigma2 < min_sigma2) sigma2 = min_sigma2;
  Vec3 axis = d * inv_r;
  float sharp = clampf(r2 / sigma2, 0.0f, kSgMax);
  *lobe = sg_product(-Vec3(node.nu[0], node.nu[1], node.nu[2]), node.lambda, axis, sharp);
  float sg_norm = fmax_num(sg_integral(node.lambda), 1.0e-30f);
  float w_amp = node.flux / (2.0f * kPi * sigma2 * sg_norm);
  *w = w_amp * std::exp(lobe->log_amplitude);
  return std::isfinite(*w) && *w > 0.0f;
}
float diffuse_importance(float rho, Vec3 n, float w, const SgLobe& lobe) {
  if (rho <= 0.0f || w <= 0.0f) return 0.0f;
  float cosine = clampf(dot(lobe.axis, n), -1.0f, 1.0f);
  float integral = sg_cc_product_over_pi(cosine, lobe.sharpness) * kPi;
  return rho * w * integral;
}

struct Query {
  Vec3 p, n;
  float rho;
};
float importance(const Query& q, const LightNode& node) {
  float w;
  SgLobe lobe;
  if (!sg_light_for_node(q.p, q.n, node, &w, &lobe)) return 0.0f;
  return diffuse_importance(q.rho, q.n, w, lobe);
}

// light_tree/traversal.rs:26-92
uint32_t sample_tree(const RenderScene& s, const Query& q, float u, float* pmf) {
  if (s.tree.empty()) return kNoNode;
  u = clampf(u, 0.0f, 1.0f - kEps);
  uint32_t idx = s.root;
  *pmf = 1.0f;
  for (;;) {
    const LightNode& node = s.tree[idx];
    if (node.leaf_instance != kNoNode) return idx;
    const LightNode& L = s.tree[node.left];
    const LightNode& R = s.tree[node.right];
    float il = importance(q, L), ir = importance(q, R);
    float total = il + ir;
    if (total <= 0.0f) {
      float lf = fmax_num(L.flux, 0.0f), rf = fmax_num(R.flux, 0.0f);
      float tf = lf + rf;
      if (tf <= 0.0f) return kNoNode;
      float pl = lf / tf;
      if (u < pl) { u /= fmax_num(pl, kMinPos); *pmf *= pl; idx = node.left; }
      else { u = (u - pl) / fmax_num(1.0f - pl, kMinPos); *pmf *= 1.0f - pl; idx = node.right; }
      continue;
    }
    float pl = il / total;
    if (u < pl) { u /= fmax_num(pl, kMinPos); *pmf *= pl; idx = node.left; }
    else { u = (u - pl) / fmax_num(1.0f - pl, kMinPos); *pmf *= 1.0f - pl; idx = node.right; }
    u = clampf(u, 0.0f, 1.0f - kEps);
  }
}

// light_tree/traversal.rs:97-143
float pdf_for_leaf(const RenderScene& s, const Query& q, uint32_t leaf) {
  if (s.tree.empty() || leaf == kNoNode) return 0.0f;
  if (s.tree[leaf].leaf_instance == kNoNode) return 0.0f;
  float pmf = 1.0f;
  uint32_t child = leaf, parent = s.tree[leaf].parent;
  while (parent != kNoNode) {
    const LightNode& P = s.tree[parent];
    const LightNode& L = s.tree[P.left];
    const LightNode& R = s.tree[P.right];
    float il = importance(q, L), ir = importance(q, R);
    float total = il + ir;
    float pl;
    if (total <= 0.0f) {
      float lf = fmax_num(L.flux, 0.0f), rf = fmax_num(R.flux, 0.0f);
      float tf = lf + rf;
      if (tf <= 0.0f) return 0.0f;
      pl = lf / tf;
    } else {
      pl = il / total;
    }
    pmf *= child == P.left ? pl : 1.0f - pl;
    child = parent;
    parent = P.parent;
  }
  return pmf;
}

// material/normalized_lambert.rs:115-228 + bsdf/normalized_lambert.rs
Vec3 lambert_eval(const Material& m, const Vertex& v, Vec3 wi) {
  if (dot(v.wo, v.ng) <= 0.0f || dot(wi, v.ng) <= 0.0f) return Vec3(0, 0, 0);
  Vec3 wo_l = normalize_or_zero(v.frame.to_local(v.wo));
  Vec3 wi_l = normalize_or_zero(v.frame.to_local(wi));
  Vec3 f(0, 0, 0);
  if (!(wo_l.z <= 0.0f || wi_l.z <= 0.0f)) f = m.rho / kPi;
  // modified_bsdf_eval (material/mod.rs:33-53), radiance transport
  if (length_squared(f) == 0.0f) return Vec3(0, 0, 0);
  float cos_geom = std::fabs(dot(wi, v.ng));
  if (cos_geom <= kGeomCosEps) return Vec3(0, 0, 0);
  return f * (std::fabs(dot(wi, v.ns)) / cos_geom);
}
float lambert_pdf(const Vertex& v, Vec3 wi) {
  if (dot(v.wo, v.ng) <= 0.0f || dot(wi, v.ng) <= 0.0f) return 0.0f;
  Vec3 wo_l = normalize_or_zero(v.frame.to_local(v.wo));
  Vec3 wi_l = normalize_or_zero(v.frame.to_local(wi));
  if (wo_l.z <= 0.0f || wi_l.z <= 0.0f) return 0.0f;
  return fmax_num(wi_l.z, 0.0f) / kPi;
}
struct MatSample {
  Vec3 weight, wi;
  float pdf;
  bool delta;
  bool has_lock = false;  // MaterialSample::wavelength_lock
  float wavelength_lock = 0;
};
bool lambert_sample(const Material& m, const Vertex& v, Vec2 u, MatSample* s) {
  Vec3 wo_l = normalize_or_zero(v.frame.to_local(v.wo));
  if (wo_l.z <= 0.0f) return false;
  float r = std::sqrt(clampf(u.x, 0.0f, 1.0f));
  float phi = kTau * u.y;
  float dx = r * std::cos(phi), dy = r * std::sin(phi);
  float z = std::sqrt(fmax_num(1.0f - (dx * dx + dy * dy), 0.0f));
  Vec3 wi_l(dx, dy, z);
  float pdf = fmax_num(wi_l.z, 0.0f) / kPi;
  if (pdf <= 0.0f) return false;
  s->wi = v.frame.to_world(wi_l);
  s->weight = m.rho;
  s->pdf = pdf;
  s->delta = false;
  return dot(s->wi, v.ng) > kGeomCosEps;
}

// OpenPbrMaterial::sample (material/open_pbr.rs:489-563), radiance transport
// (modified_bsdf_sample_weight leaves the weight unchanged).
bool openpbr_sample(const Material& m, const Vertex& v, const MaterialRandoms& r, MatSample* s) {
  if (dot(v.wo, v.ng) <= 0.0f) return false;
  Vec3 wo_l = normalize_or_zero(v.frame.to_local(v.wo));
  if (wo_l.z <= 0.0f) return false;
  OpenPbrBsdf b{make_openpbr_params(m.openpbr, v.front_face, wo_l), m.luts};
  b.p.path_throughput = v.path_throughput;
  b.p.has_lock = v.has_lock;
  b.p.wavelength_lock = v.wavelength_lock;
  BsdfSample bs;
  const float u_extra[4] = {r.u_extra0, r.u_extra1, r.u_extra2, r.u_extra3};
  if (!b.sample(wo_l, r.u_lobe, r.u_dir, kRadiance, &bs, u_extra)) return false;
  Vec3 wi = v.frame.to_world(bs.wi);
  // material/open_pbr.rs:523-531: transmission below the geometric surface
  // (delta transmission kept either way), reflection above it
  if (bs.flags & kTransmission) {
    if (dot(wi, v.ng) >= -kGeomCosEps && !(bs.flags & kDelta)) return false;
  } else if (dot(wi, v.ng) <= kGeomCosEps) {
    return false;
  }
  s->weight = bs.weight;
  s->wi = wi;
  s->pdf = bs.pdf;
  s->delta = (bs.flags & kDelta) != 0;
  s->has_lock = bs.has_lock;
  s->wavelength_lock = bs.wavelength_lock;
  return true;
}

// the path state a vertex sees (mis.rs:54-55, nee.rs:45-46, pt.rs:41-42)
struct PathLock {
  bool has = false;
  float lambda = 0;
  void stamp(Vertex& v, Vec3 beta) const {
    v.path_throughput = beta;
    v.has_lock = has;
    v.wavelength_lock = lambda;
  }
  void take(const MatSample& bs) {
    if (bs.has_lock) {
      has = true;
      lambda = bs.wavelength_lock;
    }
  }
};

Vec3 offset_origin(Vec3 p, Vec3 ng, Vec3 d) {
  Vec3 n = dot(d, ng) >= 0.0f ? ng : -ng;
  return p + 1.0e-4f * n;
}

struct LiSample {
  Vec3 radiance, wi;
  float pdf, distance;
  int inst, tri;
};

// light/area.rs:12-56 with Scene::sample_triangle_point (scene/mod.rs:620-635)
bool sample_li_triangle(const RenderScene& s, int inst, int tri, Vec3 p_ref, Vec2 us, LiSample* out) {
  Vec3 p[3];
  s.triangle_world(inst, tri, p);
  float su0 = std::sqrt(clampf(us.x, 0.0f, 1.0f));
  float u1 = clampf(us.y, 0.0f, 1.0f);
  Vec3 b(1.0f - su0, u1 * su0, (1.0f - u1) * su0);
  Vec3 pt = interp(b, p[0], p[1], p[2]);
  float area = 0.5f * length(cross(p[1] - p[0], p[2] - p[0]));
  float pdf_area = area > 0.0f ? 1.0f / area : 0.0f;
  if (pdf_area <= 0.0f) return false;
  Vec3 to_light = pt - p_ref;
  float d2 = length_squared(to_light);
  if (d2 <= 0.0f) return false;
  float dist = std::sqrt(d2);
  Vec3 wi = to_light / dist;
  const Material& lm = s.mat_of(inst);
  if (!may_emit(lm)) return false;
  Vertex lv = s.shading_vertex(inst, tri, b, wi);
  Vec3 le;
  if (!material_le(lm, lv, &le)) return false;
  float cos_light = fmax_num(dot(lv.ng, -wi), 0.0f);
  if (cos_light <= 0.0f) return false;
  out->radiance = le;
  out->wi = wi;
  out->pdf = pdf_area * d2 / cos_light;
  out->distance = dist;
  out->inst = inst;
  out->tri = tri;
  return true;
}

bool closest(const RenderScene& s, Vec3 o, Vec3 d, SceneHit* h, AuxRng* aux) {
  Ray r;
  r.origin = o;
  r.direction = d;
  return s.geo.closest_hit(r, h, nullptr, aux);
}

// point::sample_li (light/point.rs:32-50)
bool sample_li_point(const PointLight& l, Vec3 p_ref, LiSample* out) {
  Vec3 to_light = l.position - p_ref;
  float d2 = length_squared(to_light);
  if (d2 <= 0.0f) return false;
  float dist = std::sqrt(d2);
  out->wi = to_light / dist;
  out->radiance = l.color * (l.intensity / (4.0f * kPi * d2));
  out->pdf = 1.0f;
  out->distance = dist;
  out->inst = out->tri = -1;
  return true;
}
// math/mod.rs:180-183
float smoothstep(float e0, float e1, float x) {
  float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
// spot::sample_li (light/spot.rs:51-76)
bool sample_li_spot(const SpotLight& l, Vec3 p_ref, LiSample* out) {
  Vec3 to_light = l.position - p_ref;
  float d2 = length_squared(to_light);
  if (d2 <= 0.0f) return false;
  float dist = std::sqrt(d2);
  Vec3 wi = to_light / dist;
  float falloff = smoothstep(l.cos_total_width, l.cos_falloff_start, dot(-wi, l.direction));
  if (falloff <= 0.0f) return false;
  out->wi = wi;
  out->radiance = l.color * (l.intensity * falloff / (2.0f * kTau * d2));
  out->pdf = 1.0f;
  out->distance = dist;
  out->inst = out->tri = -1;
  return true;
}

// LightSampler::sample_category (light/mod.rs:197-212); -2 when empty
int sample_category(const RenderScene& s, float u, float* pmf) {
  if (s.cat_kind.empty()) return -2;
  u = clampf(u, 0.0f, 1.0f);
  size_t n = 0;
  for (size_t k = 0; k < s.cat_cdf.size(); ++k)
    if (s.cat_cdf[k] <= u) n = k + 1;
  size_t idx = std::min(n == 0 ? (size_t)0 : n - 1, s.cat_kind.size() - 1);
  *pmf = s.cat_pmf[idx];
  return s.cat_kind[idx];
}

// integrator/mis.rs:145-210 with sample_light_mis_compensated_lazy
// (light/mod.rs:296-340): the tree category needs a light-tree query (the
// diffuse material is the only one in scope that builds one); directional
// lights serve every scattering material.  Delta lights take no MIS weight.
// wi_out (optional) receives the sampled light direction.
Vec3 direct_light_impl(const RenderScene& s, const Material& m, const Vertex& v, const VertexRandoms& rnd,
                       Vec3* wi_out, int mode, AuxRng* aux) {
  const bool non_area_only = mode == kDirectBdptNonArea, nee = mode == kDirectNee;
  float cat_pmf = 0.0f;
  int cat = sample_category(s, rnd.light.u_category, &cat_pmf);
  if (cat == -2) return Vec3(0, 0, 0);  // no category
  LiSample li;
  float sel;
  bool delta = true;
  if (cat == -1) {
    if (m.kind != kLambert) return Vec3(0, 0, 0);
    Query q;
    q.rho = luminance(m.rho);
    if (q.rho <= 0.0f) return Vec3(0, 0, 0);
    q.p = v.p;
    q.n = v.ns;
    float leaf_pmf;
    uint32_t leaf = sample_tree(s, q, rnd.light.u_tree, &leaf_pmf);
    if (leaf == kNoNode) return Vec3(0, 0, 0);
    const uint32_t li_inst = s.tree[leaf].leaf_instance, li_tri = s.tree[leaf].leaf_triangle;
    if (li_inst == kLeafPoint) {
      if (!sample_li_point(s.points[li_tri], v.p, &li)) return Vec3(0, 0, 0);
    } else if (li_inst == kLeafSpot) {
      if (!sample_li_spot(s.spots[li_tri], v.p, &li)) return Vec3(0, 0, 0);
    } else {
      // bdpt.rs:424-426: BDPT's camera vertices take no area-light samples here
      if (non_area_only) return Vec3(0, 0, 0);
      if (!sample_li_triangle(s, (int)li_inst, (int)li_tri, v.p, rnd.light.u_surface, &li)) return Vec3(0, 0, 0);
      delta = false;
    }
    sel = cat_pmf * leaf_pmf;
  } else if (cat == -3) {
    // environment::sample_li_mis_compensated (light/environment.rs:258-273);
    // the NEE integrator's sample_light draws from the plain distribution
    EnvSample es;
    const bool ok = nee ? s.env.sample(rnd.light.u_surface.x, rnd.light.u_surface.y, &es)
                        : s.env.sample_mis_compensated(rnd.light.u_surface.x, rnd.light.u_surface.y, &es);
    if (!ok) return Vec3(0, 0, 0);
    if (es.pdf <= 0.0f) return Vec3(0, 0, 0);
    li.radiance = es.radiance;
    li.wi = es.direction;
    li.pdf = es.pdf;
    li.distance = INFINITY;
    li.inst = li.tri = -1;
    delta = false;
    sel = cat_pmf;
  } else {
    // directional::sample_li (light/directional.rs:33-42)
    const DirLight& d = s.dirs[cat];
    li.radiance = d.color * d.intensity;
    li.wi = -d.direction;
    li.pdf = 1.0f;
    li.distance = INFINITY;
    li.inst = li.tri = -1;
    sel = cat_pmf;
  }
  if (li.pdf <= 0.0f || sel <= 0.0f) return Vec3(0, 0, 0);
  Vec3 f;
  float bsdf_pdf = 0.0f;
  if (delta || nee) {  // nee.rs:140: Material::eval, no MIS weight
    f = m.kind == kLambert ? lambert_eval(m, v, li.wi) : material_eval(m, v, li.wi, kRadiance);
  } else if (m.kind == kLambert) {
    f = lambert_eval(m, v, li.wi);
    bsdf_pdf = length_squared(f) == 0.0f ? 0.0f : lambert_pdf(v, li.wi);
  } else {  // Material::eval_pdf (material/mod.rs:351-370): the environment at an OpenPBR vertex
    f = material_eval(m, v, li.wi, kRadiance);
    bsdf_pdf = length_squared(f) == 0.0f ? 0.0f : material_pdf(m, v, li.wi);
  }
  if (length_squared(f) == 0.0f) return Vec3(0, 0, 0);
  float cos_surface = std::fabs(dot(v.ng, li.wi));
  if (cos_surface <= 0.0f) return Vec3(0, 0, 0);
  // unoccluded_ray (integrator/mod.rs:239-265)
  SceneHit h;
  if (closest(s, offset_origin(v.p, v.ng, li.wi), li.wi, &h, aux)) {
    bool visible;
    if (li.inst >= 0) visible = h.instance == li.inst && h.triangle == li.tri;
    else if (std::isinf(li.distance)) visible = false;
    else visible = h.t >= li.distance * (1.0f - 1.0e-3f);
    if (!visible) return Vec3(0, 0, 0);
  }
  float pdf_total = sel * li.pdf;
  if (pdf_total <= 0.0f) return Vec3(0, 0, 0);
  if (wi_out) *wi_out = li.wi;
  if (delta || nee) return li.radiance * f * (cos_surface / pdf_total);
  float mis = balance(pdf_total, bsdf_pdf);
  return li.radiance * f * (cos_surface * mis / pdf_total);
}

// light/mod.rs:416-437 + scene/mod.rs:583-618
float light_pdf_for_hit(const RenderScene& s, const Material& shading, const Vertex& v, const Vertex& lv) {
  if (!s.has_tree || shading.kind != kLambert) return 0.0f;
  Query q;
  q.rho = luminance(shading.rho);
  if (q.rho <= 0.0f) return 0.0f;
  q.p = v.p;
  q.n = v.ns;
  const auto& lo = s.leaf_of[lv.inst];
  uint32_t leaf = lo.empty() ? kNoNode : lo[lv.tri];
  float leaf_pmf = pdf_for_leaf(s, q, leaf);
  if (leaf_pmf <= 0.0f) return 0.0f;
  float area = s.tree[leaf].area;
  if (area <= 0.0f) return 0.0f;
  float pdf_area = 1.0f / area;
  Vec3 to_light = lv.p - v.p;
  float d2 = length_squared(to_light);
  if (d2 <= 0.0f) return 0.0f;
  float dist = std::sqrt(d2);
  Vec3 wi = to_light / dist;
  float cos_light = fmax_num(dot(lv.ng, -wi), 0.0f);
  if (cos_light <= 0.0f) return 0.0f;
  return s.tree_cat_pmf * leaf_pmf * (pdf_area * d2 / cos_light);
}

}  // namespace

Vec3 direct_light(const RenderScene& s, const Material& m, const Vertex& v, const VertexRandoms& rnd, Vec3* wi_out,
                  int mode, AuxRng* aux) {
  return direct_light_impl(s, m, v, rnd, wi_out, mode, aux);
}

// orthonormal_basis.rs:11-56
Frame Frame::from_normal(Vec3 normal) {
  Vec3 n = length_squared(normal) > 0.0f ? normalize(normal) : Vec3(0, 0, 1);
  float sign = std::copysign(1.0f, n.z);
  float a = -1.0f / (sign + n.z);
  float b = n.x * n.y * a;
  Frame f;
  f.t = Vec3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
  f.b = Vec3(b, sign + n.y * n.y * a, -n.y);
  f.n = n;
  return f;
}
Frame Frame::from_normal_and_tangent(Vec3 normal, Vec3 hint) {
  Vec3 n = length_squared(normal) > 0.0f ? normalize(normal) : Vec3(0, 0, 1);
  Vec3 t = normalize_or_zero(hint - dot(hint, n) * n);
  if (length_squared(t) == 0.0f) return from_normal(n);
  Frame f;
  f.b = normalize_or_zero(cross(n, t));
  f.t = normalize_or_zero(cross(f.b, n));
  f.n = n;
  return f;
}

// Material::has_alpha_test and the clamped opacity any_hit compares u with
// (normalized_lambert.rs:85-107, emissive.rs:96-118, material/open_pbr.rs:
// 321-343), untextured: 1 for a material without an alpha test.
float material_alpha(const Material& m) {
  const float o = m.kind == kOpenPbr ? m.openpbr.geometry_opacity : m.opacity;
  return o < 1.0f ? clampf(o, 0.0f, 1.0f) : 1.0f;
}

void RenderScene::finalize() {
  geo.alpha.clear();
  for (size_t i = 0; i < geo.instances.size(); ++i)
    if (material_alpha(materials[geo.instances[i].material_index]) < 1.0f) geo.alpha.resize(geo.instances.size(), 1.0f);
  if (!geo.alpha.empty())
    for (size_t i = 0; i < geo.instances.size(); ++i) geo.alpha[i] = material_alpha(materials[geo.instances[i].material_index]);
  leaf_of.assign(geo.instances.size(), {});
  for (size_t i = 0; i < geo.instances.size(); ++i)
    if (may_emit(materials[geo.instances[i].material_index]))
      leaf_of[i].assign(geo.meshes[geo.instances[i].mesh_index].triangle_count(), kNoNode);
  for (uint32_t k = 0; k < tree.size(); ++k) {
    const uint32_t li = tree[k].leaf_instance;
    if (li == kNoNode || li == kLeafPoint || li == kLeafSpot) continue;
    if (!leaf_of[li].empty()) leaf_of[li][tree[k].leaf_triangle] = k;
  }
  // Scene::register_area_light_triangles (scene/mod.rs:649-684), per instance in order
  area_lights.clear();
  area_light_weight_sum = 0.0f;
  for (size_t i = 0; i < geo.instances.size(); ++i) {
    const Material& m = materials[geo.instances[i].material_index];
    if (!may_emit(m)) continue;
    const float max_em = max_emission(m);
    if (max_em <= 0.0f) continue;
    int ntri = (int)geo.meshes[geo.instances[i].mesh_index].triangle_count();
    for (int t = 0; t < ntri; ++t) {
      Vec3 p[3];
      triangle_world((int)i, t, p);
      float area = 0.5f * length(cross(p[1] - p[0], p[2] - p[0]));
      float weight = area * max_em;
      if (weight <= 0.0f) continue;
      area_light_weight_sum += weight;
      area_lights.push_back(AreaLight{(int32_t)i, t, area, weight, area_light_weight_sum});
    }
  }
  // LightSampler::build_from_scene (light/mod.rs:134-188): Tree, the
  // Environment (by total power), then one category per directional light
  // with luminance(color) * intensity > 0
  float w = tree.empty() ? 0.0f : fmax_num(tree[root].flux, 0.0f);
  has_tree = w > 0.0f;
  std::vector<float> weights;
  cat_kind.clear();
  if (w > 0.0f) {
    cat_kind.push_back(-1);
    weights.push_back(w);
  }
  const float env_w = has_env ? fmax_num(env.total_power(), 0.0f) : 0.0f;
  if (env_w > 0.0f) {
    cat_kind.push_back(-3);
    weights.push_back(env_w);
  }
  for (size_t i = 0; i < dirs.size(); ++i) {
    float dw = fmax_num(luminance(dirs[i].color) * dirs[i].intensity, 0.0f);
    if (dw > 0.0f) {
      cat_kind.push_back((int)i);
      weights.push_back(dw);
    }
  }
  cat_cdf.assign(1, 0.0f);
  float total = 0.0f;
  for (float x : weights) {
    total += x;
    cat_cdf.push_back(total);
  }
  if (total > 0.0f) {
    float inv = 1.0f / total;
    for (float& c : cat_cdf) c *= inv;
  }
  cat_pmf.assign(weights.size(), 0.0f);
  for (size_t k = 0; k < weights.size(); ++k) cat_pmf[k] = total > 0.0f ? weights[k] / total : 0.0f;
  if (!(total > 0.0f)) cat_kind.clear();
  tree_cat_pmf = has_tree && total > 0.0f ? w / total : 0.0f;
  env_cat_pmf = env_w > 0.0f && total > 0.0f ? env_w / total : 0.0f;
}

void RenderScene::triangle_world(int inst, int tri, Vec3* p) const {
  const Instance& I = geo.instances[inst];
  const Mesh& m = geo.meshes[I.mesh_index];
  m.triangle_positions(tri, p);
  for (int k = 0; k < 3; ++k) p[k] = I.local_to_world.transform_point3(p[k]);
}

// scene/mod.rs:471-544 (differentials omitted: nothing in scope reads them)
Vertex RenderScene::shading_vertex(int inst, int tri, Vec3 b, Vec3 incident) const {
  const Instance& I = geo.instances[inst];
  const Mesh& m = geo.meshes[I.mesh_index];
  Vec3 p[3], n[3];
  Vec2 uv[3];
  triangle_world(inst, tri, p);
  for (int k = 0; k < 3; ++k) {
    uint32_t vi = m.indices[3 * (size_t)tri + k];
    n[k] = normalize_or_zero(I.normal_to_world.mul_vec3(m.normals[vi]));
    uv[k] = m.uvs[vi];
  }
  Vertex v;
  v.inst = inst;
  v.tri = tri;
  v.p = interp(b, p[0], p[1], p[2]);
  Vec3 gn = normalize_or_zero(cross(p[1] - p[0], p[2] - p[0]));
  Vec3 sn = normalize_or_zero(interp(b, n[0], n[1], n[2]));
  v.front_face = dot(gn, -incident) >= 0.0f;
  v.ng = face_forward(gn, -incident);
  Vec3 raw_ns = length_squared(sn) > 0.0f ? sn : v.ng;
  v.ns = face_forward(raw_ns, v.ng);
  // compute_surface_partials (math/mod.rs:112-134)
  Vec3 dp1 = p[1] - p[0], dp2 = p[2] - p[0];
  float du1 = uv[1].x - uv[0].x, dv1 = uv[1].y - uv[0].y;
  float du2 = uv[2].x - uv[0].x, dv2 = uv[2].y - uv[0].y;
  float det = du1 * dv2 - dv1 * du2;
  Vec3 dpdu;
  bool ok = false;
  if (!(std::fabs(det) <= 1.0e-8f)) {
    float inv = 1.0f / det;
    dpdu = (dv2 * dp1 - dv1 * dp2) * inv;
    Vec3 dpdv = (-du2 * dp1 + du1 * dp2) * inv;
    ok = !(length_squared(dpdu) == 0.0f || length_squared(dpdv) == 0.0f);
  }
  if (!ok) dpdu = Frame::from_normal(v.ns).t;
  v.frame = Frame::from_normal_and_tangent(v.ns, dpdu);
  v.wo = normalize_or_zero(-incident);
  return v;
}

// emitted_radiance_from_bsdf_sample_infinite (integrator/mis.rs:238-258; in
// BDPT emitted_radiance_from_infinite_hit, bdpt.rs:466-486, with `delta` = count
// the full emission) with pdf_for_environment_hit (light/mod.rs:439-450,
// MIS-compensated), without the path throughput
Vec3 env_escape(const RenderScene& s, Vec3 dir, bool delta, float bsdf_pdf) {
  if (!s.has_env) return Vec3(0, 0, 0);  // infinite_light_le without an environment
  const Vec3 le = s.env.radiance(dir);
  if (le.x == 0.0f && le.y == 0.0f && le.z == 0.0f) return Vec3(0, 0, 0);
  if (delta) return le;
  const float light_pdf = s.env_cat_pmf <= 0.0f ? 0.0f : s.env_cat_pmf * s.env.pdf_mis_compensated(dir);
  return le * balance(bsdf_pdf, light_pdf);
}

// integrator/pt.rs:15-76: BSDF sampling only; every emitter hit and every
// escape counts in full
Vec3 trace_pt(const RenderScene& s, const Ray& ray, const PathSampler& sampler, uint32_t max_depth) {
  Vec3 L(0, 0, 0), beta(1, 1, 1);
  PathLock lock;
  Vec3 ro = ray.origin, rd = ray.direction;
  for (uint32_t depth = 0; depth < max_depth; ++depth) {
    VertexRandoms rnd = sampler.path_vertex_randoms(depth);
    AuxRng aux(rnd.aux_rng_seed);  // pt.rs:29-33: the ray arriving at this depth draws from it
    SceneHit h;
    if (!closest(s, ro, rd, &h, &aux)) {
      if (s.has_env) L += beta * s.env.radiance(rd);  // infinite_light_le
      break;
    }
    Vertex v = s.shading_vertex(h.instance, h.triangle, h.bary, rd);
    const Material& m = s.mat_of(h.instance);
    lock.stamp(v, beta);
    Vec3 le;
    if (material_le(m, v, &le)) L += beta * le;
    MatSample bs;
    bool ok = m.kind == kOpenPbr ? openpbr_sample(m, v, rnd.material, &bs)
              : m.kind == kLambert ? lambert_sample(m, v, rnd.material.u_dir, &bs)
                                   : false;  // the pure emitter samples nothing
    if (!ok) break;
    beta *= bs.weight;
    lock.take(bs);
    if (depth + 1 >= 4) {
      float q = clampf(max_element(beta), 0.05f, 1.0f);
      if (rnd.u_rr > q) break;
      beta /= q;
    }
    ro = offset_origin(v.p, v.ng, bs.wi);
    rd = bs.wi;
  }
  return L;
}

// integrator/nee.rs:15-93: light sampling without MIS (sample_light, the
// plain environment distribution), emission and escapes counted only from
// the camera and after delta samples
Vec3 trace_nee(const RenderScene& s, const Ray& ray, const PathSampler& sampler, uint32_t max_depth) {
  Vec3 L(0, 0, 0), beta(1, 1, 1);
  PathLock lock;
  Vec3 ro = ray.origin, rd = ray.direction;
  bool count_emission = true;
  for (uint32_t depth = 0; depth < max_depth; ++depth) {
    VertexRandoms rnd = sampler.path_vertex_randoms(depth);
    AuxRng aux(rnd.aux_rng_seed);  // nee.rs:31-34: the arriving ray, then the light sample
    SceneHit h;
    if (!closest(s, ro, rd, &h, &aux)) {
      if (count_emission && s.has_env) L += beta * s.env.radiance(rd);
      break;
    }
    Vertex v = s.shading_vertex(h.instance, h.triangle, h.bary, rd);
    const Material& m = s.mat_of(h.instance);
    lock.stamp(v, beta);
    Vec3 le;
    if (count_emission && material_le(m, v, &le)) L += beta * le;
    if (!is_pure_emitter(m)) L += beta * direct_light_impl(s, m, v, rnd, nullptr, kDirectNee, &aux);
    MatSample bs;
    bool ok = m.kind == kOpenPbr ? openpbr_sample(m, v, rnd.material, &bs)
              : m.kind == kLambert ? lambert_sample(m, v, rnd.material.u_dir, &bs)
                                   : false;
    if (!ok) break;
    beta *= bs.weight;
    lock.take(bs);
    if (depth + 1 >= 4) {
      float q = clampf(max_element(beta), 0.05f, 1.0f);
      if (rnd.u_rr > q) break;
      beta /= q;
    }
    ro = offset_origin(v.p, v.ng, bs.wi);
    rd = bs.wi;
    count_emission = bs.delta;
  }
  return L;
}

// integrator/mis.rs:19-139
Vec3 trace_mis(const RenderScene& s, const Ray& ray, const PathSampler& sampler, uint32_t max_depth) {
  Vec3 L(0, 0, 0), beta(1, 1, 1);
  PathLock lock;
  AuxRng aux0(sampler.initial_aux_rng_seed());  // mis.rs:28-31
  SceneHit h;
  if (!closest(s, ray.origin, ray.direction, &h, &aux0)) return s.has_env ? s.env.radiance(ray.direction) : L;
  Vertex v = s.shading_vertex(h.instance, h.triangle, h.bary, ray.direction);
  const Material* m = &s.mat_of(h.instance);
  Vec3 le0;
  if (material_le(*m, v, &le0)) L += le0;
  for (uint32_t depth = 0; depth < max_depth; ++depth) {
    VertexRandoms rnd = sampler.path_vertex_randoms(depth);
    lock.stamp(v, beta);
    // mis.rs:52: the light sample's shadow ray, then the bounce ray, draw from it
    AuxRng aux(rnd.aux_rng_seed);
    if (is_pure_emitter(*m)) break;
    L += beta * direct_light(s, *m, v, rnd, nullptr, kDirectMis, &aux);
    MatSample bs;
    bool ok = m->kind == kOpenPbr ? openpbr_sample(*m, v, rnd.material, &bs)
                                  : lambert_sample(*m, v, rnd.material.u_dir, &bs);
    if (!ok) break;
    beta *= bs.weight;
    lock.take(bs);
    if (depth + 1 >= 4) {
      float q = clampf(max_element(beta), 0.05f, 1.0f);
      if (rnd.u_rr > q) break;
      beta /= q;
    }
    SceneHit nh;
    if (!closest(s, offset_origin(v.p, v.ng, bs.wi), bs.wi, &nh, &aux)) {
      L += beta * env_escape(s, bs.wi, bs.delta, bs.pdf);
      break;
    }
    Vertex nv = s.shading_vertex(nh.instance, nh.triangle, nh.bary, bs.wi);
    const Material* nm = &s.mat_of(nh.instance);
    Vec3 le;
    if (material_le(*nm, nv, &le)) {
      if (bs.delta) L += beta * le;
      else L += beta * le * balance(bs.pdf, light_pdf_for_hit(s, *m, v, nv));
    }
    if (std::getenv("ORC_MIS_TRACE"))
      std::fprintf(stderr, "mis d=%u hit inst %d tri %d t %.9g p (%.9g %.9g %.9g) wi (%.9g %.9g %.9g) beta (%.6g %.6g %.6g) pdf %.6g delta %d L (%.6g %.6g %.6g)\n",
                   depth, nh.instance, nh.triangle, nh.t, nv.p.x, nv.p.y, nv.p.z, bs.wi.x, bs.wi.y, bs.wi.z, beta.x,
                   beta.y, beta.z, bs.pdf, (int)bs.delta, L.x, L.y, L.z);
    v = nv;
    m = nm;
  }
  return L;
}

void replay_mis(const RenderScene& s, const Ray& ray, const PathSampler& sampler, uint32_t max_depth, Vec3 L,
                AdjointVertexSink& sink) {
  Vec3 R = L, beta(1, 1, 1);
  PathLock lock;
  AuxRng aux0(sampler.initial_aux_rng_seed());
  SceneHit h;
  if (!closest(s, ray.origin, ray.direction, &h, &aux0)) return;
  Vertex v = s.shading_vertex(h.instance, h.triangle, h.bary, ray.direction);
  const Material* m = &s.mat_of(h.instance);
  uint32_t mi = s.geo.instances[h.instance].material_index;
  Vec3 le0;
  if (material_le(*m, v, &le0)) R = R - le0;
  for (uint32_t depth = 0; depth < max_depth; ++depth) {
    VertexRandoms rnd = sampler.path_vertex_randoms(depth);
    lock.stamp(v, beta);
    AuxRng aux(rnd.aux_rng_seed);
    if (is_pure_emitter(*m)) break;
    Vec3 wl(0, 0, 0);
    const Vec3 c = beta * direct_light(s, *m, v, rnd, &wl, kDirectMis, &aux);
    R = R - c;
    // a light sample at an OpenPBR vertex (directional lights): its
    // contribution scales with f at the light direction
    if (m->kind == kOpenPbr && length_squared(c) > 0.0f) sink.vertex(mi, v, wl, c);
    MatSample bs;
    bool ok = m->kind == kOpenPbr ? openpbr_sample(*m, v, rnd.material, &bs)
                                  : lambert_sample(*m, v, rnd.material.u_dir, &bs);
    if (!ok) break;
    beta *= bs.weight;
    lock.take(bs);
    if (depth + 1 >= 4) {
      float q = clampf(max_element(beta), 0.05f, 1.0f);
      if (rnd.u_rr > q) break;
      beta /= q;
    }
    if (m->kind == kOpenPbr && !bs.delta) sink.vertex(mi, v, bs.wi, R);
    SceneHit nh;
    if (!closest(s, offset_origin(v.p, v.ng, bs.wi), bs.wi, &nh, &aux)) break;  // R = the escape emission
    Vertex nv = s.shading_vertex(nh.instance, nh.triangle, nh.bary, bs.wi);
    const Material* nm = &s.mat_of(nh.instance);
    Vec3 le;
    if (material_le(*nm, nv, &le)) {
      if (bs.delta) R = R - beta * le;
      else R = R - beta * le * balance(bs.pdf, light_pdf_for_hit(s, *m, v, nv));
    }
    v = nv;
    m = nm;
    mi = s.geo.instances[nh.instance].material_index;
  }
}

namespace {
Vec3 one_sample(const RenderScene& s, const RenderJob& job, uint32_t pixel, uint32_t sample) {
  uint32_t px = pixel % job.width, py = pixel / job.width;
  PathSampler ps(px, py, sample, job.spp, job.width, job.height, job.seed);
  Vec2 us = ps.camera_sample();
  Ray r = job.cam.generate_ray_differential(job.width, job.height, px, py, us, job.spp);
  switch (job.integrator) {
    case 1: return trace_bdpt(s, r, ps, job.max_depth);
    case 2: return trace_nee(s, r, ps, job.max_depth);
    case 3: return trace_pt(s, r, ps, job.max_depth);
    default: return trace_mis(s, r, ps, job.max_depth);
  }
}
}  // namespace

void render_pixels(const RenderScene& s, const RenderJob& job, uint32_t p0, uint32_t p1, float* out, int nthreads) {
  par_for(p1 - p0, nthreads, [&](uint64_t k) {
    uint32_t pixel = p0 + (uint32_t)k;
    Vec3 color(0, 0, 0);
    for (uint32_t i = 0; i < job.spp; ++i) {
      Vec3 smp = one_sample(s, job, pixel, i);
      float n = (float)(i + 1);
      color += (smp - color) / n;
    }
    Vec3 e = color * job.cam.exposure;
    out[3 * k] = e.x;
    out[3 * k + 1] = e.y;
    out[3 * k + 2] = e.z;
  });
}

void render_samples(const RenderScene& s, const RenderJob& job, uint64_t first, uint64_t count, float* out,
                    int nthreads) {
  par_for(count, nthreads, [&](uint64_t k) {
    uint64_t path = first + k;
    Vec3 v = one_sample(s, job, (uint32_t)(path / job.spp), (uint32_t)(path % job.spp));
    out[3 * k] = v.x;
    out[3 * k + 1] = v.y;
    out[3 * k + 2] = v.z;
  });
}

}  // namespace orc

// ---- unit-level entry points (reference integrator unit tests) -------------
extern "C" {

// direct_light_mis_contribution at the shading vertex of (inst, tri, bary) seen
// along `incident` (integrator/mis.rs:145-210); mode 1: BDPT's
// direct_non_area_light_contribution (integrator/bdpt.rs:396-464); mode 2: the
// NEE integrator's direct_light_nee_contribution (integrator/nee.rs:104-150).
void orc_render_direct_light(void* h, int inst, int tri, const float* bary3, const float* incident3, float u_cat,
                             float u_tree, float us0, float us1, float* out3, int mode) {
  using namespace orc;
  const RenderScene& s = *(const RenderScene*)h;
  Vertex v = s.shading_vertex(inst, tri, Vec3(bary3[0], bary3[1], bary3[2]),
                              Vec3(incident3[0], incident3[1], incident3[2]));
  VertexRandoms rnd{};
  rnd.light.u_category = u_cat;
  rnd.light.u_tree = u_tree;
  rnd.light.u_surface = Vec2(us0, us1);
  Vec3 r = direct_light(s, s.mat_of(inst), v, rnd, nullptr, mode);
  out3[0] = r.x; out3[1] = r.y; out3[2] = r.z;
}

// The environment's contribution to a ray that left the scene after a BSDF
// sample (integrator/mis.rs:238-258, bdpt.rs:466-486), times `throughput3`.
void orc_render_env_escape(void* h, const float* dir3, const float* throughput3, float bsdf_pdf, int delta,
                           float* out3) {
  using namespace orc;
  const RenderScene& s = *(const RenderScene*)h;
  const Vec3 r = Vec3(throughput3[0], throughput3[1], throughput3[2]) *
                 env_escape(s, Vec3(dir3[0], dir3[1], dir3[2]), delta != 0, bsdf_pdf);
  out3[0] = r.x; out3[1] = r.y; out3[2] = r.z;
}

// emitted_radiance_from_bsdf_sample_area (integrator/mis.rs:212-236)
void orc_render_emitted(void* h, int inst, int tri, const float* bary3, const float* incident3, int linst, int ltri,
                        const float* lbary3, const float* lincident3, const float* throughput3, float bsdf_pdf,
                        int delta, float* out3) {
  using namespace orc;
  const RenderScene& s = *(const RenderScene*)h;
  Vertex v = s.shading_vertex(inst, tri, Vec3(bary3[0], bary3[1], bary3[2]),
                              Vec3(incident3[0], incident3[1], incident3[2]));
  Vertex lv = s.shading_vertex(linst, ltri, Vec3(lbary3[0], lbary3[1], lbary3[2]),
                               Vec3(lincident3[0], lincident3[1], lincident3[2]));
  const Material& lm = s.mat_of(linst);
  Vec3 r(0, 0, 0);
  Vec3 le;
  if (material_le(lm, lv, &le)) {
    Vec3 beta(throughput3[0], throughput3[1], throughput3[2]);
    r = delta ? beta * le : beta * le * balance(bsdf_pdf, light_pdf_for_hit(s, s.mat_of(inst), v, lv));
  }
  out3[0] = r.x; out3[1] = r.y; out3[2] = r.z;
}

// Lambert pdf at a vertex (material pdf used by the unit tests)
float orc_render_material_pdf(void* h, int inst, int tri, const float* bary3, const float* incident3,
                              const float* wi3) {
  using namespace orc;
  const RenderScene& s = *(const RenderScene*)h;
  Vertex v = s.shading_vertex(inst, tri, Vec3(bary3[0], bary3[1], bary3[2]),
                              Vec3(incident3[0], incident3[1], incident3[2]));
  return lambert_pdf(v, Vec3(wi3[0], wi3[1], wi3[2]));
}

}  // extern "C"
