// Oracle: bidirectional path tracing, integrator/bdpt.rs:70-791, for area
// lights (the only light type in scope: no environment, point, spot or
// directional lights, so the camera subpath's non-area-light NEE and the
// infinite-light terms are zero).
#include <cstdio>
#include <cstdlib>
#include "render.h"

namespace orc {

namespace {
constexpr float kShadowTolerance = 1.0e-3f;

struct PathVertex {
  bool light;  // VertexType::Light (else Surface)
  Vertex vtx;
  Vec3 beta;
  float pdf_fwd_area = 0, pdf_rev_area = 0;
  bool delta = false, connectible = false;
};

bool closest(const RenderScene& s, Vec3 o, Vec3 d, SceneHit* h, AuxRng* aux) {
  Ray r;
  r.origin = o;
  r.direction = d;
  return s.geo.closest_hit(r, h, nullptr, aux);
}
Vec3 offset_origin(Vec3 p, Vec3 ng, Vec3 d) {  // integrator/mod.rs:77-85
  Vec3 n = dot(d, ng) >= 0.0f ? ng : -ng;
  return p + 1.0e-4f * n;
}
float remap0(float x) { return x == 0.0f ? 1.0f : x; }

// bdpt.rs:626-642
float solid_angle_pdf_to_area(float pdf, Vec3 from, Vec3 to, Vec3 to_ng) {
  if (pdf <= 0.0f) return 0.0f;
  Vec3 d = to - from;
  float dist2 = length_squared(d);
  if (dist2 <= 0.0f) return 0.0f;
  Vec3 wi = normalize_or_zero(d);
  float cos_to = std::fabs(dot(to_ng, -wi));
  if (cos_to <= 0.0f) return 0.0f;
  return pdf * cos_to / dist2;
}
// bdpt.rs:644-659 (linear search over the area lights, as the reference)
float area_light_origin_pdf_area(const RenderScene& s, const PathVertex& v) {
  for (const AreaLight& a : s.area_lights) {
    if (a.inst == v.vtx.inst && a.tri == v.vtx.tri) {
      if (s.area_light_weight_sum <= 0.0f || a.area <= 0.0f) return 0.0f;
      return a.weight / s.area_light_weight_sum / a.area;
    }
  }
  return 0.0f;
}
// bdpt.rs:661-675
float light_emission_pdf_area(const PathVertex& light, const PathVertex& target) {
  Vec3 d = target.vtx.p - light.vtx.p;
  float dist2 = length_squared(d);
  if (dist2 <= 0.0f) return 0.0f;
  Vec3 dir = d / std::sqrt(dist2);
  float cos_emit = fmax_num(dot(light.vtx.ng, dir), 0.0f);
  if (cos_emit <= 0.0f) return 0.0f;
  return solid_angle_pdf_to_area(cos_emit / kPi, light.vtx.p, target.vtx.p, target.vtx.ng);
}
// bdpt.rs:677-702
float bsdf_pdf_area(const RenderScene& s, const PathVertex& from, const PathVertex* prev, const PathVertex& target) {
  Vec3 d = target.vtx.p - from.vtx.p;
  if (length_squared(d) <= 0.0f) return 0.0f;
  Vertex v = from.vtx;
  if (prev) {
    Vec3 tp = prev->vtx.p - from.vtx.p;
    if (length_squared(tp) <= 0.0f) return 0.0f;
    v.wo = normalize_or_zero(tp);
  }
  Vec3 wi = normalize_or_zero(d);
  float pdf_dir = material_pdf(s.mat_of(from.vtx.inst), v, wi);
  return solid_angle_pdf_to_area(pdf_dir, from.vtx.p, target.vtx.p, target.vtx.ng);
}
float vertex_pdf_area(const RenderScene& s, const PathVertex& from, const PathVertex* prev, const PathVertex& target) {
  return from.light ? light_emission_pdf_area(from, target) : bsdf_pdf_area(s, from, prev, target);
}

// bdpt.rs:717-746
float camera_light_hit_mis_weight(const RenderScene& s, const std::vector<PathVertex>& cp) {
  if (cp.size() <= 1) return 1.0f;
  const size_t pt = cp.size() - 1, ptm = pt - 1;
  float pt_pdf_rev = area_light_origin_pdf_area(s, cp[pt]);
  float ptm_pdf_rev = light_emission_pdf_area(cp[pt], cp[ptm]);
  float sum = 0.0f, ri = 1.0f;
  for (size_t i = cp.size() - 1; i >= 1; --i) {
    float pr = i == pt ? pt_pdf_rev : (i == ptm ? ptm_pdf_rev : cp[i].pdf_rev_area);
    ri *= remap0(pr) / remap0(cp[i].pdf_fwd_area);
    if (!cp[i].delta && !cp[i - 1].delta) sum += ri;
  }
  return 1.0f / (1.0f + fmax_num(sum, 0.0f));
}

// bdpt.rs:748-817: light_path[0..s), camera_path[0..t)
float bdpt_mis_weight(const RenderScene& s, const PathVertex* lp, size_t ns, const PathVertex* cp, size_t nt) {
  if (ns + nt <= 2) return 1.0f;
  const size_t qs = ns - 1, pt = nt - 1;
  const PathVertex* qsm = qs >= 1 ? &lp[qs - 1] : nullptr;
  const PathVertex* ptm = pt >= 1 ? &cp[pt - 1] : nullptr;
  float pt_pdf_rev = vertex_pdf_area(s, lp[qs], qsm, cp[pt]);
  float ptm_pdf_rev = ptm ? vertex_pdf_area(s, cp[pt], &lp[qs], *ptm) : 0.0f;
  float qs_pdf_rev = vertex_pdf_area(s, cp[pt], ptm, lp[qs]);
  float qsm_pdf_rev = qsm ? vertex_pdf_area(s, lp[qs], &cp[pt], *qsm) : 0.0f;
  float sum = 0.0f, ri = 1.0f;
  for (size_t i = nt - 1; i >= 1; --i) {
    float pr = i == pt ? pt_pdf_rev : ((pt >= 1 && i == pt - 1) ? ptm_pdf_rev : cp[i].pdf_rev_area);
    ri *= remap0(pr) / remap0(cp[i].pdf_fwd_area);
    if (!cp[i].delta && !cp[i - 1].delta) sum += ri;
  }
  ri = 1.0f;
  for (size_t k = ns; k-- > 0;) {
    float pr = k == qs ? qs_pdf_rev : ((qs >= 1 && k == qs - 1) ? qsm_pdf_rev : lp[k].pdf_rev_area);
    ri *= remap0(pr) / remap0(lp[k].pdf_fwd_area);
    bool prev_delta = k > 0 && lp[k - 1].delta;
    if (!lp[k].delta && !prev_delta) sum += ri;
  }
  return 1.0f / (1.0f + fmax_num(sum, 0.0f));
}

// bdpt.rs:555-575, 577-602
bool visible_between(const RenderScene& s, Vec3 o, Vec3 ng, Vec3 dir, float dist, int tinst, int ttri,
                     AuxRng* aux) {
  SceneHit h;
  if (!closest(s, offset_origin(o, ng, dir), dir, &h, aux)) return true;
  if (h.instance == tinst && h.triangle == ttri) return true;
  return h.t >= dist * (1.0f - kShadowTolerance);
}
Vec3 connect(const RenderScene& s, const PathVertex& lv, const PathVertex& cv, AuxRng* aux) {
  Vec3 delta = cv.vtx.p - lv.vtx.p;
  float dist2 = length_squared(delta);
  if (dist2 <= 0.0f) return Vec3(0, 0, 0);
  float dist = std::sqrt(dist2);
  Vec3 w_lc = delta / dist;
  Vec3 w_cl = -w_lc;
  if (!visible_between(s, lv.vtx.p, lv.vtx.ng, w_lc, dist, cv.vtx.inst, cv.vtx.tri, aux)) return Vec3(0, 0, 0);
  Vec3 f_cam = material_eval(s.mat_of(cv.vtx.inst), cv.vtx, w_cl, kRadiance);
  if (length_squared(f_cam) == 0.0f) return Vec3(0, 0, 0);
  Vec3 f_light;
  if (lv.light) {
    if (dot(lv.vtx.ng, w_lc) <= 0.0f) return Vec3(0, 0, 0);
    f_light = Vec3(1, 1, 1);
  } else {
    f_light = material_eval(s.mat_of(lv.vtx.inst), lv.vtx, w_lc, kImportance);
  }
  if (length_squared(f_light) == 0.0f) return Vec3(0, 0, 0);
  float g = std::fabs(dot(lv.vtx.ng, w_lc)) * std::fabs(dot(cv.vtx.ng, w_cl)) / dist2;
  if (g <= 0.0f) return Vec3(0, 0, 0);
  return lv.beta * f_light * g * f_cam * cv.beta;
}

// bdpt.rs:135-262
Vec3 camera_subpath(const RenderScene& s, const Ray& ray0, const PathSampler& sp, uint32_t max_depth,
                    std::vector<PathVertex>& vs, AuxRng* aux) {
  vs.clear();
  Vec3 L(0, 0, 0), beta(1, 1, 1);
  Vec3 ro = ray0.origin, rd = ray0.direction;
  bool count_emission = true;
  bool have_pending = false;
  bool has_lock = false;
  float lock = 0.0f;
  Vec3 pending_from;
  float pending_pdf = 0.0f;
  const bool non_area = scene_has_non_area_lights(s);
  for (uint32_t depth = 0; depth < max_depth; ++depth) {
    VertexRandoms rnd = sp.path_vertex_randoms(depth);
    *aux = AuxRng(rnd.aux_rng_seed);  // bdpt.rs:160: the arriving ray, then the vertex's light sample
    SceneHit h;
    if (!closest(s, ro, rd, &h, aux)) {
      // emitted_radiance_from_infinite_hit (bdpt.rs:466-486)
      L += beta * env_escape(s, rd, count_emission, pending_pdf);
      break;
    }
    Vertex v = s.shading_vertex(h.instance, h.triangle, h.bary, rd);
    // the path state the vertex keeps for its connections (bdpt.rs:177-178, 344-345)
    v.path_throughput = beta;
    v.has_lock = has_lock;
    v.wavelength_lock = lock;
    const Material& m = s.mat_of(h.instance);
    PathVertex pv;
    pv.light = false;
    pv.vtx = v;
    pv.beta = beta;
    pv.pdf_fwd_area = have_pending ? solid_angle_pdf_to_area(pending_pdf, pending_from, v.p, v.ng) : 0.0f;
    have_pending = false;
    pv.connectible = !is_pure_emitter(m);
    vs.push_back(pv);
    const size_t vi = vs.size() - 1;
    Vec3 le;
    if (material_le(m, v, &le)) {
      float w = count_emission ? 1.0f : camera_light_hit_mis_weight(s, vs);
      L += beta * le * w;
    }
    // direct_non_area_light_contribution (bdpt.rs:207-221, 396-464)
    if (non_area && !is_pure_emitter(m))
      L += beta * direct_light(s, m, v, rnd, nullptr, kDirectBdptNonArea, aux);
    MatSampleOut smp;
    if (!material_sample(m, v, rnd.material, kRadiance, &smp)) break;
    vs[vi].delta = smp.delta;
    vs[vi].connectible = !vs[vi].delta && !is_pure_emitter(m);
    if (vi > 0) vs[vi - 1].pdf_rev_area = solid_angle_pdf_to_area(smp.pdf_rev, v.p, vs[vi - 1].vtx.p, vs[vi - 1].vtx.ng);
    ro = offset_origin(v.p, v.ng, smp.wi);
    rd = smp.wi;
    beta *= smp.weight;
    if (smp.has_lock) {
      has_lock = true;
      lock = smp.wavelength_lock;
    }
    if (depth + 1 >= 4) {
      float q = clampf(max_element(beta), 0.05f, 1.0f);
      if (rnd.u_rr > q) break;
      beta /= q;
    }
    have_pending = true;
    pending_from = v.p;
    pending_pdf = smp.pdf;
    count_emission = smp.delta;
  }
  return L;
}

// bdpt.rs:264-385
void light_subpath(const RenderScene& s, const PathSampler& sp, uint32_t max_depth, std::vector<PathVertex>& vs,
                   AuxRng* aux) {
  vs.clear();
  if (max_depth == 0) return;
  VertexRandoms rnd0 = sp.path_vertex_randoms(0);
  // sample_area_light_triangle (bdpt.rs:540-553): first prefix >= u * sum
  if (s.area_light_weight_sum <= 0.0f || s.area_lights.empty()) return;
  float target = clampf(rnd0.light.u_category, 0.0f, 1.0f) * s.area_light_weight_sum;
  size_t lo = 0, hi = s.area_lights.size();
  while (lo < hi) {
    size_t mid = (lo + hi) / 2;
    if (s.area_lights[mid].prefix_weight < target) lo = mid + 1;
    else hi = mid;
  }
  const AreaLight& al = s.area_lights[std::min(lo, s.area_lights.size() - 1)];
  float pmf = al.weight / s.area_light_weight_sum;
  // Scene::sample_triangle_point (scene/mod.rs:620-635)
  Vec3 p[3];
  s.triangle_world(al.inst, al.tri, p);
  float su0 = std::sqrt(clampf(rnd0.light.u_surface.x, 0.0f, 1.0f));
  float u1 = clampf(rnd0.light.u_surface.y, 0.0f, 1.0f);
  Vec3 bary(1.0f - su0, u1 * su0, (1.0f - u1) * su0);
  float area = 0.5f * length(cross(p[1] - p[0], p[2] - p[0]));
  float pdf_point = area > 0.0f ? 1.0f / area : 0.0f;
  float pdf_area = pmf * pdf_point;
  if (pdf_area <= 0.0f) return;
  Vec3 gn = normalize_or_zero(cross(p[1] - p[0], p[2] - p[0]));
  Frame fr = Frame::from_normal(gn);
  Vec3 ld = sample_cosine_hemisphere(rnd0.material.u_dir);
  Vec3 emit = normalize_or_zero(fr.to_world(ld));
  float pdf_dir = fmax_num(ld.z, 0.0f) / kPi;
  if (length_squared(emit) == 0.0f || pdf_dir <= 0.0f) return;
  Vertex lv = s.shading_vertex(al.inst, al.tri, bary, -emit);
  lv.wo = emit;
  Vec3 le;
  if (!material_le(s.mat_of(al.inst), lv, &le)) return;
  float cos_emit = fmax_num(dot(lv.ng, emit), 0.0f);
  if (cos_emit <= 0.0f) return;
  Vec3 endpoint_beta = le / pdf_area;
  PathVertex v0;
  v0.light = true;
  v0.vtx = lv;
  v0.beta = endpoint_beta;
  v0.pdf_fwd_area = pdf_area;
  v0.connectible = true;
  vs.push_back(v0);
  Vec3 ro = offset_origin(lv.p, lv.ng, emit), rd = emit;
  Vec3 beta = endpoint_beta * (cos_emit / pdf_dir);
  Vec3 pending_from = lv.p;
  float pending_pdf = pdf_dir;
  bool have_pending = true;
  bool has_lock = false;
  float lock = 0.0f;
  for (uint32_t depth = 1; depth < max_depth; ++depth) {
    VertexRandoms rnd = sp.path_vertex_randoms(depth);
    *aux = AuxRng(rnd.aux_rng_seed);  // bdpt.rs:335
    SceneHit h;
    if (!closest(s, ro, rd, &h, aux)) break;
    Vertex v = s.shading_vertex(h.instance, h.triangle, h.bary, rd);
    // the path state the vertex keeps for its connections (bdpt.rs:177-178, 344-345)
    v.path_throughput = beta;
    v.has_lock = has_lock;
    v.wavelength_lock = lock;
    const Material& m = s.mat_of(h.instance);
    PathVertex pv;
    pv.light = false;
    pv.vtx = v;
    pv.beta = beta;
    pv.pdf_fwd_area = have_pending ? solid_angle_pdf_to_area(pending_pdf, pending_from, v.p, v.ng) : 0.0f;
    pv.connectible = !is_pure_emitter(m);
    vs.push_back(pv);
    const size_t vi = vs.size() - 1;
    MatSampleOut smp;
    if (!material_sample(m, v, rnd.material, kImportance, &smp)) break;
    vs[vi].delta = smp.delta;
    vs[vi].connectible = !vs[vi].delta && !is_pure_emitter(m);
    if (vi > 0) vs[vi - 1].pdf_rev_area = solid_angle_pdf_to_area(smp.pdf_rev, v.p, vs[vi - 1].vtx.p, vs[vi - 1].vtx.ng);
    ro = offset_origin(v.p, v.ng, smp.wi);
    rd = smp.wi;
    beta *= smp.weight;
    if (smp.has_lock) {
      has_lock = true;
      lock = smp.wavelength_lock;
    }
    pending_from = v.p;
    pending_pdf = smp.pdf;
    have_pending = true;
  }
}
}  // namespace

// ORC_BDPT_TRACE=1: print each connection strategy's MIS weight and
// unweighted contribution, and the camera subpath's radiance, to stderr
// (debugging aid of the checker; off by default).
bool trace_on() {
  static const bool on = std::getenv("ORC_BDPT_TRACE") != nullptr;
  return on;
}

Vec3 trace_bdpt(const RenderScene& s, const Ray& ray, const PathSampler& sp, uint32_t max_depth) {
  thread_local std::vector<PathVertex> cam, lig;
  // one AuxRng through both subpaths (each depth reseeds it) and then every
  // connection's visibility test in loop order (bdpt.rs:81-121)
  AuxRng aux(sp.initial_aux_rng_seed());
  Vec3 L = camera_subpath(s, ray, sp, max_depth, cam, &aux);
  light_subpath(s, sp, max_depth, lig, &aux);
  if (trace_on()) {
    std::fprintf(stderr, "bdpt camera L=(%.9g %.9g %.9g) |cam|=%zu |light|=%zu\n", L.x, L.y, L.z, cam.size(), lig.size());
    for (size_t i = 0; i < cam.size(); ++i)
      std::fprintf(stderr, "  cam %zu inst %d tri %d conn %d delta %d beta (%.6g %.6g %.6g) fwd %.6g rev %.6g\n", i,
                   cam[i].vtx.inst, cam[i].vtx.tri, (int)cam[i].connectible, (int)cam[i].delta, cam[i].beta.x,
                   cam[i].beta.y, cam[i].beta.z, cam[i].pdf_fwd_area, cam[i].pdf_rev_area);
    for (size_t i = 0; i < lig.size(); ++i)
      std::fprintf(stderr, "  lig %zu inst %d tri %d conn %d delta %d beta (%.6g %.6g %.6g) fwd %.6g rev %.6g\n", i,
                   lig[i].vtx.inst, lig[i].vtx.tri, (int)lig[i].connectible, (int)lig[i].delta, lig[i].beta.x,
                   lig[i].beta.y, lig[i].beta.z, lig[i].pdf_fwd_area, lig[i].pdf_rev_area);
  }
  for (size_t li = 0; li < lig.size(); ++li)
    for (size_t ci = 0; ci < cam.size(); ++ci) {
      if (!lig[li].connectible || !cam[ci].connectible) continue;
      float w = bdpt_mis_weight(s, lig.data(), li + 1, cam.data(), ci + 1);
      const Vec3 c = connect(s, lig[li], cam[ci], &aux);
      if (trace_on())
        std::fprintf(stderr, "bdpt s=%zu t=%zu w=%.9g c=(%.9g %.9g %.9g)\n", li + 1, ci + 1, w, c.x, c.y, c.z);
      L += w * c;
    }
  return L;
}

}  // namespace orc
