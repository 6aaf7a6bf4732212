// Bidirectional path tracing on the device, integrator/bdpt.rs:70-791: camera
// subpath, light subpath from an emissive triangle picked by power, and every
// connection between their connectible vertices with a visibility ray and the
// reference's MIS weight.  Point, spot, directional and environment lights take
// no part in the light subpaths: as in the reference, each camera vertex of a
// scene that has them takes one light sample that skips area lights, and a
// camera ray that leaves the scene reads the environment.
// Both subpaths live in the thread's local memory (interleaved across the warp
// by the hardware, so vertex k of every lane is one coalesced line).
#pragma once
#include "render.cuh"

namespace tpt {

constexpr uint32_t kBdptMaxDepth = kBdptMaxDepthApi;

// ---- material interface with transport modes (material/mod.rs:33-79): eval
// (material_eval) is in render.cuh --------------------------------------------
__device__ __forceinline__ V3 modified_weight(const Vertex& v, V3 wi, V3 w, bool delta, bool importance) {
  if (!importance || delta || length_sq(w) == 0.0f) return w;
  const float cos_wo_geom = fabsf(dot(v.wo, v.ng)), cos_wo_sh = fabsf(dot(v.wo, v.ns));
  const float cos_wi_geom = fabsf(dot(wi, v.ng)), cos_wi_sh = fabsf(dot(wi, v.ns));
  if (cos_wo_geom <= kGeomCosEps || cos_wi_sh <= kGeomCosEps) return V3{0.0f, 0.0f, 0.0f};
  return w * (cos_wo_sh / cos_wo_geom) * (cos_wi_geom / cos_wi_sh);
}
__device__ __forceinline__ float lambert_bsdf_pdf(V3 wo, V3 wi) {
  if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
  return fmaxf(wi.z, 0.0f) / kPiF;
}

// Material::pdf
static __device__ __noinline__ float material_pdf(const DevRender& S, const DevMaterialRec& m, const Vertex& v, V3 wi) {
  if (m.kind == kDevLambert) {
    if (dot(v.wo, v.ng) <= 0.0f || dot(wi, v.ng) <= 0.0f) return 0.0f;
    return lambert_bsdf_pdf(normalize_or_zero(to_local(v.frame, v.wo)), normalize_or_zero(to_local(v.frame, wi)));
  }
  if (m.kind == kDevOpenPbr) {
    if (dot(v.wo, v.ng) <= 0.0f) return 0.0f;
    const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
    const V3 wi_l = normalize_or_zero(to_local(v.frame, wi));
    if (wo_l.z <= 0.0f) return 0.0f;
    opbr::OpbrVertex s;
    opbr::init_vertex(s, S.d.openpbr + m.openpbr, S.d.cec_e, S.d.dec_e, wo_l, v.front, fabsf(wo_l.z));
    s.thr = v.thr;
    s.lock = v.lock;
    V3 f;
    float pdf;
    opbr::eval_pdf(s, s, wi_l, f, pdf);
    return pdf;
  }
  return 0.0f;
}

struct MatSample {
  V3 weight, wi;
  float pdf, pdf_rev;
  bool delta;
  float lock;  // wavelength lock set by the sample (< 0: none)
};

// Material::sample with pdf_rev
static __device__ __noinline__ bool material_sample_rev(const DevRender& S, const DevMaterialRec& m, const Vertex& v,
                                                       float u_lobe, float u0, float u1, const float* ux,
                                                       bool importance, MatSample& s) {
  s.lock = -1.0f;
  if (m.kind == kDevLambert) {
    const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
    if (wo_l.z <= 0.0f) return false;
    const V3 wi_l = opbr::sample_cosine_hemisphere(u0, u1);
    const float pdf = lambert_bsdf_pdf(wo_l, wi_l);
    if (pdf <= 0.0f) return false;
    const V3 wi = to_world(v.frame, wi_l);
    s.weight = modified_weight(v, wi, V3{m.rho[0], m.rho[1], m.rho[2]}, false, importance);
    s.wi = wi;
    s.pdf = pdf;
    s.pdf_rev = lambert_bsdf_pdf(wi_l, wo_l);
    s.delta = false;
    return dot(wi, v.ng) > kGeomCosEps;
  }
  if (m.kind == kDevOpenPbr) {
    if (dot(v.wo, v.ng) <= 0.0f) return false;
    const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
    if (wo_l.z <= 0.0f) return false;
    opbr::OpbrVertex ov;
    opbr::init_vertex(ov, S.d.openpbr + m.openpbr, S.d.cec_e, S.d.dec_e, wo_l, v.front, fabsf(wo_l.z));
    ov.thr = v.thr;
    ov.lock = v.lock;
    opbr::Sample bs;
    if (!opbr::sample(ov, u_lobe, u0, u1, bs, importance, true, ux)) return false;
    s.lock = bs.lock;
    const V3 wi = to_world(v.frame, bs.wi);
    if (!opbr_sample_side_ok(v, wi, bs.flags)) return false;
    s.delta = (bs.flags & opbr::kFlagDelta) != 0;
    s.weight = modified_weight(v, wi, bs.weight, s.delta, importance);
    s.wi = wi;
    s.pdf = bs.pdf;
    s.pdf_rev = bs.pdf_rev;
    return true;
  }
  return false;  // pure emitter
}

// ---- path vertices ---------------------------------------------------------
constexpr uint32_t kBdLight = 1u, kBdDelta = 2u, kBdConnectible = 4u;

// beta: v.thr (ShadingVertex::path_throughput is the throughput arriving at
// the vertex; the light endpoint's is its emitted radiance over its pdf)
struct BdVertex {
  Vertex v;
  float pdf_fwd, pdf_rev;
  uint32_t flags;
};

static_assert(sizeof(BdVertex) <= kBdVertexBytes, "BDPT vertex record");

__device__ __forceinline__ float remap0(float x) { return x == 0.0f ? 1.0f : x; }

// bdpt.rs:626-642
__device__ __forceinline__ float solid_angle_to_area(float pdf, V3 from, V3 to, V3 to_ng) {
  if (pdf <= 0.0f) return 0.0f;
  const V3 d = to - from;
  const float dist2 = length_sq(d);
  if (dist2 <= 0.0f) return 0.0f;
  const V3 wi = normalize_or_zero(d);
  const float cos_to = fabsf(dot(to_ng, -wi));
  if (cos_to <= 0.0f) return 0.0f;
  return pdf * cos_to / dist2;
}
// bdpt.rs:644-659 through the emitter map instead of a linear search
__device__ __forceinline__ float area_light_origin_pdf(const DevRender& S, const BdVertex& v) {
  const uint32_t base = __ldg(&S.d.inst[v.v.inst].leaf_base);
  if (base == 0xFFFFFFFFu) return 0.0f;
  const uint32_t k = __ldg(S.d.area_light_of + base + v.v.tri);
  if (k == 0xFFFFFFFFu) return 0.0f;
  const float area = __ldg(&S.d.area_lights[k].area);
  if (S.d.area_light_weight_sum <= 0.0f || area <= 0.0f) return 0.0f;
  return __ldg(&S.d.area_lights[k].weight) / S.d.area_light_weight_sum / area;
}
// bdpt.rs:661-675
__device__ __forceinline__ float light_emission_pdf(const BdVertex& light, const BdVertex& target) {
  const V3 d = target.v.p - light.v.p;
  const float dist2 = length_sq(d);
  if (dist2 <= 0.0f) return 0.0f;
  const V3 dir = d / sqrtf(dist2);
  const float cos_emit = fmaxf(dot(light.v.ng, dir), 0.0f);
  if (cos_emit <= 0.0f) return 0.0f;
  return solid_angle_to_area(cos_emit / kPiF, light.v.p, target.v.p, target.v.ng);
}
// bdpt.rs:677-715
__device__ __forceinline__ float vertex_pdf_area(const DevRender& S, const BdVertex& from, const BdVertex* prev,
                                                 const BdVertex& target) {
  if (from.flags & kBdLight) return light_emission_pdf(from, target);
  const V3 d = target.v.p - from.v.p;
  if (length_sq(d) <= 0.0f) return 0.0f;
  Vertex v = from.v;
  if (prev) {
    const V3 tp = prev->v.p - from.v.p;
    if (length_sq(tp) <= 0.0f) return 0.0f;
    v.wo = normalize_or_zero(tp);
  }
  const V3 wi = normalize_or_zero(d);
  const DevMaterialRec m = S.d.mats[__ldg(&S.d.inst[from.v.inst].material)];
  return solid_angle_to_area(material_pdf(S, m, v, wi), from.v.p, target.v.p, target.v.ng);
}

// bdpt.rs:717-746
static __device__ __noinline__ float camera_light_hit_mis(const DevRender& S, const BdVertex* cp, uint32_t n) {
  if (n <= 1) return 1.0f;
  const uint32_t pt = n - 1, ptm = pt - 1;
  const float pt_rev = area_light_origin_pdf(S, cp[pt]);
  const float ptm_rev = light_emission_pdf(cp[pt], cp[ptm]);
  float sum = 0.0f, ri = 1.0f;
  for (uint32_t i = n - 1; i >= 1; --i) {
    const float pr = i == pt ? pt_rev : (i == ptm ? ptm_rev : cp[i].pdf_rev);
    ri *= remap0(pr) / remap0(cp[i].pdf_fwd);
    if (!(cp[i].flags & kBdDelta) && !(cp[i - 1].flags & kBdDelta)) sum += ri;
  }
  return 1.0f / (1.0f + fmaxf(sum, 0.0f));
}

// bdpt.rs:748-817 for light_path[0..ns), camera_path[0..nt)
static __device__ __noinline__ float bdpt_mis(const DevRender& S, const BdVertex* lp, uint32_t ns, const BdVertex* cp,
                                              uint32_t nt) {
  if (ns + nt <= 2) return 1.0f;
  const uint32_t qs = ns - 1, pt = nt - 1;
  const BdVertex* qsm = qs >= 1 ? &lp[qs - 1] : nullptr;
  const BdVertex* ptm = pt >= 1 ? &cp[pt - 1] : nullptr;
  const float pt_rev = vertex_pdf_area(S, lp[qs], qsm, cp[pt]);
  const float ptm_rev = ptm ? vertex_pdf_area(S, cp[pt], &lp[qs], *ptm) : 0.0f;
  const float qs_rev = vertex_pdf_area(S, cp[pt], ptm, lp[qs]);
  const float qsm_rev = qsm ? vertex_pdf_area(S, lp[qs], &cp[pt], *qsm) : 0.0f;
  float sum = 0.0f, ri = 1.0f;
  for (uint32_t i = nt - 1; i >= 1; --i) {
    const float pr = i == pt ? pt_rev : ((pt >= 1 && i == pt - 1) ? ptm_rev : cp[i].pdf_rev);
    ri *= remap0(pr) / remap0(cp[i].pdf_fwd);
    if (!(cp[i].flags & kBdDelta) && !(cp[i - 1].flags & kBdDelta)) sum += ri;
  }
  ri = 1.0f;
  for (uint32_t k = ns; k-- > 0;) {
    const float pr = k == qs ? qs_rev : ((qs >= 1 && k == qs - 1) ? qsm_rev : lp[k].pdf_rev);
    ri *= remap0(pr) / remap0(lp[k].pdf_fwd);
    const bool prev_delta = k > 0 && (lp[k - 1].flags & kBdDelta);
    if (!(lp[k].flags & kBdDelta) && !prev_delta) sum += ri;
  }
  return 1.0f / (1.0f + fmaxf(sum, 0.0f));
}

// connect_vertices (bdpt.rs:488-538) up to visible_between (577-602): the
// contribution c if the two vertices see each other (zero when any other test
// already makes it zero), and the visibility ray.  The reference tests
// visibility first; each test here returns zero on its own, so the order does
// not change the result and the shadow ray is traced only for non-zero c --
// except in scenes with alpha tests, where every visibility test draws from
// the sample's AuxRng in connection order, so every pair at a non-zero
// distance traces its ray.  Returns 0: no ray (coincident vertices), 1: a ray
// and zero c, 2: a ray and non-zero c.
struct BdConnection {
  V3 c, origin, dir;
  float dist;
};
__device__ __forceinline__ int bdpt_connect_prepare(const DevRender& S, const BdVertex& lv, const BdVertex& cv,
                                                    BdConnection& out) {
  const V3 delta = cv.v.p - lv.v.p;
  const float dist2 = length_sq(delta);
  if (dist2 <= 0.0f) return 0;
  const float dist = sqrtf(dist2);
  const V3 w_lc = delta / dist;
  const V3 w_cl = -w_lc;
  out.origin = offset_origin(lv.v.p, lv.v.ng, w_lc);
  out.dir = w_lc;
  out.dist = dist;
  out.c = V3{0.0f, 0.0f, 0.0f};
  const DevMaterialRec cm = S.d.mats[__ldg(&S.d.inst[cv.v.inst].material)];
  const V3 f_cam = material_eval(S, cm, cv.v, w_cl, false);
  if (length_sq(f_cam) == 0.0f) return 1;
  V3 f_light;
  if (lv.flags & kBdLight) {
    if (dot(lv.v.ng, w_lc) <= 0.0f) return 1;
    f_light = V3{1.0f, 1.0f, 1.0f};
  } else {
    const DevMaterialRec lm = S.d.mats[__ldg(&S.d.inst[lv.v.inst].material)];
    f_light = material_eval(S, lm, lv.v, w_lc, true);
  }
  if (length_sq(f_light) == 0.0f) return 1;
  const float g = fabsf(dot(lv.v.ng, w_lc)) * fabsf(dot(cv.v.ng, w_cl)) / dist2;
  if (g <= 0.0f) return 1;
  out.c = lv.v.thr * f_light * g * f_cam * cv.v.thr;
  return 2;
}

// The subpaths and connections below are warp-synchronous: every lane of the
// warp calls them (`valid` = the lane holds a sample), lanes step through
// their loops together, and each step traces the rays of the lanes that need
// one at a single call site with the while-while traversal (lanes step through
// interior nodes together before testing leaves).  Each lane's own arithmetic
// and order are those of bdpt.rs.

// State of a camera subpath between the iterations of bdpt.rs's camera loop.
struct BdCamState {
  V3 beta, pending_from;
  float pending_pdf;
  float lock;  // the path's wavelength lock (< 0: none)
  uint32_t n;
  bool count_emission, have_pending, alive;
};
__device__ __forceinline__ void camera_state_init(BdCamState& c, bool valid) {
  c.beta = V3{1.0f, 1.0f, 1.0f};
  c.lock = -1.0f;
  c.pending_from = V3{0.0f, 0.0f, 0.0f};
  c.pending_pdf = 0.0f;
  c.n = 0;
  c.count_emission = true;
  c.have_pending = false;
  c.alive = valid;
}

// One iteration of the camera loop (bdpt.rs:135-262) after its ray (rd) was
// traced to h: the hit vertex into vs[c.n], emission (or, for a ray that left
// the scene, the environment) into L, and the next ray into (ro, rd) while
// c.alive.  In a scene with lights that are not emissive triangles, `nee` says
// whether the vertex took such a light sample (bdpt.rs:207-221): its
// contribution, times the path throughput, counts into L once the shadow ray
// of `dp` is found unoccluded, before the next iteration adds anything.
template <class Stack>
__device__ __forceinline__ void camera_step(const DevRender& S, const RenderLaunch& P, const PathSamplerDev& ps,
                                            uint32_t depth, const TraceResult& h, V3& ro, V3& rd, BdVertex* vs,
                                            BdCamState& c, V3& L, bool& nee, DirectPrep& dp) {
  nee = false;
  if (h.tri < 0) {
    // emitted_radiance_from_infinite_hit (bdpt.rs:466-486)
    if (S.d.has_env) L = L + c.beta * env_escape(S.d, rd, c.count_emission, false, c.pending_pdf);
    c.alive = false;
    return;
  }
  Vertex v = shade_hit<Stack>(S, h, rd);
  v.thr = c.beta;  // the path state the vertex keeps (bdpt.rs:177-178)
  v.lock = c.lock;
  const DevMaterialRec m = S.d.mats[__ldg(&S.d.inst[v.inst].material)];
  BdVertex& pv = vs[c.n];
  pv.v = v;
  pv.pdf_fwd = c.have_pending ? solid_angle_to_area(c.pending_pdf, c.pending_from, v.p, v.ng) : 0.0f;
  pv.pdf_rev = 0.0f;
  pv.flags = m.kind != kDevEmissive ? kBdConnectible : 0u;
  const uint32_t n = ++c.n;
  V3 le;
  if (may_emit(m) && material_le(S, m, v, le)) {
    const float w = c.count_emission ? 1.0f : camera_light_hit_mis(S, vs, n);
    L = L + c.beta * le * w;
  }
  if (m.kind == kDevEmissive) {
    c.alive = false;  // pure emitter: sample() is None
    return;
  }
  if (S.d.num_extra_lights > 0) {  // direct_non_area_light_contribution
    float us0, us1;
    ps.sample_2d(vertex_dim(depth, kOffSurface), us0, us1);
    const float u_tree = ps.sample_1d(vertex_dim(depth, kOffTree));
    const float u_cat = S.d.num_cat > 1 ? ps.sample_1d(vertex_dim(depth, kOffCategory)) : 0.0f;
    nee = prepare_direct<true, kDirectBdptNonArea>(S, m, v, u_cat, u_tree, us0, us1, dp);
    if (nee) dp.contrib = c.beta * dp.contrib;
  }
  float ud0, ud1;
  ps.sample_2d(vertex_dim(depth, kOffDir), ud0, ud1);
  const float u_lobe = m.kind == kDevOpenPbr ? ps.sample_1d(vertex_dim(depth, kOffLobe)) : 0.0f;
  float ux[4];
  extra_randoms(S.d, m, ps, depth, ux);
  MatSample s;
  if (!material_sample_rev(S, m, v, u_lobe, ud0, ud1, ux, false, s)) {
    c.alive = false;
    return;
  }
  if (s.lock >= 0.0f) c.lock = s.lock;
  pv.flags = s.delta ? kBdDelta : kBdConnectible;
  if (n >= 2) vs[n - 2].pdf_rev = solid_angle_to_area(s.pdf_rev, v.p, vs[n - 2].v.p, vs[n - 2].v.ng);
  ro = offset_origin(v.p, v.ng, s.wi);
  rd = s.wi;
  c.beta = c.beta * s.weight;
  if (depth + 1 >= 4) {
    const float q = clampf(max_element(c.beta), 0.05f, 1.0f);
    if (ps.sample_1d(vertex_dim(depth, kOffRr)) > q) {
      c.alive = false;
      return;
    }
    c.beta = c.beta / q;
  }
  c.have_pending = true;
  c.pending_from = v.p;
  c.pending_pdf = s.pdf;
  c.count_emission = s.delta;
}

// Alpha tests (aux non-NULL): one AuxRng per sample through both subpaths,
// each depth reseeding it before its ray (bdpt.rs:160, 335), and then through
// the connections' visibility tests in order (bdpt.rs:81-121).
template <class Stack>
__device__ __forceinline__ uint32_t bdpt_camera_subpath(const DevRender& S, Stack& st, bool valid,
                                                        const RenderLaunch& P, const PathSamplerDev& ps, V3 ro, V3 rd,
                                                        BdVertex* vs, V3& L, uint32_t* err, uint32_t* aux = nullptr) {
  BdCamState c;
  camera_state_init(c, valid);
  for (uint32_t depth = 0; depth < P.max_depth; ++depth) {
    const unsigned live = __ballot_sync(0xffffffffu, c.alive);
    if (!live) break;
    TraceResult h;
    if (aux && c.alive) *aux = aux_from_seed(ps, (int)depth);
    if (c.alive)
      trace_ray_ww<0>(S.geo, st, live, ro.x, ro.y, ro.z, rd.x, rd.y, rd.z, __int_as_float(0x7f800000), h, err, aux);
    bool nee = false;
    DirectPrep dp;
    if (c.alive) camera_step<Stack>(S, P, ps, depth, h, ro, rd, vs, c, L, nee, dp);
    const unsigned sm = __ballot_sync(0xffffffffu, nee);
    if (sm) {  // the light samples' shadow rays (unoccluded, integrator/mod.rs:239-265)
      TraceResult hs;
      if (nee)
        trace_ray_ww<0>(S.geo, st, sm, dp.so.x, dp.so.y, dp.so.z, dp.wi.x, dp.wi.y, dp.wi.z,
                        __int_as_float(0x7f800000), hs, err, aux);
      if (nee && shadow_visible(hs.tri, hs.inst, hs.t, dp.inst, dp.tri, dp.dist)) L = L + dp.contrib;
    }
  }
  return c.n;
}

// sample_area_light_triangle and the light endpoint (bdpt.rs:264-300, 540-553):
// false when the light subpath is empty.
__device__ __forceinline__ bool bdpt_light_endpoint(const DevRender& S, const RenderLaunch& P,
                                                    const PathSamplerDev& ps, BdVertex* vs, V3& ro, V3& rd, V3& beta,
                                                    V3& pending_from, float& pending_pdf) {
  if (P.max_depth == 0 || S.d.num_area_lights == 0 || S.d.area_light_weight_sum <= 0.0f) return false;
  // first prefix >= u * sum
  const float target = clampf(ps.sample_1d(vertex_dim(0, kOffCategory)), 0.0f, 1.0f) * S.d.area_light_weight_sum;
  uint32_t lo = 0, hi = S.d.num_area_lights;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(&S.d.area_lights[mid].prefix_weight) < target) lo = mid + 1;
    else hi = mid;
  }
  const uint32_t k = min(lo, S.d.num_area_lights - 1);
  const DevAreaLight al = S.d.area_lights[k];
  const float pmf = al.weight / S.d.area_light_weight_sum;
  TriData T;
  fetch_triangle(S, al.inst, al.tri, T, true);
  float us0, us1;
  ps.sample_2d(vertex_dim(0, kOffSurface), us0, us1);
  const float su0 = sqrtf(clampf(us0, 0.0f, 1.0f));
  const float u1 = clampf(us1, 0.0f, 1.0f);
  const float b0 = 1.0f - su0, b1 = u1 * su0, b2 = (1.0f - u1) * su0;
  const float area = 0.5f * length(cross(T.p[1] - T.p[0], T.p[2] - T.p[0]));
  const float pdf_point = area > 0.0f ? 1.0f / area : 0.0f;
  const float pdf_area = pmf * pdf_point;
  if (pdf_area <= 0.0f) return false;
  const V3 gn = normalize_or_zero(cross(T.p[1] - T.p[0], T.p[2] - T.p[0]));
  const Frame fr = frame_from_normal(gn);
  float ud0, ud1;
  ps.sample_2d(vertex_dim(0, kOffDir), ud0, ud1);
  const V3 ld = opbr::sample_cosine_hemisphere(ud0, ud1);
  const V3 emit = normalize_or_zero(to_world(fr, ld));
  const float pdf_dir = fmaxf(ld.z, 0.0f) / kPiF;
  if (length_sq(emit) == 0.0f || pdf_dir <= 0.0f) return false;
  Vertex lvx = make_vertex(T, al.inst, al.tri, b0, b1, b2, -emit);
  lvx.wo = emit;
  const DevMaterialRec lm = S.d.mats[__ldg(&S.d.inst[al.inst].material)];
  V3 le;
  if (!may_emit(lm) || !material_le(S, lm, lvx, le)) return false;  // le() is None
  const float cos_emit = fmaxf(dot(lvx.ng, emit), 0.0f);
  if (cos_emit <= 0.0f) return false;
  const V3 endpoint_beta = le / pdf_area;
  vs[0].v = lvx;
  vs[0].v.thr = endpoint_beta;
  vs[0].pdf_fwd = pdf_area;
  vs[0].pdf_rev = 0.0f;
  vs[0].flags = kBdLight | kBdConnectible;
  ro = offset_origin(lvx.p, lvx.ng, emit);
  rd = emit;
  beta = endpoint_beta * (cos_emit / pdf_dir);
  pending_from = lvx.p;
  pending_pdf = pdf_dir;
  return true;
}

// State of a light subpath between the iterations of bdpt.rs's light loop.
struct BdLightState {
  V3 beta, pending_from;
  float pending_pdf;
  float lock;  // the path's wavelength lock (< 0: none)
  uint32_t n;
  bool alive;
};

static_assert(sizeof(BdCamState) <= kBdStateBytes && sizeof(BdLightState) <= kBdStateBytes, "BDPT loop states");

// One iteration of the light loop (bdpt.rs:264-385) after its ray was traced to h.
template <class Stack>
__device__ __forceinline__ void light_step(const DevRender& S, const PathSamplerDev& ps, uint32_t depth,
                                           const TraceResult& h, V3& ro, V3& rd, BdVertex* vs, BdLightState& l) {
  if (h.tri < 0) {
    l.alive = false;
    return;
  }
  Vertex v = shade_hit<Stack>(S, h, rd);
  v.thr = l.beta;  // bdpt.rs:344-345
  v.lock = l.lock;
  const DevMaterialRec m = S.d.mats[__ldg(&S.d.inst[v.inst].material)];
  BdVertex& pv = vs[l.n];
  pv.v = v;
  pv.pdf_fwd = solid_angle_to_area(l.pending_pdf, l.pending_from, v.p, v.ng);
  pv.pdf_rev = 0.0f;
  pv.flags = m.kind != kDevEmissive ? kBdConnectible : 0u;
  const uint32_t n = ++l.n;
  if (m.kind == kDevEmissive) {
    l.alive = false;
    return;
  }
  float ud0, ud1;
  ps.sample_2d(vertex_dim(depth, kOffDir), ud0, ud1);
  const float u_lobe = m.kind == kDevOpenPbr ? ps.sample_1d(vertex_dim(depth, kOffLobe)) : 0.0f;
  float ux[4];
  extra_randoms(S.d, m, ps, depth, ux);
  MatSample s;
  if (!material_sample_rev(S, m, v, u_lobe, ud0, ud1, ux, true, s)) {
    l.alive = false;
    return;
  }
  if (s.lock >= 0.0f) l.lock = s.lock;
  pv.flags = s.delta ? kBdDelta : kBdConnectible;
  vs[n - 2].pdf_rev = solid_angle_to_area(s.pdf_rev, v.p, vs[n - 2].v.p, vs[n - 2].v.ng);
  ro = offset_origin(v.p, v.ng, s.wi);
  rd = s.wi;
  l.beta = l.beta * s.weight;
  l.pending_from = v.p;
  l.pending_pdf = s.pdf;
}

template <class Stack>
__device__ __forceinline__ uint32_t bdpt_light_subpath(const DevRender& S, Stack& st, bool valid,
                                                       const RenderLaunch& P, const PathSamplerDev& ps, BdVertex* vs,
                                                       uint32_t* err, uint32_t* aux = nullptr) {
  V3 ro, rd;
  BdLightState l;
  l.pending_pdf = 0.0f;
  l.lock = -1.0f;
  l.alive = valid && bdpt_light_endpoint(S, P, ps, vs, ro, rd, l.beta, l.pending_from, l.pending_pdf);
  l.n = l.alive ? 1u : 0u;
  for (uint32_t depth = 1; depth < P.max_depth; ++depth) {
    const unsigned live = __ballot_sync(0xffffffffu, l.alive);
    if (!live) break;
    TraceResult h;
    if (aux && l.alive) *aux = aux_from_seed(ps, (int)depth);
    if (l.alive)
      trace_ray_ww<0>(S.geo, st, live, ro.x, ro.y, ro.z, rd.x, rd.y, rd.z, __int_as_float(0x7f800000), h, err, aux);
    if (l.alive) light_step<Stack>(S, ps, depth, h, ro, rd, vs, l);
  }
  return l.n;
}

// bdpt::trace_radiance for one sample (bdpt.rs:70-131), warp-synchronous.  The
// connections run over k = li * nc + ci in the reference's (light, camera)
// order; their MIS weights are finite (in [0, 1]), so a zero connection adds
// exactly zero and is skipped with its visibility ray and pdfs.
template <class Stack>
__device__ V3 trace_bdpt(const DevRender& S, Stack& st, bool valid, const RenderLaunch& P, const PathSamplerDev& ps,
                         V3 ro, V3 rd, uint32_t* err) {
  BdVertex cam[kBdptMaxDepth], lig[kBdptMaxDepth];
  V3 L = V3{0.0f, 0.0f, 0.0f};
  const bool alpha = S.geo.inst_alpha != nullptr;
  uint32_t aux_state = alpha ? aux_from_seed(ps, -1) : 0u;
  uint32_t* aux = alpha ? &aux_state : nullptr;
  const uint32_t nc = bdpt_camera_subpath(S, st, valid, P, ps, ro, rd, cam, L, err, aux);
  const uint32_t nl = bdpt_light_subpath(S, st, valid, P, ps, lig, err, aux);
  const uint32_t np = valid ? nl * nc : 0u;
  const uint32_t max_np = __reduce_max_sync(0xffffffffu, np);
  for (uint32_t k = 0; k < max_np; ++k) {
    bool want = false;
    int prep = 0;
    BdConnection cn;
    uint32_t li = 0, ci = 0;
    if (k < np) {
      li = k / nc;
      ci = k - li * nc;
      if ((lig[li].flags & kBdConnectible) && (cam[ci].flags & kBdConnectible)) {
        prep = bdpt_connect_prepare(S, lig[li], cam[ci], cn);
        want = prep == 2 || (alpha && prep == 1);
      }
    }
    const unsigned tm = __ballot_sync(0xffffffffu, want);
    if (!tm) continue;
    TraceResult h;
    if (want)
      trace_ray_ww<0>(S.geo, st, tm, cn.origin.x, cn.origin.y, cn.origin.z, cn.dir.x, cn.dir.y, cn.dir.z,
                      __int_as_float(0x7f800000), h, err, aux);
    if (!want || prep != 2) continue;
    // visible_between (bdpt.rs:577-602)
    if (h.tri >= 0) {
      const bool target = (uint32_t)h.inst == cam[ci].v.inst && (uint32_t)h.tri == cam[ci].v.tri;
      if (!target && !(h.t >= cn.dist * (1.0f - kShadowTolerance))) continue;
    }
    const float w = bdpt_mis(S, lig, li + 1, cam, ci + 1);
    L = L + w * cn.c;
  }
  return L;
}

}  // namespace tpt
