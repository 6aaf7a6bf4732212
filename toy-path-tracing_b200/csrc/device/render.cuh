// Per-sample rendering on the device: camera ray, shading vertex, NEE through
// the SG light tree and BSDF sampling, the pieces the MIS path loop of the
// megakernel (render_kernels.cu) and of the wavefront stages
// (wavefront_kernels.cu) are built from.
//
// Restates crates/renderer/src/{scene/camera.rs, scene/mod.rs:471-635,
// light/{mod,area}.rs, material/{mod,normalized_lambert,emissive}.rs,
// bsdf/normalized_lambert.rs, integrator/{mod,mis}.rs}.  Ray differentials and
// cones are not carried: they only feed texture filtering and specular
// differentials, which no material in scope reads.
#pragma once
#include "batch_types.h"
#include "lights.cuh"
#include "openpbr.cuh"
#include "render_types.h"
#include "sampler.cuh"
#include "trace.cuh"
#include "vmath.cuh"

namespace tpt {

struct Ray3 {
  V3 o, d;
};

// sample_tent_1d (math/mod.rs:17-24)
__device__ __forceinline__ float tent(float u) {
  u = clampf(u, 0.0f, 1.0f);
  if (u < 0.5f) return sqrtf(2.0f * u) - 1.0f;
  return 1.0f - sqrtf(2.0f - 2.0f * u);
}

// PinholeCamera::direction_for_sample (camera.rs:75-82)
__device__ __forceinline__ V3 camera_dir(const DevCamera& c, uint32_t rx, uint32_t ry, float px, float py) {
  const float fx = (float)rx, fy = (float)ry;
  const float aspect = fx / fy;
  const float sx = ((2.0f * px / fx) - 1.0f) * aspect * c.tan_half_fov_y;
  const float sy = (1.0f - (2.0f * py / fy)) * c.tan_half_fov_y;
  const V3 f = V3{c.forward[0], c.forward[1], c.forward[2]};
  const V3 r = V3{c.right[0], c.right[1], c.right[2]};
  const V3 u = V3{c.up[0], c.up[1], c.up[2]};
  return normalize(f + sx * r + sy * u);
}

// ---------------------------------------------------------------------------
// Shading vertex (scene/mod.rs:471-544) restricted to what the materials read.
struct Vertex {
  V3 p, ng, ns, wo;
  Frame frame;
  uint32_t inst, tri;
  bool front;  // geometric normal faces the incoming ray (ShadingVertex::front_face)
};

struct TriData {
  V3 p[3];
  V3 n[3];
  float u[3], v[3];
};

__device__ __forceinline__ void fetch_triangle(const DevRender& S, uint32_t inst, uint32_t tri, TriData& T,
                                               bool want_shading) {
  const DevShadeInstance* I = S.d.inst + inst;
  const DevMeshInfo M = S.d.meshes[__ldg(&I->mesh)];
  float l2w[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) l2w[k] = __ldg(&I->l2w[k]);
  uint32_t vi[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) vi[k] = M.vtx_base + __ldg(S.d.idx + M.idx_base + 3 * tri + k);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const V3 lp = V3{__ldg(S.d.pos + 3 * vi[k]), __ldg(S.d.pos + 3 * vi[k] + 1), __ldg(S.d.pos + 3 * vi[k] + 2)};
    T.p[k] = xform_point(l2w, lp);
  }
  if (!want_shading) return;
  float n2w[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) n2w[k] = __ldg(&I->n2w[k]);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    V3 ln = V3{0.0f, 0.0f, 0.0f};
    if (M.flags & 1u) ln = V3{__ldg(S.d.nrm + 3 * vi[k]), __ldg(S.d.nrm + 3 * vi[k] + 1), __ldg(S.d.nrm + 3 * vi[k] + 2)};
    T.n[k] = normalize_or_zero(mat3_mul(n2w, ln));
    T.u[k] = (M.flags & 2u) ? __ldg(S.d.uv + 2 * vi[k]) : 0.0f;
    T.v[k] = (M.flags & 2u) ? __ldg(S.d.uv + 2 * vi[k] + 1) : 0.0f;
  }
}

// compute_surface_partials (math/mod.rs:112-134) for positions -> dpdu
__device__ __forceinline__ bool surface_dpdu(const TriData& T, V3& dpdu) {
  const V3 dp1 = T.p[1] - T.p[0], dp2 = T.p[2] - T.p[0];
  const float du1 = T.u[1] - T.u[0], dv1 = T.v[1] - T.v[0];
  const float du2 = T.u[2] - T.u[0], dv2 = T.v[2] - T.v[0];
  const float det = du1 * dv2 - dv1 * du2;
  if (fabsf(det) <= 1.0e-8f) return false;
  const float inv = 1.0f / det;
  dpdu = (dv2 * dp1 - dv1 * dp2) * inv;
  const V3 dpdv = (-du2 * dp1 + du1 * dp2) * inv;
  return !(length_sq(dpdu) == 0.0f || length_sq(dpdv) == 0.0f);
}

__device__ __forceinline__ Vertex make_vertex(const TriData& T, uint32_t inst, uint32_t tri, float b0, float b1,
                                              float b2, V3 incident) {
  Vertex v;
  v.inst = inst;
  v.tri = tri;
  const V3 b = V3{b0, b1, b2};
  v.p = interp3(b, T.p[0], T.p[1], T.p[2]);
  const V3 gn = normalize_or_zero(cross(T.p[1] - T.p[0], T.p[2] - T.p[0]));
  const V3 sn = normalize_or_zero(interp3(b, T.n[0], T.n[1], T.n[2]));
  const V3 minus_in = -incident;
  v.front = dot(gn, minus_in) >= 0.0f;
  v.ng = face_forward(gn, minus_in);
  const V3 raw_ns = length_sq(sn) > 0.0f ? sn : v.ng;
  v.ns = face_forward(raw_ns, v.ng);
  V3 dpdu;
  if (!surface_dpdu(T, dpdu)) dpdu = frame_from_normal(v.ns).t;
  v.frame = frame_from_normal_tangent(v.ns, dpdu);
  v.wo = normalize_or_zero(minus_in);
  return v;
}

// ---------------------------------------------------------------------------
// Materials (material/mod.rs:33-79, normalized_lambert.rs, emissive.rs)
constexpr float kGeomCosEps = 1.0e-6f;

struct BsdfSampleOut {
  V3 weight, wi;
  float pdf;
  bool delta;
};

__device__ __forceinline__ V3 lambert_eval(const DevMaterialRec& m, const Vertex& v, V3 wi) {
  if (dot(v.wo, v.ng) <= 0.0f || dot(wi, v.ng) <= 0.0f) return V3{0, 0, 0};
  const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
  const V3 wi_l = normalize_or_zero(to_local(v.frame, wi));
  V3 f = V3{0, 0, 0};
  if (!(wo_l.z <= 0.0f || wi_l.z <= 0.0f)) f = V3{m.rho[0], m.rho[1], m.rho[2]} / kPiF;
  // modified_bsdf_eval, radiance transport
  if (length_sq(f) == 0.0f) return V3{0, 0, 0};
  const float cos_geom = fabsf(dot(wi, v.ng));
  if (cos_geom <= kGeomCosEps) return V3{0, 0, 0};
  return f * (fabsf(dot(wi, v.ns)) / cos_geom);
}

__device__ __forceinline__ float lambert_pdf(const Vertex& v, V3 wi) {
  if (dot(v.wo, v.ng) <= 0.0f || dot(wi, v.ng) <= 0.0f) return 0.0f;
  const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
  const V3 wi_l = normalize_or_zero(to_local(v.frame, wi));
  if (wo_l.z <= 0.0f || wi_l.z <= 0.0f) return 0.0f;
  return fmaxf(wi_l.z, 0.0f) / kPiF;
}

__device__ __forceinline__ bool lambert_sample(const DevMaterialRec& m, const Vertex& v, float u0, float u1,
                                               BsdfSampleOut& s) {
  const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
  if (wo_l.z <= 0.0f) return false;
  // sample_cosine_weighted_hemisphere (math/mod.rs:26-36)
  const float r = sqrtf(clampf(u0, 0.0f, 1.0f));
  const float phi = kTauF * u1;
  const float dx = r * cosf(phi), dy = r * sinf(phi);
  const float z = sqrtf(fmaxf(1.0f - (dx * dx + dy * dy), 0.0f));
  const V3 wi_l = V3{dx, dy, z};
  const float pdf = fmaxf(wi_l.z, 0.0f) / kPiF;
  if (pdf <= 0.0f) return false;
  s.wi = to_world(v.frame, wi_l);
  s.weight = V3{m.rho[0], m.rho[1], m.rho[2]};
  s.pdf = pdf;
  s.delta = false;
  return dot(s.wi, v.ng) > kGeomCosEps;
}

// OpenPbrMaterial::sample (material/open_pbr.rs:489-563) in radiance transport
// (modified_bsdf_sample_weight leaves the weight unchanged there).
static __device__ __noinline__ bool openpbr_sample(const DevRenderData& d, uint32_t opbr_index, const Vertex& v,
                                            float u_lobe, float u0, float u1, BsdfSampleOut& s) {
  if (dot(v.wo, v.ng) <= 0.0f) return false;
  const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
  if (wo_l.z <= 0.0f) return false;
  opbr::OpbrVertex ov;
  opbr::init_vertex(ov, d.openpbr + opbr_index, d.cec_e, d.dec_e, wo_l, v.front, fabsf(wo_l.z));
  opbr::Sample bs;
  if (!opbr::sample(ov, u_lobe, u0, u1, bs)) return false;
  const V3 wi = to_world(v.frame, bs.wi);
  if (dot(wi, v.ng) <= kGeomCosEps) return false;  // reflection lobes only
  s.wi = wi;
  s.weight = bs.weight;
  s.pdf = bs.pdf;
  s.delta = (bs.flags & opbr::kFlagDelta) != 0;
  return true;
}

// Material::sample for the BSDF materials in scope, with the vertex's
// MaterialSampleRandoms (lobe at offset 5, direction at offset 7).
__device__ __forceinline__ bool material_sample(const DevRender& S, const DevMaterialRec& m, const Vertex& v,
                                                const PathSamplerDev& ps, uint32_t depth, BsdfSampleOut& s) {
  float ud0, ud1;
  ps.sample_2d(vertex_dim(depth, kOffDir), ud0, ud1);
  if (m.kind == kDevOpenPbr) {
    const float u_lobe = ps.sample_1d(vertex_dim(depth, kOffLobe));
    return openpbr_sample(S.d, m.openpbr, v, u_lobe, ud0, ud1, s);
  }
  return lambert_sample(m, v, ud0, ud1, s);
}

// ---------------------------------------------------------------------------
// Light sampling (light/mod.rs:296-340, light/area.rs:12-56, scene/mod.rs:583-635)
struct LightSample {
  V3 radiance, wi;
  float pdf, distance;
  uint32_t inst, tri;
};

__device__ __forceinline__ V3 emissive_le(const DevMaterialRec& m) {
  return V3{m.color[0] * m.strength, m.color[1] * m.strength, m.color[2] * m.strength};
}

__device__ __forceinline__ bool sample_li_triangle(const DevRender& S, uint32_t inst, uint32_t tri, V3 p_ref, float us0,
                                                   float us1, LightSample& out) {
  TriData T;
  fetch_triangle(S, inst, tri, T, false);
  const float su0 = sqrtf(clampf(us0, 0.0f, 1.0f));
  const float u1 = clampf(us1, 0.0f, 1.0f);
  const V3 b = V3{1.0f - su0, u1 * su0, (1.0f - u1) * su0};
  const V3 p = interp3(b, T.p[0], T.p[1], T.p[2]);
  const float area = 0.5f * length(cross(T.p[1] - T.p[0], T.p[2] - T.p[0]));
  const float pdf_area = area > 0.0f ? 1.0f / area : 0.0f;
  if (pdf_area <= 0.0f) return false;
  const V3 to_light = p - p_ref;
  const float d2 = length_sq(to_light);
  if (d2 <= 0.0f) return false;
  const float dist = sqrtf(d2);
  const V3 wi = to_light / dist;
  const DevMaterialRec lm = S.d.mats[__ldg(&S.d.inst[inst].material)];
  if (lm.kind != kDevEmissive) return false;  // may_emit
  const V3 gn = normalize_or_zero(cross(T.p[1] - T.p[0], T.p[2] - T.p[0]));
  const V3 ng = face_forward(gn, -wi);
  const float cos_light = fmaxf(dot(ng, -wi), 0.0f);
  if (cos_light <= 0.0f) return false;
  out.radiance = emissive_le(lm);
  out.wi = wi;
  out.pdf = pdf_area * d2 / cos_light;
  out.distance = dist;
  out.inst = inst;
  out.tri = tri;
  return true;
}

// spawn_ray / offset_ray_origin (integrator/mod.rs:52-85)
__device__ __forceinline__ V3 offset_origin(V3 p, V3 ng, V3 dir) {
  const V3 n = dot(dir, ng) >= 0.0f ? ng : -ng;
  return p + 1.0e-4f * n;
}

// direct_light_mis_contribution (integrator/mis.rs:145-210) for a diffuse
// vertex, up to the visibility test: returns false when the contribution is
// zero whatever the visibility; otherwise `contrib` (radiance * f * cos * mis /
// pdf) counts iff the shadow ray (so, li.wi) first hits triangle (inst, tri).
struct DirectPrep {
  V3 contrib, so, wi;
  uint32_t inst, tri;
};

__device__ __forceinline__ bool prepare_direct(const DevRender& S, const DevMaterialRec& m, const Vertex& v,
                                               float u_tree, float us0, float us1, DirectPrep& out) {
  if (!S.d.has_tree) return false;              // LightSampler::sample_category: no category
  if (m.kind != kDevLambert) return false;      // only the diffuse material builds a light-tree query
  TreeQuery q;
  q.rho = luminance(V3{m.rho[0], m.rho[1], m.rho[2]});
  if (q.rho <= 0.0f) return false;
  q.p = v.p;
  q.n = v.ns;
  float leaf_pmf;
  const uint32_t leaf = sample_light_tree(S.d.ltree, S.d.ltree_root, q, u_tree, leaf_pmf);
  if (leaf == 0xFFFFFFFFu) return false;
  LightSample li;
  if (!sample_li_triangle(S, __ldg(&S.d.ltree[leaf].leaf_instance), __ldg(&S.d.ltree[leaf].leaf_triangle), v.p, us0,
                          us1, li))
    return false;
  const float sel_pmf = S.d.tree_cat_pmf * leaf_pmf;
  if (li.pdf <= 0.0f || sel_pmf <= 0.0f) return false;
  const V3 f = lambert_eval(m, v, li.wi);
  if (length_sq(f) == 0.0f) return false;
  const float bsdf_pdf = lambert_pdf(v, li.wi);
  const float cos_surface = fabsf(dot(v.ng, li.wi));
  if (cos_surface <= 0.0f) return false;
  const float pdf_total = sel_pmf * li.pdf;
  if (pdf_total <= 0.0f) return false;
  const float mis = balance_heuristic(pdf_total, bsdf_pdf);
  out.contrib = li.radiance * f * (cos_surface * mis / pdf_total);
  out.so = offset_origin(v.p, v.ng, li.wi);  // spawn_ray of unoccluded_ray (integrator/mod.rs:239-265)
  out.wi = li.wi;
  out.inst = li.inst;
  out.tri = li.tri;
  return true;
}

// pdf_for_triangle_hit (light/mod.rs:416-437) for a BSDF-sampled emitter hit
__device__ __forceinline__ float light_pdf_for_hit(const DevRender& S, const DevMaterialRec& shading_mat,
                                                   const Vertex& v, const Vertex& lv) {
  if (!S.d.has_tree || shading_mat.kind != kDevLambert) return 0.0f;
  TreeQuery q;
  q.rho = luminance(V3{shading_mat.rho[0], shading_mat.rho[1], shading_mat.rho[2]});
  if (q.rho <= 0.0f) return 0.0f;
  q.p = v.p;
  q.n = v.ns;
  const uint32_t base = __ldg(&S.d.inst[lv.inst].leaf_base);
  if (base == 0xFFFFFFFFu) return 0.0f;
  const uint32_t leaf = __ldg(S.d.emitter_leaf + base + lv.tri);
  if (leaf == 0xFFFFFFFFu) return 0.0f;
  const float leaf_pmf = pdf_for_leaf(S.d.ltree, q, leaf);
  if (leaf_pmf <= 0.0f) return 0.0f;
  // area_light_pdf_solid_angle (scene/mod.rs:596-618)
  const float area = __ldg(&S.d.ltree[leaf].area);
  if (area <= 0.0f) return 0.0f;
  const float pdf_area = 1.0f / area;
  const V3 to_light = lv.p - v.p;
  const float d2 = length_sq(to_light);
  if (d2 <= 0.0f) return 0.0f;
  const float dist = sqrtf(d2);
  const V3 wi = to_light / dist;
  const float cos_light = fmaxf(dot(lv.ng, -wi), 0.0f);
  if (cos_light <= 0.0f) return 0.0f;
  return S.d.tree_cat_pmf * leaf_pmf * (pdf_area * d2 / cos_light);
}

template <class Stack>
__device__ __forceinline__ Vertex shade_hit(const DevRender& S, const TraceResult& h, V3 incident) {
  TriData T;
  fetch_triangle(S, (uint32_t)h.inst, (uint32_t)h.tri, T, true);
  return make_vertex(T, (uint32_t)h.inst, (uint32_t)h.tri, h.b0, h.b1, h.b2, incident);
}

}  // namespace tpt
