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
#include "environment.cuh"
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
  // ShadingVertex::wavelength_lock (< 0: none) and path_throughput: the path
  // state the integrators stamp on the vertex before shading it (read by
  // dispersive transmission only)
  float lock;
  V3 thr;
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
  v.lock = -1.0f;
  v.thr = V3{1.0f, 1.0f, 1.0f};
  return v;
}

// ---------------------------------------------------------------------------
// Materials (material/mod.rs:33-79, normalized_lambert.rs, emissive.rs)
constexpr float kGeomCosEps = 1.0e-6f;

struct BsdfSampleOut {
  V3 weight, wi;
  float pdf;
  bool delta;
  float lock;  // the wavelength the sample locks the path to (< 0: none)
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
  s.lock = -1.0f;
  return dot(s.wi, v.ng) > kGeomCosEps;
}

// material/open_pbr.rs:523-531: a transmitted direction must leave below the
// geometric surface (a delta transmission is kept either way), a reflected one
// above it.
__device__ __forceinline__ bool opbr_sample_side_ok(const Vertex& v, V3 wi, uint32_t flags) {
  if (flags & opbr::kFlagTransmission) return !(dot(wi, v.ng) >= -kGeomCosEps && !(flags & opbr::kFlagDelta));
  return dot(wi, v.ng) > kGeomCosEps;
}

// OpenPbrMaterial::sample (material/open_pbr.rs:489-563) in radiance transport
// (modified_bsdf_sample_weight leaves the weight unchanged there).
static __device__ __noinline__ bool openpbr_sample(const DevRenderData& d, uint32_t opbr_index, const Vertex& v,
                                            float u_lobe, float u0, float u1, const float* ux, BsdfSampleOut& s) {
  if (dot(v.wo, v.ng) <= 0.0f) return false;
  const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
  if (wo_l.z <= 0.0f) return false;
  opbr::OpbrVertex ov;
  opbr::init_vertex(ov, d.openpbr + opbr_index, d.cec_e, d.dec_e, wo_l, v.front, fabsf(wo_l.z));
  ov.thr = v.thr;
  ov.lock = v.lock;
  opbr::Sample bs;
  if (!opbr::sample(ov, u_lobe, u0, u1, bs, false, false, ux)) return false;
  const V3 wi = to_world(v.frame, bs.wi);
  if (!opbr_sample_side_ok(v, wi, bs.flags)) return false;
  s.wi = wi;
  s.weight = bs.weight;
  s.pdf = bs.pdf;
  s.delta = (bs.flags & opbr::kFlagDelta) != 0;
  s.lock = bs.lock;
  return true;
}

// AuxRng::from_seed (aux_rng.rs:15-19) of the vertex's seed (path_sampler.rs:
// offset 14) or, for `depth` < 0, of initial_aux_rng_seed (dimension 0x80000000)
__device__ __forceinline__ uint32_t aux_from_seed(const PathSamplerDev& ps, int depth) {
  return pcg_state_transition(ps.aux_rng_seed(depth < 0 ? 0x80000000u : vertex_dim((uint32_t)depth, kOffAuxSeed)));
}

// MaterialSampleRandoms::u_extra0..3 (offsets 9-12), drawn only for a
// dispersive material (the only reader); zeros otherwise.
__device__ __forceinline__ void extra_randoms(const DevRenderData& d, const DevMaterialRec& m,
                                              const PathSamplerDev& ps, uint32_t depth, float* ux) {
  ux[0] = ux[1] = ux[2] = ux[3] = 0.0f;
  if (m.kind != kDevOpenPbr || !(d.openpbr[m.openpbr].flags & kOpbrDisp)) return;
  ux[0] = ps.sample_1d(vertex_dim(depth, kOffExtra0));
  ux[1] = ps.sample_1d(vertex_dim(depth, kOffExtra1));
  ux[2] = ps.sample_1d(vertex_dim(depth, kOffExtra2));
  ux[3] = ps.sample_1d(vertex_dim(depth, kOffExtra3));
}

// Material::sample for the BSDF materials in scope, with the vertex's
// MaterialSampleRandoms (lobe at offset 5, direction at offset 7).
__device__ __forceinline__ bool material_sample(const DevRender& S, const DevMaterialRec& m, const Vertex& v,
                                                const PathSamplerDev& ps, uint32_t depth, BsdfSampleOut& s) {
  float ud0, ud1;
  ps.sample_2d(vertex_dim(depth, kOffDir), ud0, ud1);
  if (m.kind == kDevOpenPbr) {
    const float u_lobe = ps.sample_1d(vertex_dim(depth, kOffLobe));
    float ux[4];
    extra_randoms(S.d, m, ps, depth, ux);
    return openpbr_sample(S.d, m.openpbr, v, u_lobe, ud0, ud1, ux, s);
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

// Material::may_emit: the emissive material, and OpenPBR with emission_luminance > 0
// (emissive.rs, material/open_pbr.rs:377-379)
__device__ __forceinline__ bool may_emit(const DevMaterialRec& m) { return m.kind == kDevEmissive || m.emits != 0u; }

// OpenPBR emission leaving through the coat and fuzz layers
// (emission_exit_tint, material/open_pbr.rs:608-638, untextured): the coat's
// absorption along the refracted exit path, lerped by the coat weight, times
// the energy the fuzz lobe leaves, lerped by the fuzz weight.
__device__ __forceinline__ V3 openpbr_exit_tint(const DevOpenPbr& d, const Vertex& v) {
  const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
  const float cos_o = clampf(fabsf(wo_l.z), 0.0f, 1.0f);
  if (cos_o <= 0.0f) return V3{0.0f, 0.0f, 0.0f};
  V3 tint = V3{1.0f, 1.0f, 1.0f};
  if (d.coat > 0.0f) {  // coat weight, clamped to [0, 1]; coat_color clamped to [0, 1]
    const float eta = d.coat_eta;
    const float mu_t = fmaxf(sqrtf(fmaxf(1.0f - (1.0f - cos_o * cos_o) / (eta * eta), 0.0f)), 1.0e-4f);
    const float e = 1.0f / mu_t;
    const V3 trans = V3{powf(d.coat_color[0], e), powf(d.coat_color[1], e), powf(d.coat_color[2], e)};
    tint = tint * (V3{1.0f, 1.0f, 1.0f} + (trans - V3{1.0f, 1.0f, 1.0f}) * d.coat);
  }
  if (d.fuzz > 0.0f) {
    const float e_fuzz = opbr::zeltner_albedo(cos_o, d.fuzz_roughness);
    const float t = 1.0f + (fmaxf(1.0f - e_fuzz, 0.0f) - 1.0f) * d.fuzz;
    tint = tint * V3{t, t, t};
  }
  return tint;
}

// Material::le (emissive.rs:68-85, material/open_pbr.rs:351-375, untextured):
// the emissive material radiates colour * strength from both faces; an OpenPBR
// emitter radiates emission_color * emission_luminance from its front face
// (both faces when thin-walled), tinted by the layers above it.  False: no
// emission at this vertex.
__device__ __forceinline__ bool material_le(const DevRender& S, const DevMaterialRec& m, const Vertex& v, V3& le) {
  if (m.kind == kDevEmissive) {
    le = V3{m.color[0] * m.strength, m.color[1] * m.strength, m.color[2] * m.strength};
    return true;
  }
  if (!m.emits) return false;
  const DevOpenPbr& d = S.d.openpbr[m.openpbr];
  if (!(d.flags & kOpbrThinWalled) && !v.front) return false;
  const float lum = fmaxf(m.strength, 0.0f);
  le = V3{m.color[0], m.color[1], m.color[2]} * lum * openpbr_exit_tint(d, v);
  return true;
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
  if (!may_emit(lm)) return false;
  V3 ng;
  if (lm.kind == kDevEmissive) {
    out.radiance = V3{lm.color[0] * lm.strength, lm.color[1] * lm.strength, lm.color[2] * lm.strength};
    ng = face_forward(normalize_or_zero(cross(T.p[1] - T.p[0], T.p[2] - T.p[0])), -wi);
  } else {
    // the light's shading vertex, seen from p_ref, decides the face and the exit tint
    fetch_triangle(S, inst, tri, T, true);
    const Vertex lv = make_vertex(T, inst, tri, b.x, b.y, b.z, wi);
    if (!material_le(S, lm, lv, out.radiance)) return false;
    ng = lv.ng;
  }
  const float cos_light = fmaxf(dot(ng, -wi), 0.0f);
  if (cos_light <= 0.0f) return false;
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

// ---- material eval with transport modes (material/mod.rs:33-79) -------------
__device__ __forceinline__ V3 modified_eval(const Vertex& v, V3 wi, V3 f, bool importance) {
  if (length_sq(f) == 0.0f) return V3{0.0f, 0.0f, 0.0f};
  const V3 dir = importance ? v.wo : wi;
  const float cos_geom = fabsf(dot(dir, v.ng));
  if (cos_geom <= kGeomCosEps) return V3{0.0f, 0.0f, 0.0f};
  return f * (fabsf(dot(dir, v.ns)) / cos_geom);
}

// Material::eval (NormalizedLambert, OpenPbr; zero for the pure emitter)
static __device__ __noinline__ V3 material_eval(const DevRender& S, const DevMaterialRec& m, const Vertex& v, V3 wi,
                                               bool importance) {
  if (m.kind == kDevLambert) {
    if (dot(v.wo, v.ng) <= 0.0f || dot(wi, v.ng) <= 0.0f) return V3{0.0f, 0.0f, 0.0f};
    const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
    const V3 wi_l = normalize_or_zero(to_local(v.frame, wi));
    V3 f = V3{0.0f, 0.0f, 0.0f};
    if (!(wo_l.z <= 0.0f || wi_l.z <= 0.0f)) f = V3{m.rho[0], m.rho[1], m.rho[2]} / kPiF;
    return modified_eval(v, wi, f, importance);
  }
  if (m.kind == kDevOpenPbr) {
    if (dot(v.wo, v.ng) <= 0.0f) return V3{0.0f, 0.0f, 0.0f};
    const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
    const V3 wi_l = normalize_or_zero(to_local(v.frame, wi));
    if (wo_l.z <= 0.0f) return V3{0.0f, 0.0f, 0.0f};
    const DevOpenPbr* mp = S.d.openpbr + m.openpbr;
    opbr::OpbrVertex s;
    opbr::init_vertex(s, mp, S.d.cec_e, S.d.dec_e, wo_l, v.front, fabsf(wo_l.z));
    s.thr = v.thr;
    s.lock = v.lock;
    V3 f;
    float pdf;
    if (importance) {
      opbr::OpbrVertex lay;
      opbr::init_vertex(lay, mp, S.d.cec_e, S.d.dec_e, wi_l, v.front, fabsf(wo_l.z));
      lay.thr = v.thr;
      lay.lock = v.lock;
      opbr::eval_pdf(s, lay, wi_l, f, pdf, true, true);
    } else {
      opbr::eval_pdf(s, s, wi_l, f, pdf);
    }
    return modified_eval(v, wi, f, importance);
  }
  return V3{0.0f, 0.0f, 0.0f};
}

// ---- lights that are not emissive triangles (light/{point,spot,directional}.rs)
constexpr float kShadowTolerance = 1.0e-3f;  // integrator/mod.rs:50

// point::sample_li (light/point.rs:32-50): Li = color * P / (4 pi r^2)
__device__ __forceinline__ bool sample_li_point(const DevPointLight& l, V3 p_ref, LightSample& out) {
  const V3 to_light = V3{l.position[0], l.position[1], l.position[2]} - p_ref;
  const float d2 = length_sq(to_light);
  if (d2 <= 0.0f) return false;
  const float dist = sqrtf(d2);
  out.wi = to_light / dist;
  out.radiance = V3{l.color[0], l.color[1], l.color[2]} * (l.intensity / (4.0f * kPiF * d2));
  out.pdf = 1.0f;
  out.distance = dist;
  return true;
}

// spot::sample_li (light/spot.rs:51-76) with smoothstep (math/mod.rs:180-183)
__device__ __forceinline__ bool sample_li_spot(const DevSpotLight& l, V3 p_ref, LightSample& out) {
  const V3 to_light = V3{l.position[0], l.position[1], l.position[2]} - p_ref;
  const float d2 = length_sq(to_light);
  if (d2 <= 0.0f) return false;
  const float dist = sqrtf(d2);
  const V3 wi = to_light / dist;
  const float cos_theta = dot(-wi, V3{l.direction[0], l.direction[1], l.direction[2]});
  const float t = clampf((cos_theta - l.cos_total_width) / (l.cos_falloff_start - l.cos_total_width), 0.0f, 1.0f);
  const float falloff = t * t * (3.0f - 2.0f * t);
  if (falloff <= 0.0f) return false;
  out.wi = wi;
  out.radiance = V3{l.color[0], l.color[1], l.color[2]} * (l.intensity * falloff / (2.0f * kTauF * d2));
  out.pdf = 1.0f;
  out.distance = dist;
  return true;
}

// LightSampler::sample_category (light/mod.rs:197-212): the entry whose CDF
// interval holds u.
__device__ __forceinline__ uint32_t sample_category(const DevRenderData& d, float u, float& pmf) {
  u = clampf(u, 0.0f, 1.0f);
  uint32_t n = 0;  // entries of cdf[0..num_cat] that are <= u
  for (uint32_t k = 0; k <= d.num_cat; ++k)
    if (__ldg(d.cat_cdf + k) <= u) n = k + 1;
  const uint32_t idx = min(n == 0 ? 0u : n - 1, d.num_cat - 1);
  pmf = __ldg(d.cat_pmf + idx);
  return __ldg(d.cat_kind + idx);
}

// direct_light_mis_contribution (integrator/mis.rs:145-210) up to the
// visibility test: returns false when the contribution is zero whatever the
// visibility; otherwise `contrib` (radiance * f * cos [* mis] / pdf) counts iff
// the shadow ray (so, wi) first hits triangle (inst, tri) for an area light,
// hits nothing or nothing nearer than dist * (1 - 1e-3) for a point or spot
// light (inst = 0xFFFFFFFF, finite dist), or hits nothing for a directional
// light (inst = 0xFFFFFFFF, dist = inf) -- unoccluded_ray, integrator/mod.rs:
// 239-265.  The light tree is only queried by the diffuse material (the only
// material in scope with a light-tree query); directional lights serve every
// scattering material.
// Li of a delta light, kept out of line so the area-light path of the shade
// kernels does not carry its registers: kind 0 point light, 1 spot light,
// 2 directional light (index into the scene's arrays of that kind).
static __device__ __noinline__ bool sample_li_delta(const DevRenderData& d, uint32_t kind, uint32_t index, V3 p_ref,
                                                    LightSample& li) {
  if (kind == 0) return sample_li_point(d.points[index], p_ref, li);
  if (kind == 1) return sample_li_spot(d.spots[index], p_ref, li);
  // directional::sample_li (light/directional.rs:33-42)
  const DevDirLight& dl = d.dirs[index];
  li.radiance = V3{dl.color[0] * dl.intensity, dl.color[1] * dl.intensity, dl.color[2] * dl.intensity};
  li.wi = -V3{dl.direction[0], dl.direction[1], dl.direction[2]};
  li.pdf = 1.0f;
  li.distance = __int_as_float(0x7f800000);
  return true;
}

// Material::eval_pdf (material/mod.rs:351-370) in radiance mode: f with the
// shading-normal correction, and the BSDF's pdf when f is not zero.
static __device__ __noinline__ V3 material_eval_pdf(const DevRender& S, const DevMaterialRec& m, const Vertex& v,
                                                    V3 wi, float& pdf_out) {
  pdf_out = 0.0f;
  if (m.kind == kDevLambert) {
    const V3 f = lambert_eval(m, v, wi);
    if (length_sq(f) != 0.0f) pdf_out = lambert_pdf(v, wi);
    return f;
  }
  if (m.kind == kDevOpenPbr) {
    if (dot(v.wo, v.ng) <= 0.0f) return V3{0.0f, 0.0f, 0.0f};
    const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
    const V3 wi_l = normalize_or_zero(to_local(v.frame, wi));
    if (wo_l.z <= 0.0f) return V3{0.0f, 0.0f, 0.0f};
    opbr::OpbrVertex s;
    opbr::init_vertex(s, S.d.openpbr + m.openpbr, S.d.cec_e, S.d.dec_e, wo_l, v.front, fabsf(wo_l.z));
    s.thr = v.thr;
    s.lock = v.lock;
    V3 f;
    float pdf;
    opbr::eval_pdf(s, s, wi_l, f, pdf);
    f = modified_eval(v, wi, f, false);
    if (length_sq(f) != 0.0f) pdf_out = pdf;
    return f;
  }
  return V3{0.0f, 0.0f, 0.0f};
}

// environment::sample_li_mis_compensated (light/environment.rs:258-273), or
// with `plain` environment::sample_li (:241-256, the NEE integrator's)
static __device__ __noinline__ bool sample_li_env(const DevRenderData& d, float us0, float us1, bool plain,
                                                  LightSample& li) {
  float pdf;
  if (!env_sample(d.env, plain ? d.env.dist : d.env.mis, us0, us1, li.wi, li.radiance, pdf)) return false;
  if (pdf <= 0.0f) return false;
  li.pdf = pdf;
  li.distance = __int_as_float(0x7f800000);
  li.inst = li.tri = 0xFFFFFFFFu;
  return true;
}

// emitted_radiance_from_bsdf_sample_infinite (integrator/mis.rs:238-258) for a
// ray that left the scene after a BSDF sample of pdf `bsdf_pdf` (camera rays:
// `camera` = true, the map's radiance as is -- mis.rs:33-35).
static __device__ __noinline__ V3 env_escape(const DevRenderData& d, V3 dir, bool camera, bool delta, float bsdf_pdf) {
  const V3 le = env_radiance(d.env, dir);
  if (camera || (le.x == 0.0f && le.y == 0.0f && le.z == 0.0f) || delta) return le;
  // pdf_for_environment_hit (light/mod.rs:439-450), MIS-compensated
  const float cat = d.env.cat_pmf;
  const float light_pdf = cat <= 0.0f ? 0.0f : cat * env_pdf(d.env, d.env.mis, dir);
  return le * balance_heuristic(bsdf_pdf, light_pdf);
}

struct DirectPrep {
  V3 contrib, so, wi;
  uint32_t inst, tri;
  float dist;
};

//
// LIGHTS = false is the specialisation for scenes whose lights are all
// emissive triangles: the light sampler then has the Tree category alone (pmf
// tree_cat_pmf = 1, or no category without a tree) and every tree leaf is a
// triangle, so the category draw and the delta-light paths are compiled out.
// MODE kDirectMis: direct_light_mis_contribution, or with `nee` the NEE
// integrator's direct_light_nee_contribution (integrator/nee.rs:104-150):
// sample_light with the plain environment distribution, Material::eval and no
// MIS weight; kDirectBdptNonArea: BDPT's direct_non_area_light_contribution
// (integrator/bdpt.rs:396-464), zero when the sampled light is an area light.
enum DirectMode : int { kDirectMis = 0, kDirectBdptNonArea = 1 };
template <bool LIGHTS, int MODE = kDirectMis>
__device__ __forceinline__ bool prepare_direct(const DevRender& S, const DevMaterialRec& m, const Vertex& v,
                                               float u_cat, float u_tree, float us0, float us1, DirectPrep& out,
                                               bool nee = false) {
  float cat_pmf;
  uint32_t cat;
  if (LIGHTS) {
    if (S.d.num_cat == 0) return false;  // LightSampler::sample_category: no category
    cat = sample_category(S.d, u_cat, cat_pmf);
  } else {
    if (!S.d.has_tree) return false;
    cat = kCatTree;
    cat_pmf = S.d.tree_cat_pmf;
  }
  LightSample li;
  bool delta = true;
  float sel;
  out.inst = 0xFFFFFFFFu;
  out.tri = 0xFFFFFFFFu;
  if (cat == kCatTree) {
    if (m.kind != kDevLambert) return false;  // build_query: only the diffuse material builds one
    TreeQuery q;
    q.rho = luminance(V3{m.rho[0], m.rho[1], m.rho[2]});
    if (q.rho <= 0.0f) return false;
    q.p = v.p;
    q.n = v.ns;
    float leaf_pmf;
    const uint32_t leaf = sample_light_tree(S.d.ltree, S.d.ltree_root, q, u_tree, leaf_pmf);
    if (leaf == 0xFFFFFFFFu) return false;
    const uint32_t li_inst = __ldg(&S.d.ltree[leaf].leaf_instance), li_tri = __ldg(&S.d.ltree[leaf].leaf_triangle);
    if (LIGHTS && (li_inst == kLeafPointDev || li_inst == kLeafSpotDev)) {
      if (!sample_li_delta(S.d, li_inst == kLeafPointDev ? 0u : 1u, li_tri, v.p, li)) return false;
    } else {
      if (MODE == kDirectBdptNonArea) return false;
      if (!sample_li_triangle(S, li_inst, li_tri, v.p, us0, us1, li)) return false;
      delta = false;
      out.inst = li.inst;
      out.tri = li.tri;
    }
    sel = cat_pmf * leaf_pmf;
  } else if (cat == kCatEnv) {
    if (!sample_li_env(S.d, us0, us1, nee, li)) return false;
    delta = false;
    sel = cat_pmf;
  } else {
    if (!sample_li_delta(S.d, 2u, cat - 1, v.p, li)) return false;
    sel = cat_pmf;
  }
  if (li.pdf <= 0.0f || sel <= 0.0f) return false;
  V3 f;
  float bsdf_pdf = 0.0f;
  if (delta || nee) {
    f = m.kind == kDevLambert ? lambert_eval(m, v, li.wi) : material_eval(S, m, v, li.wi, false);
  } else if (m.kind == kDevLambert) {
    f = lambert_eval(m, v, li.wi);
    if (length_sq(f) == 0.0f) return false;
    bsdf_pdf = lambert_pdf(v, li.wi);
  } else {  // the environment at an OpenPBR vertex
    f = material_eval_pdf(S, m, v, li.wi, bsdf_pdf);
  }
  if (length_sq(f) == 0.0f) return false;
  const float cos_surface = fabsf(dot(v.ng, li.wi));
  if (cos_surface <= 0.0f) return false;
  const float pdf_total = sel * li.pdf;
  if (pdf_total <= 0.0f) return false;
  out.contrib = delta || nee
                    ? li.radiance * f * (cos_surface / pdf_total)
                    : li.radiance * f * (cos_surface * balance_heuristic(pdf_total, bsdf_pdf) / pdf_total);
  out.so = offset_origin(v.p, v.ng, li.wi);  // spawn_ray of unoccluded_ray (integrator/mod.rs:239-265)
  out.wi = li.wi;
  out.dist = li.distance;
  return true;
}

// unoccluded_ray's decision from the shadow ray's closest hit (tri < 0: none)
__device__ __forceinline__ bool shadow_visible(int32_t tri, int32_t inst, float t, uint32_t tgt_inst, uint32_t tgt_tri,
                                               float dist) {
  if (tri < 0) return true;
  if (tgt_inst != 0xFFFFFFFFu) return (uint32_t)inst == tgt_inst && (uint32_t)tri == tgt_tri;
  if (isinf(dist)) return false;
  return t >= dist * (1.0f - kShadowTolerance);
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
