// Oracle C entry points for the OpenPBR BSDF and its tables (test
// infrastructure only).
#include <cstring>
#include <thread>

#include "dispersion.h"
#include "render.h"

using namespace orc;

namespace {
int threads_or_default(int n) {
  if (n > 0) return n;
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

// OpenPbrBsdfParams in a flat float array (field order of OpenPbrParams;
// the last entry is front_face as 0/1).
OpenPbrParams params_from_flat(const float* f) {
  OpenPbrParams p;
  int i = 0;
  auto v3 = [&]() { Vec3 v(f[i], f[i + 1], f[i + 2]); i += 3; return v; };
  p.base_color = v3();
  p.base = f[i++];
  p.specular = f[i++];
  p.specular_color = v3();
  p.specular_alpha_x = f[i++];
  p.specular_alpha_y = f[i++];
  p.specular_eta = f[i++];
  p.transmission_eta = f[i++];
  p.metalness = f[i++];
  p.coat = f[i++];
  p.coat_color = v3();
  p.coat_darkening = v3();
  p.coat_alpha_x = f[i++];
  p.coat_alpha_y = f[i++];
  p.coat_eta = f[i++];
  p.fuzz = f[i++];
  p.fuzz_color = v3();
  p.fuzz_roughness = f[i++];
  p.transmission = f[i++];
  p.transmission_color = v3();
  p.transmission_alpha_x = f[i++];
  p.transmission_alpha_y = f[i++];
  p.diffuse_roughness = f[i++];
  p.subsurface = f[i++];
  p.subsurface_color = v3();
  p.thin_walled = f[i++] != 0.0f;
  p.thin_film_weight = f[i++];
  p.thin_film_thickness = f[i++];
  p.thin_film_ior = f[i++];
  p.metal_n = v3();
  p.metal_k = v3();
  p.front_face = f[i++] != 0.0f;
  p.transmission_dispersion_abbe = f[i++];
  p.path_throughput = v3();
  p.has_lock = f[i++] != 0.0f;
  p.wavelength_lock = f[i++];
  return p;
}

// path state (throughput r, g, b, wavelength lock; NaN = no lock) onto params
void apply_state(OpenPbrBsdf& b, const float* state) {
  if (!state) return;
  b.p.path_throughput = Vec3(state[0], state[1], state[2]);
  b.p.has_lock = !std::isnan(state[3]);
  b.p.wavelength_lock = b.p.has_lock ? state[3] : 0.0f;
}

// The constant tables of the reference's OpenPBR unit tests
// (bsdf/open_pbr.rs:2246-2263): albedo 0.04, e = e_avg = 0.9.
struct ConstLuts {
  DielectricAlbedoLut spec, coat;
  ConductorEcLut cec;
  DielectricEcLut dec;
  ConstLuts() {
    spec.eta = coat.eta = 1.5f;
    spec.values.assign(kDaLen, 0.04f);
    coat.values.assign(kDaLen, 0.04f);
    cec.e.assign(kCecCos * kCecRough, 0.9f);
    cec.e_avg.assign(kCecRough, 0.9f);
    dec.e.assign(kDecCos * kDecRough * kDecEta, 0.9f);
    dec.e_avg.assign(kDecRough * kDecEta, 0.9f);
  }
};

OpenPbrBsdf bsdf_from(const float* params, int lut_mode, float spec_eta, float coat_eta) {
  OpenPbrBsdf b;
  b.p = params_from_flat(params);
  if (lut_mode == 1) {
    static ConstLuts c;
    b.L = OpenPbrLuts{&c.spec, &c.coat, &c.cec, &c.dec};
  } else {
    OpenPbrDesc d{};
    d.specular_ior = spec_eta;
    d.specular_weight = 1.0f;
    d.coat_ior = coat_eta;
    b.L = openpbr_luts_for(d, threads_or_default(0));
  }
  return b;
}

OpenPbrBsdf bsdf_from_desc(const OpenPbrDesc* m, int front, const float* wo) {
  OpenPbrBsdf b;
  b.p = make_openpbr_params(*m, front != 0, Vec3(wo[0], wo[1], wo[2]));
  b.L = openpbr_luts_for(*m, threads_or_default(0));
  return b;
}

void put3(float* o, Vec3 v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

// out: weight (3), wi (3), pdf, pdf_rev, flags (bits), then with u_extra the
// sampled wavelength lock (NaN = none) as a tenth value
int do_sample(const OpenPbrBsdf& b, const float* wo, float u_lobe, float u0, float u1, int mode, float* out,
              const float* u_extra = nullptr) {
  BsdfSample s;
  if (!b.sample(Vec3(wo[0], wo[1], wo[2]), u_lobe, Vec2(u0, u1), (TransportMode)mode, &s, u_extra)) return 0;
  put3(out, s.weight);
  put3(out + 3, s.wi);
  out[6] = s.pdf;
  out[7] = s.pdf_rev;
  uint32_t fl = s.flags;
  std::memcpy(out + 8, &fl, 4);
  if (u_extra) out[9] = s.has_lock ? s.wavelength_lock : std::nanf("");
  return 1;
}
}  // namespace

extern "C" {

// Tables (built on first use, shared by every scene of the process).
void orc_lut_dielectric_albedo(float eta, float* out) {
  OpenPbrDesc d{};
  d.specular_ior = eta;
  d.specular_weight = 1.0f;
  d.coat_ior = eta;
  OpenPbrLuts L = openpbr_luts_for(d, threads_or_default(0));
  std::memcpy(out, L.spec->values.data(), sizeof(float) * kDaLen);
}
void orc_lut_conductor_ec(float* e, float* e_avg) {
  OpenPbrDesc d{};
  d.specular_ior = 1.5f;
  d.specular_weight = 1.0f;
  d.coat_ior = 1.5f;
  OpenPbrLuts L = openpbr_luts_for(d, threads_or_default(0));
  std::memcpy(e, L.conductor->e.data(), sizeof(float) * L.conductor->e.size());
  std::memcpy(e_avg, L.conductor->e_avg.data(), sizeof(float) * L.conductor->e_avg.size());
}
void orc_lut_dielectric_ec(float* e, float* e_avg) {
  OpenPbrDesc d{};
  d.specular_ior = 1.5f;
  d.specular_weight = 1.0f;
  d.coat_ior = 1.5f;
  OpenPbrLuts L = openpbr_luts_for(d, threads_or_default(0));
  std::memcpy(e, L.dielectric->e.data(), sizeof(float) * L.dielectric->e.size());
  std::memcpy(e_avg, L.dielectric->e_avg.data(), sizeof(float) * L.dielectric->e_avg.size());
}
float orc_lut_conductor_lookup_e(float c, float r) {
  OpenPbrDesc d{};
  d.specular_ior = 1.5f;
  d.specular_weight = 1.0f;
  d.coat_ior = 1.5f;
  return openpbr_luts_for(d, threads_or_default(0)).conductor->lookup_e(c, r);
}

// Bsdf-level queries on explicit OpenPbrBsdfParams (flat floats, see above).
// lut_mode 0: the scene tables for the given etas; 1: the constant test tables.
void orc_openpbr_params_eval(const float* params, int lut_mode, float spec_eta, float coat_eta, const float* wo,
                             const float* wi, int mode, float* out3) {
  OpenPbrBsdf b = bsdf_from(params, lut_mode, spec_eta, coat_eta);
  put3(out3, b.eval(Vec3(wo[0], wo[1], wo[2]), Vec3(wi[0], wi[1], wi[2]), (TransportMode)mode));
}
float orc_openpbr_params_pdf(const float* params, int lut_mode, float spec_eta, float coat_eta, const float* wo,
                             const float* wi) {
  return bsdf_from(params, lut_mode, spec_eta, coat_eta).pdf(Vec3(wo[0], wo[1], wo[2]), Vec3(wi[0], wi[1], wi[2]));
}
int orc_openpbr_params_sample(const float* params, int lut_mode, float spec_eta, float coat_eta, const float* wo,
                              float u_lobe, float u0, float u1, int mode, float* out9) {
  return do_sample(bsdf_from(params, lut_mode, spec_eta, coat_eta), wo, u_lobe, u0, u1, mode, out9);
}

// Batched evaluation over n directions wi (n x 3): f (n x 3) and pdf (n).
void orc_openpbr_params_eval_batch(const float* params, int lut_mode, float spec_eta, float coat_eta,
                                   const float* wo, const float* wi, uint64_t n, int mode, float* f, float* pdf) {
  OpenPbrBsdf b = bsdf_from(params, lut_mode, spec_eta, coat_eta);
  Vec3 o(wo[0], wo[1], wo[2]);
  for (uint64_t k = 0; k < n; ++k) {
    Vec3 i(wi[3 * k], wi[3 * k + 1], wi[3 * k + 2]);
    if (f) put3(f + 3 * k, b.eval(o, i, (TransportMode)mode));
    if (pdf) pdf[k] = b.pdf(o, i);
  }
}
void orc_eon_eval_batch(const float* rho, float r, const float* wo, const float* wi, uint64_t n, float* f,
                        float* pdf) {
  Vec3 o(wo[0], wo[1], wo[2]), rh(rho[0], rho[1], rho[2]);
  for (uint64_t k = 0; k < n; ++k) {
    Vec3 i(wi[3 * k], wi[3 * k + 1], wi[3 * k + 2]);
    if (f) put3(f + 3 * k, eon_eval(rh, r, o, i));
    if (pdf) pdf[k] = eon_pdf(r, o, i);
  }
}
int orc_eon_sample(const float* rho, float r, const float* wo, float u0, float u1, float* out9) {
  BsdfSample s;
  if (!eon_sample(Vec3(rho[0], rho[1], rho[2]), r, Vec3(wo[0], wo[1], wo[2]), Vec2(u0, u1), &s)) return 0;
  put3(out9, s.weight);
  put3(out9 + 3, s.wi);
  out9[6] = s.pdf;
  out9[7] = s.pdf_rev;
  uint32_t fl = s.flags;
  std::memcpy(out9 + 8, &fl, 4);
  return 1;
}

// Material-level queries: make_bsdf of an untextured material for a local wo.
void orc_openpbr_eval(const void* desc, int front, const float* wo, const float* wi, int mode, float* out3) {
  OpenPbrBsdf b = bsdf_from_desc((const OpenPbrDesc*)desc, front, wo);
  put3(out3, b.eval(Vec3(wo[0], wo[1], wo[2]), Vec3(wi[0], wi[1], wi[2]), (TransportMode)mode));
}
float orc_openpbr_pdf(const void* desc, int front, const float* wo, const float* wi) {
  return bsdf_from_desc((const OpenPbrDesc*)desc, front, wo).pdf(Vec3(wo[0], wo[1], wo[2]), Vec3(wi[0], wi[1], wi[2]));
}
int orc_openpbr_sample(const void* desc, int front, const float* wo, float u_lobe, float u0, float u1, int mode,
                       float* out9) {
  return do_sample(bsdf_from_desc((const OpenPbrDesc*)desc, front, wo), wo, u_lobe, u0, u1, mode, out9);
}

// OpenPbrMaterial::le (material/open_pbr.rs:351-375) at a vertex whose shading
// frame is the identity, for a local wo; 0: no emission (le() is None).
int orc_openpbr_le(const void* desc, int front, const float* wo, float* out3) {
  Material m;
  m.kind = kOpenPbr;
  m.openpbr = *(const OpenPbrDesc*)desc;
  Vertex v{};
  v.frame.t = Vec3(1, 0, 0);
  v.frame.b = Vec3(0, 1, 0);
  v.frame.n = Vec3(0, 0, 1);
  v.ng = v.ns = v.frame.n;
  v.wo = Vec3(wo[0], wo[1], wo[2]);
  v.front_face = front != 0;
  Vec3 le;
  if (!material_le(m, v, &le)) return 0;
  put3(out3, le);
  return 1;
}

// The same queries with the path state a shading vertex carries (throughput,
// wavelength lock) and the dispersion randoms u_extra0..3.
void orc_openpbr_eval_ex(const void* desc, int front, const float* wo, const float* wi, const float* state, int mode,
                         float* out3) {
  OpenPbrBsdf b = bsdf_from_desc((const OpenPbrDesc*)desc, front, wo);
  apply_state(b, state);
  put3(out3, b.eval(Vec3(wo[0], wo[1], wo[2]), Vec3(wi[0], wi[1], wi[2]), (TransportMode)mode));
}
float orc_openpbr_pdf_ex(const void* desc, int front, const float* wo, const float* wi, const float* state) {
  OpenPbrBsdf b = bsdf_from_desc((const OpenPbrDesc*)desc, front, wo);
  apply_state(b, state);
  return b.pdf(Vec3(wo[0], wo[1], wo[2]), Vec3(wi[0], wi[1], wi[2]));
}
int orc_openpbr_sample_ex(const void* desc, int front, const float* wo, float u_lobe, float u0, float u1,
                          const float* u_extra, const float* state, int mode, float* out10) {
  OpenPbrBsdf b = bsdf_from_desc((const OpenPbrDesc*)desc, front, wo);
  apply_state(b, state);
  return do_sample(b, wo, u_lobe, u0, u1, mode, out10, u_extra);
}
int orc_openpbr_params_sample_ex(const float* params, int lut_mode, float spec_eta, float coat_eta, const float* wo,
                                 float u_lobe, float u0, float u1, const float* u_extra, int mode, float* out10) {
  return do_sample(bsdf_from(params, lut_mode, spec_eta, coat_eta), wo, u_lobe, u0, u1, mode, out10, u_extra);
}
// bsdf/dispersion.rs entry points (their unit tests restated in tests/)
float orc_cauchy_ior(float lambda_nm, float n_d, float abbe) { return cauchy_ior(lambda_nm, n_d, abbe); }
float orc_sample_dispersion_wavelength(float u, const float* throughput, float* basis3) {
  Vec3 b;
  const float l = sample_dispersion_wavelength_weighted(u, Vec3(throughput[0], throughput[1], throughput[2]), &b);
  put3(basis3, b);
  return l;
}
float orc_sample_camera_channel_wavelength(int channel, float u) { return sample_camera_channel_wavelength(channel, u); }
float orc_camera_wavelength_sampling_pdf(float lambda_nm, const float* throughput) {
  return camera_wavelength_sampling_pdf(lambda_nm, Vec3(throughput[0], throughput[1], throughput[2]));
}
void orc_camera_rgb_basis_at(float lambda_nm, float* out3) { put3(out3, camera_rgb_basis_at(lambda_nm)); }

// Scene material: OpenPBR parameters of material `index` (kind must be 2).
const char* orc_render_scene_set_openpbr(void* h, uint32_t index, const void* desc) {
  auto* s = (RenderScene*)h;
  const OpenPbrDesc& d = *(const OpenPbrDesc*)desc;
  s->materials[index].openpbr = d;
  s->materials[index].luts = openpbr_luts_for(d, threads_or_default(0));
  return "";
}

}  // extern "C"
