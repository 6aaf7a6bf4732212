// Oracle: OpenPBR BSDF (evaluation, pdf, sampling), its lobes and the
// directional-albedo / energy-compensation lookup tables it reads.  Restates
// crates/renderer/src/{bsdf/open_pbr.rs, bsdf/eon.rs, bsdf/smith_ggx.rs,
// bsdf/dielectric_ggx.rs (the reflection/transmission GGX used to build the
// tables), bsdf/directional_albedo.rs, material/open_pbr.rs}.
//
// Covered: base (EON diffuse), metal (F82-tint + multiple scattering), specular
// reflection (GGX + multiple scattering), specular transmission (GGX BTDF +
// multiple scattering, rough and smooth), thin-walled surfaces (the two-interface
// slab of thin_wall_coefficients, the thin-wall BTDF and the diffuse BTDF),
// coat, fuzz (LTC), with optional anisotropy and smooth (delta) lobes.  Not
// covered: opacity and textures; the material lowering rejects parameters
// that would need them.  Thin film (bsdf/thin_film.rs) modulates the specular,
// metal and transmission Fresnel terms; dispersion (bsdf/dispersion.rs) makes
// the transmission IOR a Cauchy function of wavelength: camera-integrated
// evaluation while the path is unlocked, a wavelength lock once a dispersive
// refraction is sampled.
#pragma once
#include "common.h"

namespace orc {

// Mirrors `struct tpt_openpbr_desc` of the C ABI field for field
// (OpenPbrMaterial's untextured parameters, material/open_pbr.rs:23-78).
struct OpenPbrDesc {
  float base_weight;
  float base_color[3];
  float base_diffuse_roughness;
  float base_metalness;
  float specular_weight;
  float specular_color[3];
  float specular_roughness;
  float specular_ior;
  float specular_roughness_anisotropy;
  float transmission_weight;
  float transmission_color[3];
  float subsurface_weight;
  float subsurface_color[3];
  float fuzz_weight;
  float fuzz_color[3];
  float fuzz_roughness;
  float coat_weight;
  float coat_color[3];
  float coat_roughness;
  float coat_roughness_anisotropy;
  float coat_ior;
  float coat_darkening;
  float thin_film_weight;
  float thin_film_thickness;
  float thin_film_ior;
  float emission_luminance;
  float emission_color[3];
  float geometry_opacity;
  uint32_t geometry_thin_walled;
  float transmission_dispersion_scale;
  float transmission_dispersion_abbe_number;
};
static_assert(sizeof(OpenPbrDesc) == 45 * 4, "OpenPbrDesc layout");

// ---- lookup tables (bsdf/directional_albedo.rs) ------------------------------
constexpr int kDaCos = 64, kDaPhi = 16, kDaRough = 64, kDaAniso = 16;
constexpr int kDaLen = kDaCos * kDaPhi * kDaRough * kDaAniso;
constexpr int kCecCos = 64, kCecRough = 64;
constexpr int kDecCos = 32, kDecRough = 32, kDecEta = 32;

struct DielectricAlbedoLut {  // DielectricGgxDirectionalAlbedoLut
  float eta = 1.5f;
  std::vector<float> values;
  void build(float eta, int nthreads);
  float lookup(Vec3 w, float roughness, float anisotropy) const;
};
struct ConductorEcLut {  // ConductorGgxEnergyCompensationLut
  std::vector<float> e, e_avg;
  void build(int nthreads);
  float lookup_e(float cos_theta, float roughness) const;
  float lookup_e_avg(float roughness) const;
};
struct DielectricEcLut {  // DielectricGgxEnergyCompensationLut
  std::vector<float> e, e_avg;
  void build(int nthreads);
  float lookup_e(float cos_theta, float roughness, float eta) const;
  float lookup_e_avg(float roughness, float eta) const;
};
float sanitize_dielectric_eta(float eta);

// ---- shared lobe math ------------------------------------------------------
constexpr float kMinAlpha = 1.0e-4f;
constexpr float kSmoothAlpha = 1.0e-3f;
float powi(float x, int n);  // llvm.powi expansion (binary exponentiation)
float fresnel_dielectric(float cos_i, float eta_i, float eta_t);
float ggx_d(Vec3 wm, float ax, float ay);
float ggx_lambda(Vec3 w, float ax, float ay);
float ggx_g1(Vec3 w, float ax, float ay);
float ggx_g2(Vec3 wo, Vec3 wi, float ax, float ay);
Vec3 reflect_local(Vec3 wo, Vec3 wm);
bool reflection_half_vector(Vec3 wo, Vec3 wi, Vec3* wm);
float pdf_wm_vndf(Vec3 wo, Vec3 wm, float ax, float ay);
bool sample_wm_vndf(Vec3 wo, float ax, float ay, Vec2 us, Vec3* wm);
bool sample_wm_bounded_vndf(Vec3 wo, float ax, float ay, Vec2 us, Vec3* wm);
float pdf_wm_bounded_vndf(Vec3 wo, Vec3 wm, float ax, float ay);
Vec3 sample_cosine_hemisphere(Vec2 us);

enum BsdfFlag : uint32_t { kReflection = 1, kTransmission = 2, kDiffuse = 4, kGlossy = 8, kDelta = 16 };
enum TransportMode : int { kRadiance = 0, kImportance = 1 };

struct BsdfSample {
  Vec3 weight, wi;
  float pdf = 0, pdf_rev = 0, eta = 1;
  uint32_t flags = 0;
  bool has_lock = false;  // BsdfSample::wavelength_lock is Some(wavelength_lock)
  float wavelength_lock = 0;
};

// OpenPbrBsdfParams (bsdf/open_pbr.rs:33-70) restricted to the covered lobes.
struct OpenPbrParams {
  Vec3 base_color;
  float base;
  float specular;
  Vec3 specular_color;
  float specular_alpha_x, specular_alpha_y, specular_eta, transmission_eta;
  float metalness;
  float coat;
  Vec3 coat_color, coat_darkening;
  float coat_alpha_x, coat_alpha_y, coat_eta;
  float fuzz;
  Vec3 fuzz_color;
  float fuzz_roughness;
  float transmission;
  Vec3 transmission_color;
  float transmission_alpha_x, transmission_alpha_y;
  float diffuse_roughness;
  float subsurface;
  Vec3 subsurface_color;
  bool thin_walled;
  float thin_film_weight, thin_film_thickness, thin_film_ior;  // thickness in nm
  Vec3 metal_n, metal_k;                                       // artist_friendly_complex_ior
  bool front_face;
  // dispersion (bsdf/open_pbr.rs:58, 69-70): the Abbe number (0 = off), the
  // path throughput arriving at the vertex, and the path's wavelength lock
  float transmission_dispersion_abbe = 0;
  Vec3 path_throughput = Vec3(1, 1, 1);
  bool has_lock = false;
  float wavelength_lock = 0;
};

// bsdf/thin_film.rs:11-45 and bsdf/conductor_complex.rs:132-147
Vec3 thin_film_dielectric(float cos_i, float eta_outside, float eta_film, float eta_base, float thickness_nm);
Vec3 thin_film_conductor(float cos_i, float eta_outside, float eta_film, Vec3 n, Vec3 k, float thickness_nm);
void artist_friendly_complex_ior(Vec3 face, Vec3 edge, Vec3* n, Vec3* k);

struct OpenPbrLuts {
  const DielectricAlbedoLut* spec;
  const DielectricAlbedoLut* coat;
  const ConductorEcLut* conductor;
  const DielectricEcLut* dielectric;
};

struct OpenPbrBsdf {
  OpenPbrParams p;
  OpenPbrLuts L;
  Vec3 eval(Vec3 wo, Vec3 wi, TransportMode mode) const;
  float pdf(Vec3 wo, Vec3 wi) const;
  // u_extra: MaterialSampleRandoms::u_extra0..3 (the dispersion randoms); NULL = zeros
  bool sample(Vec3 wo, float u_lobe, Vec2 u_dir, TransportMode mode, BsdfSample* out,
              const float* u_extra = nullptr) const;
};

// EonBsdf (bsdf/eon.rs) with an arbitrary albedo.
Vec3 eon_eval(Vec3 rho, float roughness, Vec3 wo, Vec3 wi);
float eon_pdf(float roughness, Vec3 wo, Vec3 wi);
bool eon_sample(Vec3 rho, float roughness, Vec3 wo, Vec2 us, BsdfSample* s);

// zeltner_dir_albedo (material/open_pbr.rs:888-897): the fuzz lobe's albedo
float openpbr_fuzz_albedo(float ndot_v, float roughness);

// OpenPbrMaterial::make_bsdf (material/open_pbr.rs:393-487) for an untextured
// material seen from `wo_local` on the front (or back) face.
OpenPbrParams make_openpbr_params(const OpenPbrDesc& m, bool front_face, Vec3 wo_local);
// The dielectric eta whose albedo table the specular lobe reads
// (OpenPbrMaterial::requires_specular_eta, material/open_pbr.rs:293-298).
float openpbr_specular_eta(const OpenPbrDesc& m);

}  // namespace orc
