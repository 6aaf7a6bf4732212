// OpenPBR tables of a context (DirectionalAlbedoCache, directional_albedo.rs:
// 38-118: built on first use, shared by every scene of the context) and the C
// entry points that export them and query the device BSDF.
#include <cmath>
#include <cstring>

#include "../host/openpbr_lower.h"
#include "internal.h"

namespace tpt {

namespace {
// Uploads the host sample tables, runs `build` on the context stream, and frees
// the temporaries after the copy back.
struct DevTables {
  float* p = nullptr;
  ~DevTables() {
    if (p) cudaFree(p);
  }
};
tpt_status upload_samples(tpt_context* ctx, const std::vector<float>& a, DevTables* out) {
  tpt_status st = cuda_check(ctx, cudaMalloc(&out->p, std::max<size_t>(4, a.size() * 4)), "cudaMalloc(lut samples)");
  if (st) return st;
  return cuda_check(ctx, cudaMemcpy(out->p, a.data(), a.size() * 4, cudaMemcpyHostToDevice), "cudaMemcpy(lut samples)");
}
}  // namespace

tpt_status ensure_ec_tables(tpt_context* ctx) {
  if (ctx->d_cec_e && ctx->d_dec_e) return TPT_OK;
  LutSampleTables t;
  lut_sample_tables(&t);
  DevTables cu, ccs, uc, ux, dcs;
  tpt_status st;
  if ((st = upload_samples(ctx, t.cec_u, &cu)) || (st = upload_samples(ctx, t.cec_cs, &ccs)) ||
      (st = upload_samples(ctx, t.dec_uc, &uc)) || (st = upload_samples(ctx, t.dec_ux, &ux)) ||
      (st = upload_samples(ctx, t.dec_cs, &dcs)))
    return st;
  float *cec = nullptr, *dec = nullptr;
  if ((st = cuda_check(ctx, cudaMalloc(&cec, kCecLen * 4), "cudaMalloc(conductor table)"))) return st;
  // the dielectric table with its E_avg behind it (the device's dispersive
  // BTDF looks up E_avg at arbitrary etas)
  if ((st = cuda_check(ctx, cudaMalloc(&dec, (kDecLen + kDecAvgLen) * 4), "cudaMalloc(dielectric table)"))) {
    cudaFree(cec);
    return st;
  }
  cudaError_t e = launch_lut_conductor_e(cu.p, ccs.p, cec, ctx->stream);
  if (e == cudaSuccess) e = launch_lut_dielectric_e(uc.p, ux.p, dcs.p, dec, ctx->stream);
  std::vector<float> he(kCecLen), hd(kDecLen);
  if (e == cudaSuccess) e = cudaMemcpyAsync(he.data(), cec, kCecLen * 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hd.data(), dec, kDecLen * 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cudaFree(cec);
    cudaFree(dec);
    return cuda_check(ctx, e, "energy-compensation table build");
  }
  ctx->h_cec_e = std::move(he);
  ctx->h_dec_e = std::move(hd);
  ctx->h_cec_e_avg.assign(kCecAvgLen, 0.0f);
  ctx->h_dec_e_avg.assign(kDecAvgLen, 0.0f);
  conductor_e_avg(ctx->h_cec_e.data(), ctx->h_cec_e_avg.data());
  dielectric_e_avg(ctx->h_dec_e.data(), ctx->h_dec_e_avg.data());
  e = cudaMemcpy(dec + kDecLen, ctx->h_dec_e_avg.data(), kDecAvgLen * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(cec);
    cudaFree(dec);
    return cuda_check(ctx, e, "dielectric E_avg upload");
  }
  ctx->d_cec_e = cec;
  ctx->d_dec_e = dec;
  return TPT_OK;
}

tpt_status ensure_da_table(tpt_context* ctx, float eta, const float** out) {
  uint32_t key;
  std::memcpy(&key, &eta, 4);
  auto it = ctx->da_tables.find(key);
  if (it != ctx->da_tables.end()) {
    *out = it->second;
    return TPT_OK;
  }
  LutSampleTables t;
  lut_sample_tables(&t);
  DevTables dirs, cs;
  tpt_status st;
  if ((st = upload_samples(ctx, t.da_dirs, &dirs)) || (st = upload_samples(ctx, t.da_phi_cs, &cs))) return st;
  float* tab = nullptr;
  if ((st = cuda_check(ctx, cudaMalloc(&tab, (size_t)kDaLen * 4), "cudaMalloc(albedo table)"))) return st;
  cudaError_t e = launch_lut_dielectric_albedo(eta, dirs.p, cs.p, tab, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cudaFree(tab);
    return cuda_check(ctx, e, "directional-albedo table build");
  }
  ctx->da_tables[key] = tab;
  *out = tab;
  return TPT_OK;
}

}  // namespace tpt

using namespace tpt;

extern "C" {

tpt_status tpt_lut_dielectric_albedo(tpt_context* ctx, float eta, float* out) {
  if (!ctx || !out) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL argument");
  tpt_status st = cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (st) return st;
  const float* tab = nullptr;
  float key = (std::isfinite(eta) && eta > 0.0f) ? eta : 1.5f;  // sanitize_dielectric_eta
  if ((st = ensure_da_table(ctx, key, &tab))) return st;
  return cuda_check(ctx, cudaMemcpy(out, tab, (size_t)kDaLen * 4, cudaMemcpyDeviceToHost), "cudaMemcpy(table)");
}

tpt_status tpt_lut_conductor_ec(tpt_context* ctx, float* e, float* e_avg) {
  if (!ctx || !e || !e_avg) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL argument");
  tpt_status st = cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (st || (st = ensure_ec_tables(ctx))) return st;
  std::memcpy(e, ctx->h_cec_e.data(), kCecLen * 4);
  std::memcpy(e_avg, ctx->h_cec_e_avg.data(), kCecAvgLen * 4);
  return TPT_OK;
}

tpt_status tpt_lut_dielectric_ec(tpt_context* ctx, float* e, float* e_avg) {
  if (!ctx || !e || !e_avg) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL argument");
  tpt_status st = cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (st || (st = ensure_ec_tables(ctx))) return st;
  std::memcpy(e, ctx->h_dec_e.data(), kDecLen * 4);
  std::memcpy(e_avg, ctx->h_dec_e_avg.data(), kDecAvgLen * 4);
  return TPT_OK;
}

static tpt_status check_query(tpt_context* ctx, const tpt_scene* scene, uint32_t material) {
  if (!ctx || !scene) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL argument");
  if (material >= scene->render.num_materials) return set_error(ctx, TPT_ERR_INVALID_ARG, "material out of range");
  if (scene->material_kinds[material] != TPT_MATERIAL_OPENPBR)
    return set_error(ctx, TPT_ERR_INVALID_ARG, "material is not OpenPBR");
  return cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
}

tpt_status tpt_bsdf_eval_device(tpt_context* ctx, const tpt_scene* scene, uint32_t material, uint64_t n,
                                const float* wo, const float* wi, const uint32_t* front_face, uint32_t mode, float* f,
                                float* pdf, void* stream) {
  tpt_status st = check_query(ctx, scene, material);
  if (st) return st;
  if (n && (!wo || !wi || !front_face || !f || !pdf)) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL buffer");
  if (mode > 1) return set_error(ctx, TPT_ERR_INVALID_ARG, "mode must be 0 (radiance) or 1 (importance)");
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return cuda_check(ctx, launch_bsdf_eval(scene->render, material, n, wo, wi, front_face, mode, nullptr, f, pdf, s),
                    "bsdf eval launch");
}

tpt_status tpt_bsdf_sample_device(tpt_context* ctx, const tpt_scene* scene, uint32_t material, uint64_t n,
                                  const float* wo, const float* u, const uint32_t* front_face, uint32_t mode,
                                  float* out, void* stream) {
  tpt_status st = check_query(ctx, scene, material);
  if (st) return st;
  if (n && (!wo || !u || !front_face || !out)) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL buffer");
  if (mode > 1) return set_error(ctx, TPT_ERR_INVALID_ARG, "mode must be 0 (radiance) or 1 (importance)");
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return cuda_check(ctx, launch_bsdf_sample(scene->render, material, n, wo, u, front_face, mode, nullptr, out, s),
                    "bsdf sample launch");
}

tpt_status tpt_bsdf_eval_path_device(tpt_context* ctx, const tpt_scene* scene, uint32_t material, uint64_t n,
                                     const float* wo, const float* wi, const uint32_t* front_face, const float* state,
                                     uint32_t mode, float* f, float* pdf, void* stream) {
  tpt_status st = check_query(ctx, scene, material);
  if (st) return st;
  if (n && (!wo || !wi || !front_face || !state || !f || !pdf))
    return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL buffer");
  if (mode > 1) return set_error(ctx, TPT_ERR_INVALID_ARG, "mode must be 0 (radiance) or 1 (importance)");
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return cuda_check(ctx, launch_bsdf_eval(scene->render, material, n, wo, wi, front_face, mode, state, f, pdf, s),
                    "bsdf eval launch");
}

tpt_status tpt_bsdf_sample_path_device(tpt_context* ctx, const tpt_scene* scene, uint32_t material, uint64_t n,
                                       const float* wo, const float* u, const uint32_t* front_face, const float* state,
                                       uint32_t mode, float* out, void* stream) {
  tpt_status st = check_query(ctx, scene, material);
  if (st) return st;
  if (n && (!wo || !u || !front_face || !state || !out)) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL buffer");
  if (mode > 1) return set_error(ctx, TPT_ERR_INVALID_ARG, "mode must be 0 (radiance) or 1 (importance)");
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return cuda_check(ctx, launch_bsdf_sample(scene->render, material, n, wo, u, front_face, mode, state, out, s),
                    "bsdf sample launch");
}

}  // extern "C"
