// C ABI: material updates and the path-replay adjoint of the MIS renderer.
//
// Neither has a counterpart in the reference, whose renderer is neither
// differentiable nor able to change a material after Scene::add_material.
// tpt_adjoint_device runs, per chunk of paths, the forward wavefront (per-path
// radiance into the context's sample scratch) and then its adjoint replay over
// the same paths (wavefront_kernels.cu, ADJ = true), which adds every rough
// OpenPBR vertex's contribution to per-material FP64 gradients.
#include <cstring>
#include <string>

#include "../host/openpbr_lower.h"
#include "internal.h"

using namespace tpt;

namespace {

constexpr float kDefaultFdStep = 1.0e-3f;

float* group_field(tpt_openpbr_desc& d, uint32_t g, int c) {
  switch (g) {
    case 0: return &d.base_color[c];
    case 1: return &d.specular_roughness;
    case 2: return &d.base_metalness;
    case 3: return &d.specular_ior;
    default: return &d.coat_weight;
  }
}

// Parameter range of each group: [0, 1] for the weights, colours and
// roughness, [1, 10] for the specular IOR.
void group_range(uint32_t g, float* lo, float* hi) {
  *lo = g == 3 ? 1.0f : 0.0f;
  *hi = g == 3 ? 10.0f : 1.0f;
}

// Lowers the theta - h / theta + h copies of every OpenPBR material for the
// groups in `mask` and uploads them with their spans.
tpt_status ensure_adjoint_tables(tpt_context* ctx, tpt_scene* s, uint32_t mask, float step) {
  if (s->d_adj && s->adj_version == s->mat_version && s->adj_mask == mask && s->adj_step == step) return TPT_OK;
  const size_t n = s->opbr_desc.size();
  std::vector<DevOpenPbr> pert(std::max<size_t>(1, n * kGradGroups * 2));
  std::vector<float> span(std::max<size_t>(1, n * kGradGroups * 3), 0.0f);
  for (size_t t = 0; t < n; ++t) {
    for (uint32_t g = 0; g < kGradGroups; ++g) {
      DevOpenPbr* rec = &pert[(t * kGradGroups + g) * 2];
      if (!(mask & (1u << g))) {
        std::memset(rec, 0, 2 * sizeof(DevOpenPbr));
        continue;
      }
      tpt_openpbr_desc lo = s->opbr_desc[t], hi = s->opbr_desc[t];
      float rlo, rhi;
      group_range(g, &rlo, &rhi);
      for (int c = 0; c < (g == 0 ? 3 : 1); ++c) {
        const float x = *group_field(lo, g, c);
        const float a = std::max(x - step, rlo), b = std::min(x + step, rhi);
        *group_field(lo, g, c) = a;
        *group_field(hi, g, c) = b;
        span[(t * kGradGroups + g) * 3 + c] = b - a;
      }
      tpt_status st = lower_openpbr_material(ctx, lo, rec);
      if (!st) st = lower_openpbr_material(ctx, hi, rec + 1);
      if (st) return st;
    }
  }
  const size_t pb = pert.size() * sizeof(DevOpenPbr), sb = span.size() * sizeof(float);
  const size_t bytes = pb + sb;
  if (s->d_adj_bytes < bytes) {
    if (s->d_adj) {
      cudaStreamSynchronize(ctx->stream);
      cudaDeviceSynchronize();
      cudaFree(s->d_adj);
    }
    s->d_adj = nullptr;
    s->d_adj_bytes = 0;
    tpt_status st = cuda_check(ctx, cudaMalloc(&s->d_adj, bytes), "cudaMalloc(adjoint tables)");
    if (st) return st;
    s->d_adj_bytes = bytes;
  } else {
    cudaDeviceSynchronize();  // earlier adjoint launches may still read the old tables
  }
  tpt_status st = cuda_check(ctx, cudaMemcpy(s->d_adj, pert.data(), pb, cudaMemcpyHostToDevice), "upload adjoint tables");
  if (!st)
    st = cuda_check(ctx, cudaMemcpy((char*)s->d_adj + pb, span.data(), sb, cudaMemcpyHostToDevice),
                    "upload adjoint spans");
  if (st) return st;
  s->adj_version = s->mat_version;
  s->adj_mask = mask;
  s->adj_step = step;
  return TPT_OK;
}

}  // namespace

extern "C" {

tpt_status tpt_scene_set_openpbr(tpt_context* ctx, tpt_scene* scene, uint32_t count, const uint32_t* material_ids,
                                 const tpt_openpbr_desc* descs, void* stream) {
  if (!ctx || !scene) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL context or scene");
  if (count && (!material_ids || !descs)) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL material list");
  if (tpt_status st = set_device(ctx)) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  std::vector<DevOpenPbr> recs(count);
  for (uint32_t k = 0; k < count; ++k) {
    const uint32_t m = material_ids[k];
    if (m >= scene->opbr_of_material.size() || scene->opbr_of_material[m] == kInvalidNode)
      return set_error(ctx, TPT_ERR_INVALID_ARG, "material " + std::to_string(m) + " is not an OpenPBR material");
    // the light tree and the material record were built from the uploaded emission
    const tpt_openpbr_desc& old = scene->opbr_desc[scene->opbr_of_material[m]];
    if (descs[k].emission_luminance != old.emission_luminance ||
        std::memcmp(descs[k].emission_color, old.emission_color, sizeof old.emission_color) != 0)
      return set_error(ctx, TPT_ERR_INVALID_ARG,
                       "material " + std::to_string(m) + ": emission differs from the uploaded scene's");
    tpt_status st = lower_openpbr_material(ctx, descs[k], &recs[k]);
    if (st) return st;
  }
  DevOpenPbr* table = const_cast<DevOpenPbr*>(scene->render.openpbr);
  for (uint32_t k = 0; k < count; ++k) {
    const uint32_t t = scene->opbr_of_material[material_ids[k]];
    tpt_status st = cuda_check(
        ctx, cudaMemcpyAsync(table + t, &recs[k], sizeof(DevOpenPbr), cudaMemcpyHostToDevice, s), "material update");
    if (st) return st;
    scene->opbr_desc[t] = descs[k];
  }
  // the records above are pageable host memory: the copies are staged before return
  scene->mat_version++;
  return TPT_OK;
}

tpt_status tpt_adjoint_device(tpt_context* ctx, const tpt_render_job* job, const tpt_adjoint_desc* adesc,
                              const float* d_image, double* grad, void* stream) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  if (!d_image || !grad) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL d_image or gradient buffer");
  RenderLaunch L;
  tpt_status st = render_launch_params(ctx, job, &L);
  if (st) return st;
  if (job->integrator != TPT_INTEGRATOR_MIS)
    return set_error(ctx, TPT_ERR_INVALID_ARG, "the adjoint covers the MIS integrator only");
  uint32_t mask = adesc ? adesc->param_mask : 0u;
  if (mask == 0) mask = TPT_GRAD_ALL;
  if (mask & ~(uint32_t)TPT_GRAD_ALL) return set_error(ctx, TPT_ERR_INVALID_ARG, "unknown gradient group bits");
  const float step = adesc && adesc->fd_step > 0.0f ? adesc->fd_step : kDefaultFdStep;
  if (!(step < 0.5f)) return set_error(ctx, TPT_ERR_INVALID_ARG, "fd_step must be in (0, 0.5)");
  tpt_scene* scene = const_cast<tpt_scene*>(job->scene);
  for (const tpt_openpbr_desc& d : scene->opbr_desc)
    if (d.transmission_dispersion_scale > 0.0f && d.transmission_weight > 0.0f)
      return set_error(ctx, TPT_ERR_INVALID_ARG, "dispersive OpenPBR transmission is not differentiated");
  if (mask & TPT_GRAD_MASK_COAT) {
    // emission leaving through a coat depends on coat_weight, and the replay
    // differentiates the BSDF only
    for (const tpt_openpbr_desc& d : scene->opbr_desc)
      if (d.emission_luminance > 0.0f && d.coat_weight > 0.0f)
        return set_error(ctx, TPT_ERR_INVALID_ARG,
                         "coat gradients of a scene with a coated OpenPBR emitter are not differentiated");
  }
  if ((st = set_device(ctx))) return st;
  note_device_call(ctx, "tpt_adjoint_device");
  if ((st = ensure_adjoint_tables(ctx, scene, mask, step))) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  const size_t gbytes = (size_t)scene->render.num_materials * kGradParams * sizeof(double);
  if ((st = cuda_check(ctx, cudaMemsetAsync(grad, 0, gbytes, s), "clear gradients"))) return st;
  DevAdjoint A;
  A.pert = (const DevOpenPbr*)scene->d_adj;
  A.span = (const float*)((const char*)scene->d_adj +
                          std::max<size_t>(1, scene->opbr_desc.size() * kGradGroups * 2) * sizeof(DevOpenPbr));
  A.d_image = d_image;
  A.grad = grad;
  A.scale = L.cam.exposure / (float)L.spp;
  A.mask = mask;
  A.s_grad = nullptr;
  A.s_gkey = nullptr;
  const uint32_t npix = L.width * L.height;
  uint32_t pix_begin = 0, pix_end = npix;
  if (adesc && adesc->num_pixels) {
    if (adesc->first_pixel > npix || adesc->num_pixels > npix - adesc->first_pixel)
      return set_error(ctx, TPT_ERR_INVALID_ARG, "adjoint pixel range out of bounds");
    pix_begin = adesc->first_pixel;
    pix_end = adesc->first_pixel + adesc->num_pixels;
  }
  A.pixel_base = pix_begin;
  const uint32_t cp = chunk_pixels(L, ctx->batch_capacity);
  // light samples at OpenPBR vertices come from directional lights and the
  // environment only (the light tree serves diffuse vertices): their gradient
  // planes follow the samples in the scratch buffer, sized for the
  // wavefront's capacity
  const bool light_grads = scene->num_directional_lights > 0 || scene->render.has_env;
  if ((st = ensure_wavefront(ctx, cp * L.spp))) return st;
  const size_t sample_bytes = ((size_t)cp * L.spp * 12 + 255) & ~(size_t)255;
  const size_t plane_bytes = light_grads ? (size_t)(kGradParams + 1) * ctx->wf.capacity * 4 : 0;
  if ((st = ensure_scratch(ctx, sample_bytes + plane_bytes))) return st;
  float* samples = (float*)ctx->d_scratch;
  if (light_grads) {
    A.s_grad = (float*)((char*)ctx->d_scratch + sample_bytes);
    A.s_gkey = (uint32_t*)(A.s_grad + (size_t)kGradParams * ctx->wf.capacity);
  }
  for (uint32_t p0 = pix_begin; p0 < pix_end; p0 += cp) {
    const uint32_t n = std::min(cp, pix_end - p0);
    const uint64_t first = (uint64_t)p0 * L.spp;
    if ((st = render_wavefront(ctx, job, L, first, n * L.spp, samples, s))) return st;
    if ((st = render_wavefront(ctx, job, L, first, n * L.spp, samples, s, &A))) return st;
  }
  return TPT_OK;
}

tpt_status tpt_adjoint(tpt_context* ctx, const tpt_render_job* job, const tpt_adjoint_desc* adesc,
                       const float* d_image, double* grad) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  if (!job || !job->scene || !d_image || !grad) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL argument");
  if (tpt_status st = set_device(ctx)) return st;
  const size_t ibytes =
      (size_t)(adesc && adesc->num_pixels ? adesc->num_pixels : (uint64_t)job->width * job->height) * 12;
  const size_t gbytes = (size_t)job->scene->render.num_materials * kGradParams * sizeof(double);
  float* di = nullptr;
  double* dg = nullptr;
  tpt_status st = cuda_check(ctx, cudaMallocAsync((void**)&di, ibytes, ctx->stream), "cudaMallocAsync(d_image)");
  if (!st) st = cuda_check(ctx, cudaMallocAsync((void**)&dg, gbytes, ctx->stream), "cudaMallocAsync(gradients)");
  if (!st)
    st = cuda_check(ctx, cudaMemcpyAsync(di, d_image, ibytes, cudaMemcpyHostToDevice, ctx->stream), "H2D d_image");
  if (!st) st = tpt_adjoint_device(ctx, job, adesc, di, dg, nullptr);
  if (!st) st = cuda_check(ctx, cudaMemcpyAsync(grad, dg, gbytes, cudaMemcpyDeviceToHost, ctx->stream), "D2H gradients");
  if (di) cudaFreeAsync(di, ctx->stream);
  if (dg) cudaFreeAsync(dg, ctx->stream);
  if (!st) st = check_device_errors(ctx, ctx->stream);
  return st;
}

}  // extern "C"
