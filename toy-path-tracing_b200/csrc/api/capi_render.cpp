// C ABI: rendering (the rayon per-pixel loop of main.rs:99-126 as device launches).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "internal.h"

using namespace tpt;

namespace {

uint32_t log2_int(uint32_t v) { return 31u - (uint32_t)__builtin_clz(v); }
uint32_t round_up_pow2(uint32_t v) { return v <= 1 ? 1u : 1u << (32u - (uint32_t)__builtin_clz(v - 1)); }

struct F3 {
  float x, y, z;
};
F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
F3 cross(F3 a, F3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
F3 normalize(F3 a) {
  float r = 1.0f / std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  return {a.x * r, a.y * r, a.z * r};
}

tpt_status make_launch(tpt_context* ctx, const tpt_render_job* job, RenderLaunch* L) {
  if (!job || !job->scene) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL job or scene");
  if (job->width == 0 || job->height == 0 || job->spp == 0)
    return set_error(ctx, TPT_ERR_INVALID_ARG, "width, height and spp must be positive");
  if (job->integrator != TPT_INTEGRATOR_MIS && job->integrator != TPT_INTEGRATOR_BDPT &&
      job->integrator != TPT_INTEGRATOR_NEE && job->integrator != TPT_INTEGRATOR_PT)
    return set_error(ctx, TPT_ERR_INVALID_ARG, "unknown integrator");
  if (job->integrator == TPT_INTEGRATOR_BDPT && job->max_depth > kBdptMaxDepthApi)
    return set_error(ctx, TPT_ERR_CAPACITY,
                     "BDPT max_depth " + std::to_string(job->max_depth) + " above the device limit of " +
                         std::to_string(kBdptMaxDepthApi));
  if (job->execution != TPT_EXEC_WAVEFRONT && job->execution != TPT_EXEC_MEGAKERNEL &&
      job->execution != TPT_EXEC_AUTO)
    return set_error(ctx, TPT_ERR_INVALID_ARG, "unknown execution mode");
  if (job->scene->render.num_materials == 0)
    return set_error(ctx, TPT_ERR_INVALID_ARG, "scene has no materials: upload materials to render");
  if (job->spp > (1u << 24)) return set_error(ctx, TPT_ERR_INVALID_ARG, "spp above 2^24");
  std::memset(L, 0, sizeof *L);
  // PinholeCamera::new (scene/camera.rs:22-39)
  const tpt_camera_desc& c = job->camera;
  F3 eye{c.eye[0], c.eye[1], c.eye[2]}, at{c.look_at[0], c.look_at[1], c.look_at[2]}, up{c.up[0], c.up[1], c.up[2]};
  F3 fwd = normalize(sub(at, eye));
  F3 right = normalize(cross(fwd, up));
  F3 iup = normalize(cross(right, fwd));
  const float v[12] = {eye.x, eye.y, eye.z, fwd.x, fwd.y, fwd.z, right.x, right.y, right.z, iup.x, iup.y, iup.z};
  std::memcpy(L->cam.eye, v, 12);
  std::memcpy(L->cam.forward, v + 3, 12);
  std::memcpy(L->cam.right, v + 6, 12);
  std::memcpy(L->cam.up, v + 9, 12);
  L->cam.tan_half_fov_y = std::tan(0.5f * c.fov_y);
  L->cam.exposure = c.exposure;
  L->width = job->width;
  L->height = job->height;
  L->spp = job->spp;
  L->max_depth = job->max_depth;
  L->integrator = job->integrator;
  L->seed = job->seed;
  // IndexSampler::new (sampler/zsobol.rs:213-224)
  L->log2_spp = log2_int(round_up_pow2(job->spp));
  const uint32_t res = round_up_pow2(std::max(job->width, job->height));
  L->n_base4_digits = log2_int(res) + (L->log2_spp + 1) / 2;
  if (2 * L->n_base4_digits + 2 > 64) return set_error(ctx, TPT_ERR_CAPACITY, "resolution x spp beyond 64-bit Morton index");
  return TPT_OK;
}

}  // namespace

namespace tpt {
tpt_status ensure_scratch(tpt_context* ctx, size_t bytes) {
  if (ctx->d_scratch_bytes >= bytes) return TPT_OK;
  if (ctx->d_scratch) {
    cudaDeviceSynchronize();
    cudaFree(ctx->d_scratch);
  }
  ctx->d_scratch = nullptr;
  ctx->d_scratch_bytes = 0;
  tpt_status st = cuda_check(ctx, cudaMalloc(&ctx->d_scratch, bytes), "cudaMalloc(render scratch)");
  if (st) return st;
  ctx->d_scratch_bytes = bytes;
  return TPT_OK;
}

// The arena as a render sees it: without alpha tests its AuxRng planes are
// left out (NULL), so the stages skip that bookkeeping.
WfBuffers wavefront_view(const WfBuffers& B, bool alpha) {
  WfBuffers v = B;
  if (!alpha) {
    v.q_aux = nullptr;
    v.s_aux = nullptr;
    v.s_aux_cont = nullptr;
  }
  return v;
}

// Carves the wavefront arena for `capacity` path slots.
tpt_status ensure_wavefront(tpt_context* ctx, uint32_t capacity) {
  if (ctx->wf.capacity >= capacity && ctx->d_wf) return TPT_OK;
  const size_t C = capacity;
  // float planes: beta 3, L 3, prev 7, q_ray 2*7, h_t 1, h_bary 3, s_ray 7, s_contrib 3, s_t 1, s_dist 1
  // u32 planes: prev_mat, depth, q_slot 2, h_tri, h_inst, s_slot, s_target 2, s_tri, s_inst,
  // job, q_job 2, s_job; lock 1; q_aux, s_aux, s_aux_cont
  const size_t planes = 3 + 3 + 7 + 14 + 1 + 3 + 7 + 3 + 1 + 1 + 1 + 1 + 2 + 1 + 1 + 1 + 2 + 1 + 1 + 4 + 1 + 3;
  const size_t bytes = planes * C * 4 + 256;
  if (ctx->d_wf) {
    cudaDeviceSynchronize();
    cudaFree(ctx->d_wf);
    ctx->d_wf = nullptr;
    ctx->d_wf_bytes = 0;
    ctx->wf = WfBuffers{};
  }
  tpt_status st = cuda_check(ctx, cudaMalloc(&ctx->d_wf, bytes), "cudaMalloc(wavefront arena)");
  if (st) return st;
  ctx->d_wf_bytes = bytes;
  char* p = (char*)ctx->d_wf;
  auto take = [&](size_t n_planes) {
    char* r = p;
    p += n_planes * C * 4;
    return r;
  };
  WfBuffers& B = ctx->wf;
  B.capacity = capacity;
  B.beta = (float*)take(3);
  B.L = (float*)take(3);
  B.prev = (float*)take(7);
  B.prev_mat = (uint32_t*)take(1);
  B.depth = (uint32_t*)take(1);
  B.lock = (float*)take(1);
  B.q_aux = (uint32_t*)take(1);
  B.s_aux = (uint32_t*)take(1);
  B.s_aux_cont = (uint32_t*)take(1);
  B.q_slot[0] = (uint32_t*)take(1);
  B.q_slot[1] = (uint32_t*)take(1);
  B.q_ray[0] = (float*)take(7);
  B.q_ray[1] = (float*)take(7);
  B.h_tri = (int32_t*)take(1);
  B.h_inst = (int32_t*)take(1);
  B.h_t = (float*)take(1);
  B.h_bary = (float*)take(3);
  B.s_slot = (uint32_t*)take(1);
  B.s_ray = (float*)take(7);
  B.s_contrib = (float*)take(3);
  B.s_target = (uint32_t*)take(2);
  B.s_tri = (int32_t*)take(1);
  B.s_inst = (int32_t*)take(1);
  B.s_t = (float*)take(1);
  B.s_dist = (float*)take(1);
  B.job = (uint32_t*)take(1);
  B.q_job[0] = (uint32_t*)take(1);
  B.q_job[1] = (uint32_t*)take(1);
  B.s_job = (uint32_t*)take(1);
  B.counts = (uint32_t*)p;
  return TPT_OK;
}

// Paths [first, first + n) through the wavefront stages; radiance per path into
// samples.  With A, the adjoint replay instead: samples holds the paths'
// radiance from a forward pass and the gradients go to A->grad.
tpt_status render_wavefront(tpt_context* ctx, const tpt_render_job* job, const RenderLaunch& L, uint64_t first,
                            uint32_t n, float* samples, cudaStream_t s, const DevAdjoint* A) {
  tpt_status st = ensure_wavefront(ctx, n);
  if (st) return st;
  const DevGeometry& geo = job->scene->geo;
  const WfBuffers B = wavefront_view(ctx->wf, geo.inst_alpha != nullptr);
  const DevRenderData& rd = job->scene->render;
  cudaError_t e = launch_wf_generate(geo, rd, L, B, first, n, s, A ? samples : nullptr);
  // direct launches for the adjoint replay and while render statistics are on
  const bool direct = A || ctx->render_stats;
  unsigned long long* tot = ctx->render_stats;
  for (uint32_t b = 0; !direct && e == cudaSuccess && b <= L.max_depth; ++b)
    e = enqueue_bounce(ctx, s, geo, rd, L, B, nullptr, (int)(b & 1u), b > 0);
  // the step order of the bounce graphs: step b runs the shadow stage of
  // bounce b - 1 on the side stream beside bounce b's path traversal (joined
  // before shade; in sequence with alpha tests or without a side stream)
  const bool branch = direct && !B.q_aux && !B.s_aux && ensure_branch(ctx);
  for (uint32_t b = 0; direct && e == cudaSuccess && b <= L.max_depth; ++b) {
    const int cur = (int)(b & 1u);
    const bool split = branch && b > 0;
    if (split) {
      e = cudaEventRecord(ctx->cap_fork, s);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->cap_side, ctx->cap_fork, 0);
    }
    const cudaStream_t ss = split ? ctx->cap_side : s;
    if (e == cudaSuccess && b > 0)
      e = launch_traverse_strided(geo, B.s_ray, B.capacity, B.capacity, TPT_CLOSEST_HIT, B.s_tri, B.s_t, B.s_inst,
                                  nullptr, B.capacity, next_counter(ctx), ctx->d_err, ctx->num_sms, ss, nullptr,
                                  nullptr, B.counts + 2, nullptr, nullptr, tot ? tot + 4 : nullptr, B.s_aux);
    if (e == cudaSuccess && b > 0) e = launch_wf_resolve(B, ss, A);
    if (e == cudaSuccess) e = cudaMemsetAsync(B.counts + (cur ^ 1), 0, 4, s);
    if (e == cudaSuccess)
      e = launch_traverse_strided(geo, B.q_ray[cur], B.capacity, B.capacity, TPT_CLOSEST_HIT, B.h_tri, B.h_t,
                                  B.h_inst, B.h_bary, B.capacity, next_counter(ctx), ctx->d_err, ctx->num_sms, s,
                                  nullptr, nullptr, B.counts + cur, nullptr, nullptr, tot, B.q_aux, B.q_slot[cur]);
    if (split) {  // join even after an error: no branch is left open on the caller's stream
      const cudaError_t ej = cudaEventRecord(ctx->cap_join, ctx->cap_side);
      const cudaError_t ew = ej == cudaSuccess ? cudaStreamWaitEvent(s, ctx->cap_join, 0) : ej;
      if (e == cudaSuccess) e = ew;
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(B.counts + 2, 0, 4, s);
    if (e == cudaSuccess) e = launch_wf_shade(geo, rd, L, B, cur, s, A);
  }
  if (e == cudaSuccess && !A) e = launch_wf_finalize(B, n, samples, s);
  return cuda_check(ctx, e, "wavefront launch");
}

// BDPT wavefront arena for `max_vertices` vertices per subpath and a job of
// `n` samples: a chunk holds all of them, or as many as keep the connection
// queue at 2^TPT_BD_PAIRS_LOG2 slots (each sample has at most max_vertices^2
// connections; 2^27 slots are about 14 GB at 10 vertices, which large chunks
// repay: the late subpath steps, with few rays left, run once per chunk), a
// multiple of 128 so that no warp of bd_step straddles the camera and light
// halves of a ray queue.  The arena only grows.
#ifndef TPT_BD_PAIRS_LOG2
#define TPT_BD_PAIRS_LOG2 27
#endif
tpt_status ensure_bdpt_wavefront(tpt_context* ctx, uint32_t max_vertices, uint64_t n) {
  const uint32_t mv = std::max<uint32_t>(1, max_vertices);
  const uint64_t cap = std::max<uint64_t>(1024, ((1ull << TPT_BD_PAIRS_LOG2) / ((uint64_t)mv * mv)) & ~(uint64_t)127);
  const uint64_t samples = std::min<uint64_t>(cap, std::max<uint64_t>(1024, (n + 127) & ~(uint64_t)127));
  const uint64_t pairs = samples * mv * mv;
  if (ctx->d_bd && ctx->bd.max_vertices == mv && ctx->bd.sample_capacity >= samples) return TPT_OK;
  const uint64_t q = 2 * samples;  // subpath ray queue slots (camera + light per sample)
  const size_t bytes = samples * 2 * mv * (size_t)kBdVertexBytes + samples * (3 * 4 + 3 * 4) +
                       pairs * (4 + 12 + 12 + 4) + pairs * (7 * 4 + 4 + 4 + 4 + 4) +
                       samples * 2 * (size_t)kBdStateBytes + q * (2 * 7 * 4 + 2 * 4 + 4 + 4 + 4 + 12) + 32 * 256;
  if (ctx->d_bd) {
    cudaDeviceSynchronize();
    cudaFree(ctx->d_bd);
    ctx->d_bd = nullptr;
    ctx->d_bd_bytes = 0;
    ctx->bd = BdWfBuffers{};
  }
  tpt_status st = cuda_check(ctx, cudaMalloc(&ctx->d_bd, bytes), "cudaMalloc(BDPT wavefront arena)");
  if (st) return st;
  ctx->d_bd_bytes = bytes;
  char* p = (char*)ctx->d_bd;
  auto take = [&](size_t b) {
    char* r = p;
    p += (b + 255) & ~(size_t)255;
    return r;
  };
  BdWfBuffers& B = ctx->bd;
  B.sample_capacity = (uint32_t)samples;
  B.pair_capacity = (uint32_t)pairs;
  B.max_vertices = mv;
  B.verts = (BdVertex*)take(samples * 2 * mv * (size_t)kBdVertexBytes);
  B.nc = (uint32_t*)take(samples * 4);
  B.nl = (uint32_t*)take(samples * 4);
  B.pair_base = (uint32_t*)take(samples * 4);
  B.L0 = (float*)take(samples * 12);
  B.pair_sample = (uint32_t*)take(pairs * 4);
  B.c = (float*)take(pairs * 12);
  B.contrib = (float*)take(pairs * 12);
  B.dist = (float*)take(pairs * 4);
  B.s_ray = (float*)take(pairs * 28);
  B.s_pair = (uint32_t*)take(pairs * 4);
  B.s_tri = (int32_t*)take(pairs * 4);
  B.s_inst = (int32_t*)take(pairs * 4);
  B.s_t = (float*)take(pairs * 4);
  B.cam_state = (BdCamState*)take(samples * kBdStateBytes);
  B.light_state = (BdLightState*)take(samples * kBdStateBytes);
  for (int k = 0; k < 2; ++k) {
    B.q_ray[k] = (float*)take(q * 28);
    B.q_tag[k] = (uint32_t*)take(q * 4);
  }
  B.h_tri = (int32_t*)take(q * 4);
  B.h_inst = (int32_t*)take(q * 4);
  B.h_t = (float*)take(q * 4);
  B.h_bary = (float*)take(q * 12);
  B.counts = (uint32_t*)take(256);
  return TPT_OK;
}

tpt_status render_bdpt_wavefront(tpt_context* ctx, const tpt_render_job* job, const RenderLaunch& L, uint64_t first,
                                 uint64_t n, float* samples, cudaStream_t s) {
  // Alpha tests draw every connection's visibility test from one AuxRng per
  // sample, in connection order (bdpt.rs:81-121): the one-kernel execution,
  // whose lanes run their connections in that order, renders such scenes.
  if (job->scene->geo.inst_alpha)
    return cuda_check(ctx,
                      launch_render(job->scene->geo, job->scene->render, L, samples, first, n, ctx->d_err,
                                    ctx->num_sms, s, next_counter(ctx)),
                      "render kernel launch");
  tpt_status st = ensure_bdpt_wavefront(ctx, L.max_depth, n);
  if (st) return st;
  const BdWfBuffers& B = ctx->bd;
  for (uint64_t b = 0; b < n; b += B.sample_capacity) {
    const uint32_t m = (uint32_t)std::min<uint64_t>(B.sample_capacity, n - b);
    const bool branch = ensure_branch(ctx);
    cudaError_t e = launch_bdpt_wavefront(job->scene->geo, job->scene->render, L, B, first + b, m, samples + 3 * b,
                                          next_counter(ctx), ctx->d_err, ctx->num_sms, s, ctx->render_stats,
                                          next_counter(ctx), branch ? ctx->cap_side : nullptr, ctx->cap_fork,
                                          ctx->cap_join);
    if ((st = cuda_check(ctx, e, "BDPT wavefront launch"))) return st;
  }
  return TPT_OK;
}

// Pixels per chunk: the per-sample buffer stays below 1 GiB and a chunk has at
// most `capacity` paths (the wavefront arena's slot count; 0 = the default).
uint32_t chunk_pixels(const RenderLaunch& L, uint32_t capacity) {
  if (capacity == 0) capacity = kDefaultWavefrontSlots;
  const uint64_t per_pixel = 12ull * L.spp;
  uint64_t n = std::min<uint64_t>((1ull << 30) / per_pixel, std::max<uint64_t>(1, (uint64_t)capacity / L.spp));
  const uint64_t total = (uint64_t)L.width * L.height;
  return (uint32_t)std::max<uint64_t>(1, std::min(n, total));
}


tpt_status render_launch_params(tpt_context* ctx, const tpt_render_job* job, RenderLaunch* out) {
  return make_launch(ctx, job, out);
}
}  // namespace tpt

extern "C" {

tpt_status tpt_context_set_wavefront_capacity(tpt_context* ctx, uint32_t slots) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  if (slots != 0 && (slots < 1024 || slots > (1u << 26)))
    return set_error(ctx, TPT_ERR_INVALID_ARG, "wavefront capacity must be 0 or in [1024, 2^26]");
  ctx->batch_capacity = slots;
  ctx->batch_per_job = false;  // a capacity set by hand is for batched launches
  return TPT_OK;
}

tpt_status tpt_context_set_shade_block(tpt_context* ctx, uint32_t threads) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  if (threads != 128 && threads != 256) return set_error(ctx, TPT_ERR_INVALID_ARG, "shade block must be 128 or 256");
  ctx->shade_block = threads;
  return TPT_OK;
}

tpt_status tpt_context_set_render_stats(tpt_context* ctx, uint64_t* d_counters) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  ctx->render_stats = reinterpret_cast<unsigned long long*>(d_counters);
  return TPT_OK;
}

tpt_status tpt_context_set_graphs(tpt_context* ctx, int enable) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  ctx->use_graphs = enable != 0;
  return TPT_OK;
}

uint32_t tpt_context_wavefront_capacity(const tpt_context* ctx) {
  return ctx ? (ctx->batch_capacity ? ctx->batch_capacity : kDefaultWavefrontSlots) : 0u;
}

tpt_status tpt_render_device(tpt_context* ctx, const tpt_render_job* job, float* out_rgb, void* stream) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  if (!job) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL job");
  return tpt_render_pixels_device(ctx, job, 0, (uint64_t)job->width * job->height, out_rgb, stream);
}

tpt_status tpt_render_pixels_device(tpt_context* ctx, const tpt_render_job* job, uint64_t first_pixel,
                                    uint64_t num_pixels, float* out_rgb, void* stream) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  if (!out_rgb) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL output");
  RenderLaunch L;
  tpt_status st = make_launch(ctx, job, &L);
  if (st) return st;
  const uint64_t total = (uint64_t)L.width * L.height;
  if (first_pixel > total || num_pixels > total - first_pixel)
    return set_error(ctx, TPT_ERR_INVALID_ARG, "pixel range out of bounds");
  if ((st = set_device(ctx))) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  note_device_call(ctx, first_pixel == 0 && num_pixels == total ? "tpt_render_device" : "tpt_render_pixels_device");
  const uint32_t pix_begin = (uint32_t)first_pixel, pix_end = (uint32_t)(first_pixel + num_pixels);
  const uint32_t cp = chunk_pixels(L, ctx->batch_capacity);
  if ((st = ensure_scratch(ctx, (size_t)cp * L.spp * 12))) return st;
  float* samples = (float*)ctx->d_scratch;
  const uint32_t exec = job->execution == TPT_EXEC_AUTO ? ctx->tuned_execution : job->execution;
  for (uint32_t p0 = pix_begin; p0 < pix_end; p0 += cp) {
    const uint32_t n = std::min(cp, pix_end - p0);
    if (job->integrator == TPT_INTEGRATOR_BDPT && exec != TPT_EXEC_MEGAKERNEL) {
      if ((st = render_bdpt_wavefront(ctx, job, L, (uint64_t)p0 * L.spp, (uint64_t)n * L.spp, samples, s))) return st;
    } else if (exec == TPT_EXEC_MEGAKERNEL || job->integrator == TPT_INTEGRATOR_BDPT) {
      cudaError_t e = launch_render(job->scene->geo, job->scene->render, L, samples, (uint64_t)p0 * L.spp,
                                    (uint64_t)n * L.spp, ctx->d_err, ctx->num_sms, s, next_counter(ctx));
      if ((st = cuda_check(ctx, e, "render kernel launch"))) return st;
    } else {
      if ((st = render_wavefront(ctx, job, L, (uint64_t)p0 * L.spp, n * L.spp, samples, s))) return st;
    }
    cudaError_t e = launch_accumulate(samples, L.spp, p0 - pix_begin, n, L.cam.exposure, out_rgb, s);
    if ((st = cuda_check(ctx, e, "accumulate kernel launch"))) return st;
  }
  return TPT_OK;
}

tpt_status tpt_render_samples_device(tpt_context* ctx, const tpt_render_job* job, uint64_t first, uint64_t count,
                                     float* out_samples, void* stream) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  RenderLaunch L;
  tpt_status st = make_launch(ctx, job, &L);
  if (st) return st;
  const uint64_t total = (uint64_t)L.width * L.height * L.spp;
  if (first > total || count > total - first) return set_error(ctx, TPT_ERR_INVALID_ARG, "path range out of bounds");
  if (count && !out_samples) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL output");
  if ((st = set_device(ctx))) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  note_device_call(ctx, "tpt_render_samples_device");
  const uint32_t exec = job->execution == TPT_EXEC_AUTO ? ctx->tuned_execution : job->execution;
  if (job->integrator == TPT_INTEGRATOR_BDPT && exec != TPT_EXEC_MEGAKERNEL)
    return render_bdpt_wavefront(ctx, job, L, first, count, out_samples, s);
  if (exec == TPT_EXEC_MEGAKERNEL || job->integrator == TPT_INTEGRATOR_BDPT)
    return cuda_check(ctx,
                      launch_render(job->scene->geo, job->scene->render, L, out_samples, first, count, ctx->d_err,
                                    ctx->num_sms, s, next_counter(ctx)),
                      "render kernel launch");
  const uint64_t step = ctx->batch_capacity ? ctx->batch_capacity : 1ull << 22;
  for (uint64_t b = 0; b < count; b += step) {
    st = render_wavefront(ctx, job, L, first + b, (uint32_t)std::min(step, count - b), out_samples + 3 * b, s);
    if (st) return st;
  }
  return TPT_OK;
}

tpt_status tpt_render(tpt_context* ctx, const tpt_render_job* jobs, int n_jobs, float* const* out_rgb) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  if (n_jobs < 0 || (n_jobs && (!jobs || !out_rgb))) return set_error(ctx, TPT_ERR_INVALID_ARG, "bad job list");
  if (tpt_status st = set_device(ctx)) return st;
  // several MIS wavefront jobs: one batched launch sequence
  bool batch = n_jobs > 1;
  for (int j = 0; j < n_jobs && batch; ++j) {
    const uint32_t ex = jobs[j].execution == TPT_EXEC_AUTO ? ctx->tuned_execution : jobs[j].execution;
    batch = jobs[j].integrator != TPT_INTEGRATOR_BDPT && ex == TPT_EXEC_WAVEFRONT && out_rgb[j] && jobs[j].scene;
  }
  if (batch) {
    std::vector<float*> d(n_jobs, nullptr);
    std::vector<size_t> bytes(n_jobs);
    tpt_status st = TPT_OK;
    for (int j = 0; j < n_jobs && !st; ++j) {
      bytes[j] = (size_t)jobs[j].width * jobs[j].height * 12;
      st = cuda_check(ctx, cudaMallocAsync((void**)&d[j], std::max<size_t>(bytes[j], 16), ctx->stream),
                      "cudaMallocAsync(image)");
    }
    if (!st) st = render_batch(ctx, jobs, n_jobs, d.data(), ctx->stream, ctx->batch_capacity);
    for (int j = 0; j < n_jobs && !st; ++j)
      st = cuda_check(ctx, cudaMemcpyAsync(out_rgb[j], d[j], bytes[j], cudaMemcpyDeviceToHost, ctx->stream),
                      "D2H image");
    for (float* p : d)
      if (p) cudaFreeAsync(p, ctx->stream);
    if (!st) st = check_device_errors(ctx, ctx->stream);
    return st;
  }
  for (int j = 0; j < n_jobs; ++j) {
    if (!out_rgb[j]) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL output image");
    RenderLaunch L;
    tpt_status st = make_launch(ctx, &jobs[j], &L);
    if (st) return st;
    const size_t img_bytes = (size_t)L.width * L.height * 12;
    float* d_img = nullptr;
    if ((st = cuda_check(ctx, cudaMallocAsync((void**)&d_img, img_bytes, ctx->stream), "cudaMallocAsync(image)")))
      return st;
    st = tpt_render_device(ctx, &jobs[j], d_img, nullptr);
    if (!st)
      st = cuda_check(ctx, cudaMemcpyAsync(out_rgb[j], d_img, img_bytes, cudaMemcpyDeviceToHost, ctx->stream),
                      "D2H image");
    cudaFreeAsync(d_img, ctx->stream);
    if (!st) st = check_device_errors(ctx, ctx->stream);
    if (st) return st;
  }
  return TPT_OK;
}

}  // extern "C"
