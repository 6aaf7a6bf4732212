// C ABI: batched rendering — many jobs of uneven resolution, spp, depth and
// scene through one wavefront launch sequence (the rayon loop of main.rs:
// 99-126, once per image there, as one device pipeline here).
//
// The jobs' paths form one index space (job after job, path = pixel * spp +
// sample within a job).  It is cut into chunks of at most the wavefront
// capacity, on pixel boundaries so that each pixel's samples are accumulated
// in order within one chunk.  Each chunk runs generate -> (traverse -> shade
// -> shadow traverse -> resolve) x (deepest job in the chunk + 1) -> finalize,
// with every stage reading each slot's job record, then one accumulate launch
// per job segment of the chunk.
#include <algorithm>
#include <cstring>
#include <string>

#include "internal.h"

using namespace tpt;

namespace {

struct Segment {  // the pixels [p0, p0 + n) of job j inside one chunk
  uint32_t job;
  uint32_t p0, n;
  uint64_t sample_offset;  // first sample of the segment, chunk-relative
};
struct Chunk {
  uint64_t first_path;
  uint32_t n_paths;
  uint32_t max_depth;
  std::vector<Segment> segs;
};

std::vector<Chunk> plan_chunks(const std::vector<RenderLaunch>& L, const std::vector<uint64_t>& path_base,
                               uint32_t capacity) {
  std::vector<Chunk> chunks;
  Chunk cur{path_base.empty() ? 0 : path_base[0], 0, 0, {}};
  for (uint32_t j = 0; j < L.size(); ++j) {
    const uint32_t npix = L[j].width * L[j].height;
    uint32_t p = 0;
    while (p < npix) {
      uint64_t room = capacity - cur.n_paths;
      uint64_t fit = room / L[j].spp;
      if (fit == 0) {
        chunks.push_back(cur);
        cur = Chunk{path_base[j] + (uint64_t)p * L[j].spp, 0, 0, {}};
        continue;
      }
      const uint32_t take = (uint32_t)std::min<uint64_t>(fit, npix - p);
      if (cur.n_paths == 0) cur.first_path = path_base[j] + (uint64_t)p * L[j].spp;
      cur.segs.push_back(Segment{j, p, take, (uint64_t)cur.n_paths});
      cur.n_paths += take * L[j].spp;
      cur.max_depth = std::max(cur.max_depth, L[j].max_depth);
      p += take;
    }
  }
  if (cur.n_paths) chunks.push_back(cur);
  return chunks;
}

tpt_status ensure_jobs(tpt_context* ctx, size_t n) {
  if (ctx->d_jobs_cap >= n) return TPT_OK;
  if (ctx->d_jobs) {
    cudaDeviceSynchronize();
    cudaFree(ctx->d_jobs);
  }
  ctx->d_jobs = nullptr;
  ctx->d_jobs_cap = 0;
  tpt_status st = cuda_check(ctx, cudaMalloc((void**)&ctx->d_jobs, n * sizeof(DevJob)), "cudaMalloc(job table)");
  if (st) return st;
  ctx->d_jobs_cap = n;
  return TPT_OK;
}

}  // namespace

namespace tpt {

tpt_status render_batch(tpt_context* ctx, const tpt_render_job* jobs, int n_jobs, float* const* out_rgb,
                        cudaStream_t s, uint32_t capacity) {
  std::vector<RenderLaunch> L(n_jobs);
  std::vector<DevJob> dj(n_jobs);
  std::vector<uint64_t> path_base(n_jobs);
  uint64_t paths = 0, pixels = 0;
  for (int j = 0; j < n_jobs; ++j) {
    tpt_status st = render_launch_params(ctx, &jobs[j], &L[j]);
    if (st) return st;
    if (jobs[j].integrator == TPT_INTEGRATOR_BDPT)
      return set_error(ctx, TPT_ERR_INVALID_ARG, "batched rendering covers the MIS, NEE and PT integrators");
    if (!out_rgb[j]) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL output image for job " + std::to_string(j));
    std::memset(&dj[j], 0, sizeof(DevJob));
    dj[j].render = DevRender{jobs[j].scene->geo, jobs[j].scene->render};
    dj[j].P = L[j];
    dj[j].path_base = paths;
    dj[j].pixel_base = pixels;
    dj[j].out = out_rgb[j];
    path_base[j] = paths;
    paths += (uint64_t)L[j].width * L[j].height * L[j].spp;
    pixels += (uint64_t)L[j].width * L[j].height;
  }
  if (n_jobs == 0) return TPT_OK;
  if (capacity == 0) capacity = kDefaultWavefrontSlots;
  uint32_t max_spp = 0;
  for (auto& l : L) max_spp = std::max(max_spp, l.spp);
  if (max_spp > capacity)
    return set_error(ctx, TPT_ERR_CAPACITY, "a pixel's spp exceeds the wavefront capacity of the batch");
  tpt_status st = ensure_jobs(ctx, n_jobs);
  if (!st) st = ensure_wavefront(ctx, capacity);
  if (!st) st = ensure_scratch(ctx, (size_t)capacity * 12);
  if (st) return st;
  if ((st = cuda_check(ctx, cudaMemcpyAsync(ctx->d_jobs, dj.data(), n_jobs * sizeof(DevJob), cudaMemcpyHostToDevice, s),
                       "upload job table")))
    return st;
  bool alpha = false;
  for (int j = 0; j < n_jobs; ++j) alpha = alpha || jobs[j].scene->geo.inst_alpha != nullptr;
  const WfBuffers B = wavefront_view(ctx->wf, alpha);
  float* samples = (float*)ctx->d_scratch;
  const DevGeometry no_geo{};
  bool lights = false;
  for (int j = 0; j < n_jobs; ++j) lights = lights || jobs[j].scene->render.num_extra_lights > 0;
  for (const Chunk& c : plan_chunks(L, path_base, capacity)) {
    cudaError_t e = launch_wf_generate_batch(ctx->d_jobs, (uint32_t)n_jobs, B, c.first_path, c.n_paths, s);
    for (uint32_t b = 0; e == cudaSuccess && b <= c.max_depth; ++b)
      e = enqueue_bounce(ctx, s, no_geo, DevRenderData{}, RenderLaunch{}, B, ctx->d_jobs, (int)(b & 1u), b > 0,
                         lights);
    if (e == cudaSuccess) e = launch_wf_finalize(B, c.n_paths, samples, s);
    for (const Segment& g : c.segs) {
      if (e != cudaSuccess) break;
      e = launch_accumulate(samples + 3 * g.sample_offset, L[g.job].spp, g.p0, g.n, L[g.job].cam.exposure,
                            out_rgb[g.job], s);
    }
    if ((st = cuda_check(ctx, e, "batched wavefront launch"))) return st;
  }
  return TPT_OK;
}

}  // namespace tpt

extern "C" {

tpt_status tpt_render_batch_device(tpt_context* ctx, const tpt_render_job* jobs, int n_jobs, float* const* out_rgb,
                                   void* stream) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  if (n_jobs < 0 || (n_jobs && (!jobs || !out_rgb))) return set_error(ctx, TPT_ERR_INVALID_ARG, "bad job list");
  if (tpt_status st = set_device(ctx)) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  note_device_call(ctx, "tpt_render_batch_device");
  if (ctx->batch_per_job) {  // tpt_autotune found the jobs faster one after another
    for (int j = 0; j < n_jobs; ++j)
      if (tpt_status st = tpt_render_device(ctx, &jobs[j], out_rgb[j], (void*)s)) return st;
    return TPT_OK;
  }
  return render_batch(ctx, jobs, n_jobs, out_rgb, s, ctx->batch_capacity);
}

}  // extern "C"
