// C ABI: the autotuner — picks, for a list of render jobs, the execution
// (wavefront, batched when there are several jobs, or megakernel), the
// wavefront's queue capacity and whether bounces replay captured graphs, by
// timing each candidate on a pilot of the workload on the device.
//
// No counterpart in the reference (one CPU code path).  The pilot keeps every
// job's scene, camera, spp and depth and scales its rows down (the same field
// of view at a lower vertical resolution) until the pilot holds at most
// 2^24 paths, or the whole workload when it is smaller.  Each candidate runs
// once to warm up (graph capture, arena growth) and once timed with CUDA
// events on the context's stream.  Results do not depend on any of the tuned
// settings (the tests check this), only the time does.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "internal.h"

using namespace tpt;

namespace {

constexpr uint64_t kPilotPaths = 1ull << 24;

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~Timer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

}  // namespace

extern "C" {

tpt_status tpt_autotune(tpt_context* ctx, const tpt_render_job* jobs, int n_jobs, tpt_tune_result* out) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  if (n_jobs <= 0 || !jobs || !out) return set_error(ctx, TPT_ERR_INVALID_ARG, "bad job list");
  cudaSetDevice(ctx->device);
  uint64_t total = 0;
  for (int j = 0; j < n_jobs; ++j) {
    RenderLaunch L;
    tpt_status st = render_launch_params(ctx, &jobs[j], &L);
    if (st) return st;
    if (jobs[j].integrator != TPT_INTEGRATOR_MIS)
      return set_error(ctx, TPT_ERR_INVALID_ARG, "the autotuner covers MIS jobs");
    total += (uint64_t)L.width * L.height * L.spp;
  }
  // pilot: rows scaled by f
  const double f = total > kPilotPaths ? (double)kPilotPaths / (double)total : 1.0;
  std::vector<tpt_render_job> pilot(jobs, jobs + n_jobs);
  std::vector<float*> imgs(n_jobs, nullptr);
  uint64_t pilot_paths = 0;
  tpt_status st = TPT_OK;
  for (int j = 0; j < n_jobs && !st; ++j) {
    pilot[j].height = std::max<uint32_t>(1, (uint32_t)std::ceil(jobs[j].height * f));
    pilot_paths += (uint64_t)pilot[j].width * pilot[j].height * pilot[j].spp;
    st = cuda_check(ctx, cudaMalloc((void**)&imgs[j], (size_t)pilot[j].width * pilot[j].height * 12),
                    "cudaMalloc(pilot image)");
  }
  const uint32_t saved_cap = ctx->batch_capacity;
  const bool saved_graphs = ctx->use_graphs;
  Timer T;
  auto run = [&](uint32_t exec, uint32_t cap, bool graphs, float* ms) -> tpt_status {
    ctx->batch_capacity = cap;
    ctx->use_graphs = graphs;
    for (int rep = 0; rep < 2; ++rep) {
      if (rep == 1) cudaEventRecord(T.a, ctx->stream);
      tpt_status s2 = TPT_OK;
      if (exec == TPT_EXEC_WAVEFRONT && n_jobs > 1) {
        s2 = render_batch(ctx, pilot.data(), n_jobs, imgs.data(), ctx->stream, cap);
      } else {
        for (int j = 0; j < n_jobs && !s2; ++j) {
          tpt_render_job pj = pilot[j];
          pj.execution = exec;
          s2 = tpt_render_device(ctx, &pj, imgs[j], nullptr);
        }
      }
      if (s2) return s2;
    }
    cudaEventRecord(T.b, ctx->stream);
    cudaError_t e = cudaEventSynchronize(T.b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, T.a, T.b);
    return cuda_check(ctx, e, "autotune timing");
  };
  tpt_tune_result best{};
  best.ms = 1e30f;
  float ms_default = 0.0f, ms_mk = 0.0f;
  if (!st) st = run(TPT_EXEC_MEGAKERNEL, 0, false, &ms_mk);
  const uint32_t caps[] = {1u << 18, 1u << 19, 1u << 20, 1u << 21, 1u << 22, 1u << 23};
  for (uint32_t cap : caps) {
    if (st) break;
    if (cap > 2 * std::max<uint64_t>(pilot_paths, 1u << 18)) break;  // larger queues than the pilot gain nothing
    for (int g = 1; g >= 0 && !st; --g) {
      float ms = 0.0f;
      st = run(TPT_EXEC_WAVEFRONT, cap, g != 0, &ms);
      if (st) break;
      if (cap == (1u << 22) && g == 1) ms_default = ms;
      if (ms < best.ms) {
        best.ms = ms;
        best.execution = TPT_EXEC_WAVEFRONT;
        best.wavefront_capacity = cap;
        best.graphs = (uint32_t)g;
      }
    }
  }
  for (float* p : imgs)
    if (p) cudaFree(p);
  ctx->batch_capacity = saved_cap;
  ctx->use_graphs = saved_graphs;
  if (st) return st;
  if (ms_mk < best.ms) {
    best.ms = ms_mk;
    best.execution = TPT_EXEC_MEGAKERNEL;
    best.wavefront_capacity = saved_cap;
    best.graphs = saved_graphs ? 1u : 0u;
  }
  best.ms_megakernel = ms_mk;
  best.ms_wavefront_default = ms_default;
  best.pilot_paths = pilot_paths;
  // apply
  ctx->tuned_execution = best.execution;
  if (best.execution == TPT_EXEC_WAVEFRONT) {
    ctx->batch_capacity = best.wavefront_capacity;
    ctx->use_graphs = best.graphs != 0;
  }
  *out = best;
  return TPT_OK;
}

}  // extern "C"
