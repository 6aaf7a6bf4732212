// C ABI: the autotuner — picks, for a list of render jobs, the execution
// (wavefront, batched when there are several jobs, or megakernel), the
// wavefront's queue capacity and whether bounces replay captured graphs, by
// timing each candidate on a pilot of the workload on the device.
//
// No counterpart in the reference (one CPU code path).  A pilot keeps every
// job's scene, camera, spp and depth and scales its rows down (the same field
// of view at a lower vertical resolution).  Stage 1 times every candidate on a
// pilot of at most 2^24 paths (the whole workload when it is smaller); stage 2
// re-times the candidates within 5 % of the best, the default and the
// megakernel on a pilot four times larger, whose chunks look more like the
// full workload's.  On the last pilot the best wavefront candidate is also
// timed with the other shade-stage block size (128 or 256 threads).  Every time
// the result reports comes from that last pilot, so they compare directly.
// Each timing is one warm-up (graph capture, arena growth) and the median of
// three runs, CUDA events on the context's stream.  A candidate replaces the
// default wavefront settings (kDefaultWavefrontSlots slots, graphs, the context's block size)
// only when it is more than 3 % faster.  Results do not depend on any of the
// tuned settings (the tests check this), only the time does.
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
  if (tpt_status st = set_device(ctx)) return st;
  uint64_t total = 0;
  for (int j = 0; j < n_jobs; ++j) {
    RenderLaunch L;
    tpt_status st = render_launch_params(ctx, &jobs[j], &L);
    if (st) return st;
    if (jobs[j].integrator == TPT_INTEGRATOR_BDPT)
      return set_error(ctx, TPT_ERR_INVALID_ARG, "the autotuner covers MIS, NEE and PT jobs");
    total += (uint64_t)L.width * L.height * L.spp;
  }
  struct Pilot {
    std::vector<tpt_render_job> jobs;
    std::vector<float*> imgs;
    uint64_t paths = 0;
  };
  // pilot of at most `limit` paths: every job's rows scaled by the same factor
  auto make_pilot = [&](uint64_t limit, Pilot& p) -> tpt_status {
    const double f = total > limit ? (double)limit / (double)total : 1.0;
    p.jobs.assign(jobs, jobs + n_jobs);
    p.imgs.assign(n_jobs, nullptr);
    for (int j = 0; j < n_jobs; ++j) {
      p.jobs[j].height = std::max<uint32_t>(1, (uint32_t)std::ceil(jobs[j].height * f));
      p.paths += (uint64_t)p.jobs[j].width * p.jobs[j].height * p.jobs[j].spp;
      tpt_status s2 = cuda_check(ctx, cudaMalloc((void**)&p.imgs[j], (size_t)p.jobs[j].width * p.jobs[j].height * 12),
                                 "cudaMalloc(pilot image)");
      if (s2) return s2;
    }
    return TPT_OK;
  };
  auto free_pilot = [](Pilot& p) {
    for (float* x : p.imgs)
      if (x) cudaFree(x);
    p.imgs.clear();
  };
  struct Cand {
    uint32_t exec, cap, graphs, block;
    float ms;
    bool per_job = false;  // several jobs: wavefront job by job instead of one batch
  };
  const uint32_t saved_cap = ctx->batch_capacity;
  const bool saved_graphs = ctx->use_graphs;
  const uint32_t saved_block = ctx->shade_block;
  Timer T;
  // one warm-up, then the median of three timed runs
  auto run = [&](Pilot& p, const Cand& c, float* ms) -> tpt_status {
    ctx->batch_capacity = c.cap;
    ctx->use_graphs = c.graphs != 0;
    ctx->shade_block = c.block;
    float t[3] = {0.0f, 0.0f, 0.0f};
    for (int rep = 0; rep < 4; ++rep) {
      cudaEventRecord(T.a, ctx->stream);
      tpt_status s2 = TPT_OK;
      if (c.exec == TPT_EXEC_WAVEFRONT && n_jobs > 1 && !c.per_job) {
        s2 = render_batch(ctx, p.jobs.data(), n_jobs, p.imgs.data(), ctx->stream, c.cap);
      } else {
        for (int j = 0; j < n_jobs && !s2; ++j) {
          tpt_render_job pj = p.jobs[j];
          pj.execution = c.exec;
          s2 = tpt_render_device(ctx, &pj, p.imgs[j], nullptr);
        }
      }
      if (s2) return s2;
      cudaEventRecord(T.b, ctx->stream);
      cudaError_t e = cudaEventSynchronize(T.b);
      if (e == cudaSuccess && rep > 0) e = cudaEventElapsedTime(&t[rep - 1], T.a, T.b);
      if (e != cudaSuccess) return cuda_check(ctx, e, "autotune timing");
    }
    std::sort(t, t + 3);
    *ms = t[1];
    return TPT_OK;
  };
  // stage 1: every candidate on a pilot of at most 2^24 paths
  Pilot p1;
  tpt_status st = make_pilot(kPilotPaths, p1);
  std::vector<Cand> cands;
  cands.push_back(Cand{TPT_EXEC_MEGAKERNEL, 0, 0, 256, 0.0f});
  const uint32_t caps[] = {1u << 18, 1u << 19, 1u << 20, 1u << 21, 1u << 22, 1u << 23, 1u << 24};
  for (uint32_t cap : caps) {
    if (cap > 2 * std::max<uint64_t>(p1.paths, 1u << 18) && cap != kDefaultWavefrontSlots) continue;  // queues beyond the work
    for (uint32_t g : {1u, 0u}) cands.push_back(Cand{TPT_EXEC_WAVEFRONT, cap, g, saved_block, 0.0f});
  }
  if (n_jobs > 1) cands.push_back(Cand{TPT_EXEC_WAVEFRONT, kDefaultWavefrontSlots, 1u, saved_block, 0.0f, true});
  for (Cand& c : cands) {
    if (st) break;
    st = run(p1, c, &c.ms);
  }
  uint32_t stage = 1;
  Pilot* last = &p1;
  Pilot p2;
  // stage 2: the candidates within 5 % of the best, the default and the
  // megakernel on a pilot four times larger, closer to the full workload's
  // chunk composition
  if (!st && total > kPilotPaths) {
    float best1 = 1e30f;
    for (const Cand& c : cands) best1 = std::min(best1, c.ms);
    st = make_pilot(4 * kPilotPaths, p2);
    for (Cand& c : cands) {
      if (st) break;
      const bool is_default = c.exec == TPT_EXEC_WAVEFRONT && c.cap == kDefaultWavefrontSlots && c.graphs;
      if (c.ms <= 1.05f * best1 || is_default || c.exec == TPT_EXEC_MEGAKERNEL) st = run(p2, c, &c.ms);
      else c.ms = 1e30f;
    }
    stage = 2;
    last = &p2;
  }
  // the other shade block size for the best wavefront candidate, on the last pilot
  if (!st) {
    const Cand* bw = nullptr;
    for (const Cand& c : cands)
      if (c.exec == TPT_EXEC_WAVEFRONT && (!bw || c.ms < bw->ms)) bw = &c;
    if (bw) {
      Cand alt = *bw;
      alt.block = bw->block == 256 ? 128 : 256;
      st = run(*last, alt, &alt.ms);
      cands.push_back(alt);
    }
  }
  free_pilot(p1);
  free_pilot(p2);
  const float ms_mk = cands[0].ms;  // the megakernel on the last pilot
  ctx->batch_capacity = saved_cap;
  ctx->use_graphs = saved_graphs;
  ctx->shade_block = saved_block;
  if (st) return st;
  tpt_tune_result best{};
  best.ms = 1e30f;
  float ms_default = 0.0f;
  for (const Cand& c : cands) {
    if (c.exec == TPT_EXEC_WAVEFRONT && c.cap == kDefaultWavefrontSlots && c.graphs && c.block == saved_block &&
        !c.per_job)
      ms_default = c.ms;
    if (c.ms < best.ms) {
      best.ms = c.ms;
      best.batched = c.per_job ? 0u : 1u;
      best.execution = c.exec;
      best.wavefront_capacity = c.exec == TPT_EXEC_WAVEFRONT ? c.cap : saved_cap;
      best.graphs = c.exec == TPT_EXEC_WAVEFRONT ? c.graphs : (saved_graphs ? 1u : 0u);
      best.shade_block = c.exec == TPT_EXEC_WAVEFRONT ? c.block : saved_block;
    }
  }
  // keep the default wavefront settings unless a wavefront candidate beats
  // them by 3 %: the pilots are scaled-down workloads and carry noise
  if (best.execution == TPT_EXEC_WAVEFRONT && ms_default > 0.0f && best.ms > 0.97f * ms_default) {
    best.ms = ms_default;
    best.batched = 1;
    best.wavefront_capacity = kDefaultWavefrontSlots;
    best.graphs = 1;
    best.shade_block = saved_block;
  }
  best.pilot_paths = std::min<uint64_t>(total, total > kPilotPaths ? 4 * kPilotPaths : total);
  best.ms_megakernel = ms_mk;
  best.ms_wavefront_default = ms_default;
  best.stage = stage;
  best.candidates = (uint32_t)cands.size();
  // apply
  if (n_jobs <= 1) best.batched = 1;
  ctx->tuned_execution = best.execution;
  ctx->batch_per_job = best.execution == TPT_EXEC_WAVEFRONT && best.batched == 0;
  if (best.execution == TPT_EXEC_WAVEFRONT) {
    ctx->batch_capacity = best.wavefront_capacity;
    ctx->use_graphs = best.graphs != 0;
    ctx->shade_block = best.shade_block;
  }
  *out = best;
  return TPT_OK;
}

}  // extern "C"
