// One captured CUDA graph per wavefront bounce.
//
// Step b of the loop b = 0 .. max_depth is a fixed sequence: the shadow stage
// of bounce b - 1 (shadow traversal, resolve) when b > 0, the closest-hit
// traversal of bounce b's ray queue, then its shade stage, which fills the next
// ray queue and the shadow queue.  The shadow stage and the traversal touch
// disjoint buffers (shadow queue, its hit records and the paths' radiance;
// path queue and its hit records), so in a graph they are two branches: a late
// bounce's traversals hold few rays and last as long as their longest ray's
// chain of node loads, and two of them overlap.  Both branches join before
// shade, so every path's radiance receives its additions in the sequential
// order.  With alpha tests the shadow rays' AuxRng draws come before the next
// path ray's (resolve hands the state back), so those steps stay in order.
// A step's launch shapes depend on the arena capacity only (queue lengths
// live on the device) and every chunk-specific value is read from the device
// (the chunk's first path is written by generate), so the same four graphs
// (current queue 0 or 1, with or without a shadow stage before) serve every
// chunk and every bounce of a given (scene, camera, arena) and are replayed
// instead of re-launching ~8 operations per bounce.  Graphs are captured on a
// private non-blocking stream (with a second one for the shadow branch) and
// launched on the caller's stream; a stream that is itself being captured gets
// the plain launches in sequence (they join the caller's graph).
#include <cstring>

#include "internal.h"

namespace tpt {

namespace {

constexpr size_t kMaxGraphSets = kGraphCounterSlots / 2;

struct BounceKey {
  DevRender S;
  RenderLaunch P;
  WfBuffers B;
  const DevJob* jobs;
  uint32_t* err;
  int num_sms;
  int shade_block;
  int batch_lights;
};

// The operations of one step (the shared body of the direct and the captured
// path).  With `side` (capture only) and no alpha tests, the shadow stage runs
// on `side` between the fork and join events; otherwise everything is in
// sequence on `s`.
cudaError_t step_ops(const BounceKey& k, int cur, bool prev_shadow, unsigned long long* c0, unsigned long long* c1,
                     cudaStream_t s, cudaStream_t side = nullptr, cudaEvent_t fork = nullptr,
                     cudaEvent_t join = nullptr) {
  const WfBuffers& B = k.B;
  const bool split = side && prev_shadow && !B.q_aux && !B.s_aux;
  cudaError_t e = cudaSuccess;
  if (split) {
    e = cudaEventRecord(fork, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(side, fork, 0);
  }
  const cudaStream_t ss = split ? side : s;
  if (e == cudaSuccess && prev_shadow)
    e = launch_traverse_strided(k.S.geo, B.s_ray, B.capacity, B.capacity, TPT_CLOSEST_HIT, B.s_tri, B.s_t, B.s_inst,
                                nullptr, B.capacity, c1, k.err, k.num_sms, ss, nullptr, nullptr, B.counts + 2, k.jobs,
                                k.jobs ? B.s_job : nullptr, nullptr, B.s_aux);
  if (e == cudaSuccess && prev_shadow) e = launch_wf_resolve(B, ss);
  if (e == cudaSuccess) e = cudaMemsetAsync(B.counts + (cur ^ 1), 0, 4, s);
  if (e == cudaSuccess)
    e = launch_traverse_strided(k.S.geo, B.q_ray[cur], B.capacity, B.capacity, TPT_CLOSEST_HIT, B.h_tri, B.h_t,
                                B.h_inst, B.h_bary, B.capacity, c0, k.err, k.num_sms, s, nullptr, nullptr,
                                B.counts + cur, k.jobs, k.jobs ? B.q_job[cur] : nullptr, nullptr, B.q_aux,
                                B.q_slot[cur]);
  if (split) {  // join even after an error, so that a capture ends with every branch joined
    const cudaError_t ej = cudaEventRecord(join, side);
    const cudaError_t ew = ej == cudaSuccess ? cudaStreamWaitEvent(s, join, 0) : ej;
    if (e == cudaSuccess) e = ew;
  }
  // the shadow queue of bounce b - 1 is consumed: shade refills it from zero
  if (e == cudaSuccess) e = cudaMemsetAsync(B.counts + 2, 0, 4, s);
  if (e == cudaSuccess)
    e = k.jobs ? launch_wf_shade_batch(k.jobs, B, cur, s, k.shade_block, k.batch_lights != 0)
               : launch_wf_shade(k.S.geo, k.S.d, k.P, B, cur, s, nullptr, k.shade_block);
  return e;
}

}  // namespace

struct BounceGraphSet {
  BounceKey key;
  cudaGraphExec_t exec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  bool failed = false;
  uint64_t last_use = 0;
  uint32_t slot = 0;  // index of its two dedicated work counters
};

bool ensure_branch(tpt_context* ctx) {
  if (!ctx->cap_side && cudaStreamCreateWithFlags(&ctx->cap_side, cudaStreamNonBlocking) != cudaSuccess)
    ctx->cap_side = nullptr;
  if (!ctx->cap_fork && cudaEventCreateWithFlags(&ctx->cap_fork, cudaEventDisableTiming) != cudaSuccess)
    ctx->cap_fork = nullptr;
  if (!ctx->cap_join && cudaEventCreateWithFlags(&ctx->cap_join, cudaEventDisableTiming) != cudaSuccess)
    ctx->cap_join = nullptr;
  cudaGetLastError();  // a failed creation is not sticky
  return ctx->cap_side && ctx->cap_fork && ctx->cap_join;
}

void destroy_bounce_graphs(tpt_context* ctx) {
  for (BounceGraphSet* g : ctx->graphs) {
    for (auto& row : g->exec)
      for (cudaGraphExec_t x : row)
        if (x) cudaGraphExecDestroy(x);
    delete g;
  }
  ctx->graphs.clear();
  if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  ctx->cap_stream = nullptr;
  if (ctx->cap_side) cudaStreamDestroy(ctx->cap_side);
  ctx->cap_side = nullptr;
  if (ctx->cap_fork) cudaEventDestroy(ctx->cap_fork);
  if (ctx->cap_join) cudaEventDestroy(ctx->cap_join);
  ctx->cap_fork = ctx->cap_join = nullptr;
}

cudaError_t enqueue_bounce(tpt_context* ctx, cudaStream_t s, const DevGeometry& geo, const DevRenderData& rd,
                           const RenderLaunch& P, const WfBuffers& B, const DevJob* jobs, int cur, bool prev_shadow,
                           bool batch_lights) {
  BounceKey key;
  std::memset(&key, 0, sizeof key);
  if (!jobs) {
    std::memcpy(&key.S.geo, &geo, sizeof geo);
    std::memcpy(&key.S.d, &rd, sizeof rd);
    std::memcpy(&key.P, &P, sizeof P);
  }
  std::memcpy(&key.B, &B, sizeof B);
  key.jobs = jobs;
  key.err = ctx->d_err;
  key.num_sms = ctx->num_sms;
  key.shade_block = (int)ctx->shade_block;
  key.batch_lights = jobs && batch_lights ? 1 : 0;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  const bool capturing = cudaStreamIsCapturing(s, &cap) == cudaSuccess && cap != cudaStreamCaptureStatusNone;
  if (!ctx->use_graphs || capturing) return step_ops(key, cur, prev_shadow, next_counter(ctx), next_counter(ctx), s);
  BounceGraphSet* g = nullptr;
  for (BounceGraphSet* x : ctx->graphs)
    if (std::memcmp(&x->key, &key, sizeof key) == 0) g = x;
  if (!g) {
    uint32_t slot = (uint32_t)ctx->graphs.size();
    if (ctx->graphs.size() >= kMaxGraphSets) {  // evict the least recently used set
      size_t lru = 0;
      for (size_t i = 1; i < ctx->graphs.size(); ++i)
        if (ctx->graphs[i]->last_use < ctx->graphs[lru]->last_use) lru = i;
      BounceGraphSet* old = ctx->graphs[lru];
      slot = old->slot;
      for (auto& row : old->exec)
        for (cudaGraphExec_t x : row)
          if (x) cudaGraphExecDestroy(x);  // an in-flight launch completes first
      delete old;
      ctx->graphs.erase(ctx->graphs.begin() + lru);
    }
    g = new BounceGraphSet();
    g->key = key;
    g->slot = slot;
    ctx->graphs.push_back(g);
  }
  g->last_use = ++ctx->graph_clock;
  unsigned long long* c0 = ctx->d_counters + kCounterSlots - 2 * kMaxGraphSets + 2 * g->slot;
  if (g->failed) return step_ops(key, cur, prev_shadow, c0, c0 + 1, s);
  cudaGraphExec_t& x = g->exec[cur][prev_shadow ? 1 : 0];
  if (!x) {
    if (!ctx->cap_stream && cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
      ctx->cap_stream = nullptr;
      g->failed = true;
      cudaGetLastError();
      return step_ops(key, cur, prev_shadow, c0, c0 + 1, s);
    }
    // the shadow branch's stream and events (without them the step is captured in sequence)
    const bool branches = ensure_branch(ctx);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const cudaError_t e_ops = step_ops(key, cur, prev_shadow, c0, c0 + 1, ctx->cap_stream,
                                         branches ? ctx->cap_side : nullptr, ctx->cap_fork, ctx->cap_join);
      e = cudaStreamEndCapture(ctx->cap_stream, &graph);
      if (e == cudaSuccess) e = e_ops;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&x, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      x = nullptr;
      g->failed = true;
      cudaGetLastError();  // capture errors are not sticky; fall back to plain launches
      return step_ops(key, cur, prev_shadow, c0, c0 + 1, s);
    }
  }
  return cudaGraphLaunch(x, s);
}

}  // namespace tpt
