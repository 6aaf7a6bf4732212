// tpt_render_device_noalloc: the megakernel render of tpt_render_device with
// its per-sample scratch in a fixed device array instead of memory it would
// have to allocate.
//
// Who needs it: code that must not call cudaMalloc at the time it renders —
// work recorded inside a CUDA stream capture (an allocation there breaks or
// invalidates the capture), hosts whose device memory is owned by another
// allocator with a fixed budget (a framework's caching pool that has already
// reserved the card), and latency-critical loops that must never enter the
// driver's allocator.  Such callers still pass their own input (the uploaded
// scene) and output (the image buffer); this call itself allocates nothing.
//
// The scratch is `g_noalloc_samples`: 3 floats per path for at most
// kNoAllocMaxPaths = 2^20 paths (12 MiB), resident on every device that loads
// the library until the process exits, and `g_noalloc_counter`, the persistent
// kernel's work counter (its own word: the context's ring of counters serves
// every other launch, and a slot of that ring could be handed to a concurrent
// launch while a graph captured from this call still uses it).  Every call on
// a device shares both and they keep the last call's contents; each call
// resets the counter (a stream-ordered memset, not an allocation) and writes
// every sample it later reads.  Two calls whose work overlaps on the GPU
// (different streams, or different threads without ordering) race on them.
#include <mutex>

#include "../api/internal.h"

namespace tpt {

constexpr uint64_t kNoAllocMaxPaths = 1ull << 20;

static __device__ __align__(256) float g_noalloc_samples[3 * kNoAllocMaxPaths];
static __device__ __align__(256) unsigned long long g_noalloc_counter;

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
float* g_scratch[kMaxDevices] = {};
unsigned long long* g_counter[kMaxDevices] = {};

// Device addresses of the scratch and the counter on `device` (which must be
// current).  Done once per device, on the first call there: in host code the
// arrays' names are only host-side stand-ins, never device addresses.
tpt_status scratch_for(tpt_context* ctx, int device, float** out, unsigned long long** counter) {
  if (device < 0 || device >= kMaxDevices) return set_error(ctx, TPT_ERR_INVALID_ARG, "device index out of range");
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_scratch[device]) {
    void *p = nullptr, *c = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_samples);
    if (e != cudaSuccess || !p) return cuda_check(ctx, e == cudaSuccess ? cudaErrorInvalidSymbol : e,
                                                  "cudaGetSymbolAddress(no-alloc render scratch)");
    e = cudaGetSymbolAddress(&c, g_noalloc_counter);
    if (e != cudaSuccess || !c) return cuda_check(ctx, e == cudaSuccess ? cudaErrorInvalidSymbol : e,
                                                  "cudaGetSymbolAddress(no-alloc render counter)");
    g_counter[device] = (unsigned long long*)c;
    g_scratch[device] = (float*)p;
  }
  *out = g_scratch[device];
  *counter = g_counter[device];
  return TPT_OK;
}
}  // namespace

}  // namespace tpt

using namespace tpt;

extern "C" tpt_status tpt_render_device_noalloc(tpt_context* ctx, const tpt_render_job* job, float* out_rgb,
                                                void* stream) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  if (!out_rgb) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL output");
  RenderLaunch L;
  tpt_status st = render_launch_params(ctx, job, &L);
  if (st) return st;
  const uint64_t n_paths = (uint64_t)L.width * L.height * L.spp;
  if (n_paths > kNoAllocMaxPaths)
    return set_error(ctx, TPT_ERR_CAPACITY,
                     "tpt_render_device_noalloc: width * height * spp = " + std::to_string(n_paths) +
                         " paths exceeds its fixed scratch of " + std::to_string(kNoAllocMaxPaths) +
                         " paths; use tpt_render_device or split the image");
  if ((st = set_device(ctx))) return st;
  float* scratch = nullptr;
  unsigned long long* counter = nullptr;
  if ((st = scratch_for(ctx, ctx->device, &scratch, &counter))) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  note_device_call(ctx, "tpt_render_device_noalloc");
  cudaError_t e = launch_render(job->scene->geo, job->scene->render, L, scratch, 0, n_paths, ctx->d_err,
                                ctx->num_sms, s, counter);
  if ((st = cuda_check(ctx, e, "render kernel launch"))) return st;
  e = launch_accumulate(scratch, L.spp, 0, L.width * L.height, L.cam.exposure, out_rgb, s);
  return cuda_check(ctx, e, "accumulate kernel launch");
}
