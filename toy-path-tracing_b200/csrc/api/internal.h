// Host-side objects behind the opaque C handles.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "../../../include/tpt.h"
#include "../device/batch_types.h"
#include "../device/dev_types.cuh"
#include "../device/render_types.h"
#include "../host/host_scene.h"
#include "../host/host_types.h"

namespace tpt {

// Path slots of a wavefront chunk when the context sets none (about 4 GB of
// queues; chunks of 2^24 paths keep more of the late, short bounces busy than
// 2^22: 13 % more MIS samples per second on the 2.1M-triangle scene).
constexpr uint32_t kDefaultWavefrontSlots = 1u << 24;
struct BounceGraphSet;
}

struct tpt_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t* d_err = nullptr;  // device error word
  int num_sms = 0;
  std::string last_error;
  // *_device entry points that queued work since the device error word was
  // last read (tpt_context_check, or a host-buffer call that synchronises)
  std::vector<std::string> unchecked_calls;
  // pinned staging for the host-pointer entry points
  void* h_stage = nullptr;
  size_t h_stage_bytes = 0;
  void* d_stage = nullptr;
  size_t d_stage_bytes = 0;
  cudaStream_t pipe[2] = {nullptr, nullptr};  // copy/compute pipeline of tpt_traverse
  cudaEvent_t ev_slot[2] = {nullptr, nullptr};
  cudaEvent_t ev_start = nullptr;
  // pinned-buffer pipeline of tpt_traverse: one stream per copy direction
  // (each feeds its own copy engine) and per-chunk events
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  std::vector<cudaEvent_t> ev_in, ev_done;
  unsigned long long* d_counters = nullptr;  // work-distribution counters, one per in-flight launch
  uint32_t counter_next = 0;
  // device scratch for per-sample radiance of render calls (grown on demand)
  void* d_scratch = nullptr;
  size_t d_scratch_bytes = 0;
  // wavefront arena (grown on demand) and its layout
  void* d_wf = nullptr;
  size_t d_wf_bytes = 0;
  tpt::WfBuffers wf{};
  // BDPT wavefront arena (grown on demand) and its layout
  void* d_bd = nullptr;
  size_t d_bd_bytes = 0;
  tpt::BdWfBuffers bd{};
  // batched renders: device job table (grown on demand) and the wavefront
  // capacity (path slots per chunk; 0 = kDefaultWavefrontSlots)
  tpt::DevJob* d_jobs = nullptr;
  size_t d_jobs_cap = 0;
  uint32_t batch_capacity = 0;
  // per-bounce CUDA graphs of the wavefront (bounce_graphs.cpp)
  bool use_graphs = true;
  uint32_t tuned_execution = 0;  // what TPT_EXEC_AUTO means (tpt_autotune)
  bool batch_per_job = false;    // tpt_render_batch_device renders job by job (tpt_autotune)
  uint32_t shade_block = 256;    // threads per block of the wavefront shade stage (128 or 256)
  // tpt_context_set_render_stats: device counters the wavefront traversals add
  // to (queue rays at [0..3], shadow/visibility rays at [4..7]); NULL = off
  unsigned long long* render_stats = nullptr;
  bool gpu_build = false;        // scene upload builds missing QBVHs on the GPU (tpt_context_set_gpu_build)
  // stream-ordered pool of the GPU QBVH build: keeps up to 1 GiB mapped between
  // builds (the default pool unmaps every freed block at the next synchronisation)
  cudaMemPool_t build_pool = nullptr;
  std::vector<tpt::BounceGraphSet*> graphs;
  uint64_t graph_clock = 0;
  cudaStream_t cap_stream = nullptr;
  // second stream and fork/join events of two-branch launch sequences
  // (created on first use by ensure_branch): the shadow stage of a bounce
  // beside the next bounce's traversal in the captured bounce graphs, and the
  // light half of the BDPT subpath queue beside its camera half
  cudaStream_t cap_side = nullptr;
  cudaEvent_t cap_fork = nullptr, cap_join = nullptr;
  // OpenPBR tables (built on the GPU on first use, kept until destroy)
  std::map<uint32_t, float*> da_tables;  // directional albedo per eta (bit pattern)
  float* d_cec_e = nullptr;              // conductor E (64 x 64)
  float* d_dec_e = nullptr;              // dielectric E (32 x 32 x 32)
  std::vector<float> h_cec_e, h_cec_e_avg, h_dec_e, h_dec_e_avg;
};

struct tpt_qbvh {
  tpt::QbvhHost q;
};

struct tpt_scene {
  tpt_context* ctx = nullptr;
  tpt::DevGeometry geo{};
  std::vector<void*> allocations;
  uint64_t device_bytes = 0;
  uint32_t num_meshes = 0;
  uint32_t num_instances = 0;
  std::vector<uint32_t> mesh_tri_counts;
  tpt::DevRenderData render{};          // shading data for the render kernels
  tpt::LightTreeHost light_tree;        // host copy of the light tree
  std::vector<uint32_t> material_kinds; // tpt_material_kind per material
  uint32_t num_point_lights = 0, num_spot_lights = 0, num_directional_lights = 0;
  // OpenPBR materials: host copy of each table entry's parameters and the
  // material -> table index map (0xFFFFFFFF: not OpenPBR)
  std::vector<tpt_openpbr_desc> opbr_desc;
  std::vector<uint32_t> opbr_of_material;
  uint32_t mat_version = 0;  // bumped by tpt_scene_set_openpbr
  // adjoint perturbation tables (lowered on demand, owned by the scene)
  void* d_adj = nullptr;
  size_t d_adj_bytes = 0;
  uint32_t adj_version = 0xFFFFFFFFu, adj_mask = 0;
  float adj_step = 0.0f;
};

namespace tpt {

constexpr uint32_t kCounterSlots = 1024;
constexpr uint32_t kGraphCounterSlots = 32;  // the last slots: two per cached bounce-graph set

tpt_status set_error(tpt_context* ctx, tpt_status st, const std::string& msg);
tpt_status cuda_check(tpt_context* ctx, cudaError_t e, const char* what);
// Reads and clears the device error word (synchronising `stream`); an error
// names the *_device calls whose work ran since the last read.
tpt_status check_device_errors(tpt_context* ctx, cudaStream_t stream);
// Records that entry point `name` queued device work whose checks are read later.
void note_device_call(tpt_context* ctx, const char* name);
// cudaSetDevice(ctx->device) with its status checked.
tpt_status set_device(tpt_context* ctx);

// kernels (traverse_kernels.cu).  Ray plane p of ray i at rays[p * rs + i];
// barycentric output plane p at bary[p * bs + i].  `counter` is a device word
// the launch resets and uses for its work distribution (one per concurrent launch).
cudaError_t launch_traverse_strided(const DevGeometry& geo, const float* rays, uint64_t rs, uint64_t n, int mode,
                                    int32_t* prim, float* t, int32_t* inst, float* bary, uint64_t bs,
                                    unsigned long long* counter, uint32_t* err, int num_sms, cudaStream_t stream,
                                    uint32_t* node_tests, uint32_t* tri_tests, const uint32_t* n_dev = nullptr,
                                    const DevJob* jobs = nullptr, const uint32_t* ray_job = nullptr,
                                    unsigned long long* totals = nullptr, uint32_t* aux = nullptr,
                                    const uint32_t* aux_index = nullptr);
// aux: per-ray AuxRng states for the alpha tests (NULL: no alpha tests), read
// at aux[aux_index ? aux_index[i] : i] and advanced in place by the draws.

// qbvh_build_gpu.cu: the QBVH of n primitive boxes (device, n x 6 floats) built
// on the device, equal to build_qbvh_host's (a box face at zero may be +0.0
// where the host keeps -0.0).  Errors: allocation, or capacity (never expected;
// callers fall back to the host builder).
// Scratch comes from `pool` (NULL: the device's default pool).
cudaError_t build_qbvh_gpu(const float* d_bounds6, uint32_t n, QbvhHost* out, cudaStream_t s,
                           cudaMemPool_t pool = nullptr);
// The context's build pool, created on first use (NULL if that fails: the
// default pool then serves the build).
cudaMemPool_t build_pool(tpt_context* ctx);
// The QBVH of host boxes: on the GPU when the context asks for it and the set is
// large enough to gain, else (or if the GPU build fails) on the host.
void build_qbvh_for(tpt_context* ctx, const float* bounds6, uint32_t n, int threads, QbvhHost* out);

// A work counter slot for the next launch (ring of kCounterSlots per context).
unsigned long long* next_counter(tpt_context* ctx);

// render_kernels.cu
// `counter`: a work-distribution word (next_counter) the launch resets.
cudaError_t launch_render(const DevGeometry& geo, const DevRenderData& rd, const RenderLaunch& P, float* samples,
                          uint64_t first_path, uint64_t n_paths, uint32_t* err, int num_sms, cudaStream_t stream,
                          unsigned long long* counter);
cudaError_t launch_accumulate(const float* samples, uint32_t spp, uint32_t first_pixel, uint32_t n_pixels,
                              float exposure, float* image, cudaStream_t stream);
// bdpt_wavefront.cu: n samples (paths first_path..) of a BDPT job through the
// wavefront stages (n <= B.sample_capacity); per-sample radiance into samples.
cudaError_t launch_bdpt_wavefront(const DevGeometry& geo, const DevRenderData& rd, const RenderLaunch& P,
                                  const BdWfBuffers& B, uint64_t first_path, uint32_t n, float* samples,
                                  unsigned long long* counter, uint32_t* err, int num_sms, cudaStream_t s,
                                  unsigned long long* totals = nullptr, unsigned long long* counter2 = nullptr,
                                  cudaStream_t side = nullptr, cudaEvent_t fork = nullptr,
                                  cudaEvent_t join = nullptr);
// With `side` (and its own work counter2) the light half of each subpath step's
// traversal runs on `side` beside the camera half (fork/join events around it).

// capi_render.cpp: BDPT paths [first, first + n) through the wavefront, in chunks.
tpt_status render_bdpt_wavefront(tpt_context* ctx, const tpt_render_job* job, const RenderLaunch& L, uint64_t first,
                                 uint64_t n, float* samples, cudaStream_t s);
// bdpt_kernels.cu (launch_render dispatches to it for TPT_INTEGRATOR_BDPT)
cudaError_t launch_render_bdpt(const DevGeometry& geo, const DevRenderData& rd, const RenderLaunch& P, float* samples,
                               uint64_t first_path, uint64_t n_paths, uint32_t* err, int num_sms, cudaStream_t stream);

// capi_render.cpp: validates a job and derives its launch parameters.
tpt_status render_launch_params(tpt_context* ctx, const tpt_render_job* job, RenderLaunch* out);
// The wavefront arena with its alpha-test planes, or without them (NULL).
WfBuffers wavefront_view(const WfBuffers& B, bool alpha);
// The context's per-sample scratch (grown on demand) and wavefront arena.
tpt_status ensure_scratch(tpt_context* ctx, size_t bytes);
tpt_status ensure_wavefront(tpt_context* ctx, uint32_t capacity);
// Pixels per chunk of a job: at most `capacity` paths (0 = kDefaultWavefrontSlots) and 1 GiB of samples.
uint32_t chunk_pixels(const RenderLaunch& L, uint32_t capacity);
// Paths [first, first + n) through the wavefront stages (forward: radiance into
// samples; with A: the adjoint replay of samples' paths, gradients to A->grad).
tpt_status render_wavefront(tpt_context* ctx, const tpt_render_job* job, const RenderLaunch& L, uint64_t first,
                            uint32_t n, float* samples, cudaStream_t s, const DevAdjoint* A = nullptr);

// wavefront_kernels.cu
// primal != NULL / A != NULL / adjoint: the adjoint instantiation (path replay
// with R; primal = per-sample radiance of the forward pass, path order).
cudaError_t launch_wf_generate(const DevGeometry& geo, const DevRenderData& rd, const RenderLaunch& P,
                               const WfBuffers& B, uint64_t first_path, uint32_t n_paths, cudaStream_t s,
                               const float* primal = nullptr);
// shade reads the chunk's first path from the queue counters (written by generate)
// `block`: threads per block of the (forward) shade stage, 128 or 256 (tpt_autotune picks it)
cudaError_t launch_wf_shade(const DevGeometry& geo, const DevRenderData& rd, const RenderLaunch& P,
                            const WfBuffers& B, int cur, cudaStream_t s, const DevAdjoint* A = nullptr,
                            int block = 256);
cudaError_t launch_wf_resolve(const WfBuffers& B, cudaStream_t s, const DevAdjoint* A = nullptr);
// Batched stages: slot i is global path first_path + i of the jobs' index space.
cudaError_t launch_wf_generate_batch(const DevJob* jobs, uint32_t n_jobs, const WfBuffers& B, uint64_t first_path,
                                     uint32_t n_paths, cudaStream_t s);
cudaError_t launch_wf_shade_batch(const DevJob* jobs, const WfBuffers& B, int cur, cudaStream_t s, int block,
                                  bool lights);
cudaError_t launch_wf_finalize(const WfBuffers& B, uint32_t n_paths, float* samples, cudaStream_t s);

// bounce_graphs.cpp: step b of the wavefront loop b = 0 .. max_depth (single
// job when jobs == nullptr, else batched) on `s`, replayed from a cached CUDA
// graph when possible: the shadow stage of bounce b - 1 when prev_shadow
// (b > 0), then bounce b's closest-hit traversal and shade.  The last bounce's
// shadow rays are never traced, as in the sequential order.
// batch_lights: some job of the batch `jobs` has point, spot or directional lights
cudaError_t enqueue_bounce(tpt_context* ctx, cudaStream_t s, const DevGeometry& geo, const DevRenderData& rd,
                           const RenderLaunch& P, const WfBuffers& B, const DevJob* jobs, int cur, bool prev_shadow,
                           bool batch_lights = false);
void destroy_bounce_graphs(tpt_context* ctx);
// Creates ctx->cap_side / cap_fork / cap_join when missing; false when they
// cannot be created (the caller then launches its branches in sequence).
bool ensure_branch(tpt_context* ctx);

// capi_batch.cpp: jobs (MIS) through one wavefront launch sequence; out_rgb are
// device images; capacity = path slots per chunk (0 = kDefaultWavefrontSlots).
tpt_status render_batch(tpt_context* ctx, const tpt_render_job* jobs, int n_jobs, float* const* out_rgb,
                        cudaStream_t s, uint32_t capacity);

// capi_openpbr.cpp: the context's OpenPBR tables, built on first use.
tpt_status ensure_ec_tables(tpt_context* ctx);
tpt_status ensure_da_table(tpt_context* ctx, float eta, const float** out);

// lut_kernels.cu: table construction (bit-exact with the reference's loops;
// the sample tables come from lut_sample_tables).
cudaError_t launch_lut_dielectric_albedo(float eta, const float* dirs, const float* phi_cs, float* out,
                                         cudaStream_t s);
cudaError_t launch_lut_conductor_e(const float* u, const float* cs, float* e, cudaStream_t s);
cudaError_t launch_lut_dielectric_e(const float* uc, const float* ux, const float* cs, float* e, cudaStream_t s);
// openpbr_query.cu: batched BSDF queries of one material; `state` (n x 4:
// path throughput, wavelength lock or NaN) may be NULL (the defaults), and
// with it u has 7 values per sample (with u_extra0..3) and out 10 (with the lock).
cudaError_t launch_bsdf_eval(const DevRenderData& rd, uint32_t material, uint64_t n, const float* wo, const float* wi,
                             const uint32_t* front, uint32_t mode, const float* state, float* f, float* pdf,
                             cudaStream_t s);
cudaError_t launch_bsdf_sample(const DevRenderData& rd, uint32_t material, uint64_t n, const float* wo,
                               const float* u, const uint32_t* front, uint32_t mode, const float* state, float* out,
                               cudaStream_t s);

// scene_render_upload.cpp: materials, shading arrays, light tree, emitter map.
tpt_status upload_render_data(tpt_scene* s, const tpt_scene_desc* desc);
// One OpenPBR material lowered for the device (make_bsdf's material part),
// building the tables it reads on first use.
tpt_status lower_openpbr_material(tpt_context* ctx, const tpt_openpbr_desc& d, DevOpenPbr* out);
// Device allocation owned by the scene.
tpt_status scene_alloc(tpt_scene* s, size_t bytes, void** out);

}  // namespace tpt
