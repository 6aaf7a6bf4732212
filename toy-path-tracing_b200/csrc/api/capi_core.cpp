// C ABI: context, host QBVH builder, scene upload and ray queries.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "internal.h"

namespace {
std::mutex g_err_mu;
std::string g_global_error;
}  // namespace

namespace tpt {

tpt_status set_error(tpt_context* ctx, tpt_status st, const std::string& msg) {
  if (ctx) {
    ctx->last_error = msg;
  } else {
    std::lock_guard<std::mutex> g(g_err_mu);
    g_global_error = msg;
  }
  return st;
}

tpt_status cuda_check(tpt_context* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return TPT_OK;
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  if (e == cudaErrorMemoryAllocation) return set_error(ctx, TPT_ERR_OUT_OF_MEMORY, m);
  return set_error(ctx, TPT_ERR_CUDA, m);
}

void note_device_call(tpt_context* ctx, const char* name) {
  auto& v = ctx->unchecked_calls;
  for (const std::string& n : v)
    if (n == name) return;
  if (v.size() < 16) v.emplace_back(name);
}

tpt_status set_device(tpt_context* ctx) { return cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice"); }

tpt_status check_device_errors(tpt_context* ctx, cudaStream_t stream) {
  uint32_t h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, ctx->d_err, 4, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "reading device error word");
  std::string who;
  for (const std::string& n : ctx->unchecked_calls) who += (who.empty() ? "" : ", ") + n;
  ctx->unchecked_calls.clear();
  if (h == 0) return TPT_OK;
  cudaMemsetAsync(ctx->d_err, 0, 4, stream);
  cudaStreamSynchronize(stream);
  const std::string from = who.empty() ? std::string() : " (in work queued by " + who + ")";
  if (h & kDevErrTimeout) return set_error(ctx, TPT_ERR_TIMEOUT, "device-side bounded wait expired" + from);
  if (h & kDevErrCapacity) return set_error(ctx, TPT_ERR_CAPACITY, "device queue capacity exceeded" + from);
  if (h & kDevErrStackOverflow)
    return set_error(ctx, TPT_ERR_DEVICE_CHECK,
                     "traversal stack depth 128 exceeded (reference limit, qbvh.rs:609)" + from);
  return set_error(ctx, TPT_ERR_DEVICE_CHECK, "device index check failed (flags " + std::to_string(h) + ")" + from);
}

unsigned long long* next_counter(tpt_context* ctx) {
  uint32_t k = ctx->counter_next++ % (kCounterSlots - kGraphCounterSlots);
  return ctx->d_counters + k;
}

}  // namespace tpt

using namespace tpt;

namespace {

int host_threads(int requested) {
  if (requested > 0) return requested;
  unsigned hc = std::thread::hardware_concurrency();
  return hc ? (int)hc : 1;
}

tpt_status ensure_host_staging(tpt_context* ctx, size_t bytes) {
  if (ctx->h_stage_bytes >= bytes) return TPT_OK;
  if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
  ctx->h_stage = nullptr;
  ctx->h_stage_bytes = 0;
  tpt_status st = cuda_check(ctx, cudaMallocHost(&ctx->h_stage, bytes), "cudaMallocHost(staging)");
  if (st) return st;
  ctx->h_stage_bytes = bytes;
  return TPT_OK;
}

tpt_status ensure_device_staging(tpt_context* ctx, size_t bytes) {
  if (ctx->d_stage_bytes >= bytes) return TPT_OK;
  if (ctx->d_stage) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_stage);
  }
  ctx->d_stage = nullptr;
  ctx->d_stage_bytes = 0;
  tpt_status st = cuda_check(ctx, cudaMalloc(&ctx->d_stage, bytes), "cudaMalloc(staging)");
  if (st) return st;
  ctx->d_stage_bytes = bytes;
  return TPT_OK;
}

tpt_status ensure_pipeline(tpt_context* ctx) {
  if (ctx->pipe[0]) return TPT_OK;
  for (int k = 0; k < 2; ++k) {
    tpt_status st = cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->pipe[k], cudaStreamNonBlocking), "stream");
    if (st) return st;
    st = cuda_check(ctx, cudaEventCreateWithFlags(&ctx->ev_slot[k], cudaEventDisableTiming), "event");
    if (st) return st;
  }
  return cuda_check(ctx, cudaEventCreateWithFlags(&ctx->ev_start, cudaEventDisableTiming), "event");
}

// Chunk sizes of a pinned-buffer traversal: a ramp up from chunk / 8 (the
// first kernel starts after a short copy), `chunk` in the middle, and halving
// pieces at the end (the last copy-out follows a short kernel).
std::vector<uint64_t> chunk_schedule(uint64_t n, uint64_t chunk) {
  std::vector<uint64_t> out;
  const uint64_t min_chunk = 1u << 16;
  uint64_t left = n, s = std::max<uint64_t>(min_chunk, chunk / 8);
  while (left > 0 && s < chunk) {
    const uint64_t m = std::min(s, left);
    out.push_back(m);
    left -= m;
    s *= 2;
  }
  while (left > 0) {
    uint64_t m;
    if (left > 2 * chunk) m = chunk;
    else if (left > 2 * min_chunk) m = std::max<uint64_t>(min_chunk, (left + 1) / 2);
    else m = left;
    out.push_back(m);
    left -= m;
  }
  return out;
}

tpt_status ensure_copy_pipeline(tpt_context* ctx, size_t n_chunks) {
  tpt_status st = TPT_OK;
  if (!ctx->copy_in) st = cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking), "stream");
  if (!st && !ctx->copy_out)
    st = cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking), "stream");
  while (!st && ctx->ev_in.size() < n_chunks) {
    cudaEvent_t a = nullptr, b = nullptr;
    st = cuda_check(ctx, cudaEventCreateWithFlags(&a, cudaEventDisableTiming), "event");
    if (!st) st = cuda_check(ctx, cudaEventCreateWithFlags(&b, cudaEventDisableTiming), "event");
    if (a) ctx->ev_in.push_back(a);
    if (b) ctx->ev_done.push_back(b);
  }
  return st;
}

bool is_pinned(const void* p);

}  // namespace

cudaMemPool_t tpt::build_pool(tpt_context* ctx) {
  if (ctx->build_pool) return ctx->build_pool;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = ctx->device;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  uint64_t keep = 1ull << 30;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  ctx->build_pool = pool;
  return pool;
}

void tpt::build_qbvh_for(tpt_context* ctx, const float* bounds6, uint32_t n, int threads, QbvhHost* out) {
  constexpr uint32_t kGpuBuildMin = 4096;  // below this the host builds faster than a launch sequence
  if (ctx && ctx->gpu_build && n >= kGpuBuildMin) {
    float* d = nullptr;
    cudaMemPool_t pool = build_pool(ctx);
    const size_t bytes = (size_t)6 * n * 4;
    cudaError_t e = pool ? cudaMallocFromPoolAsync((void**)&d, bytes, pool, ctx->stream)
                         : cudaMallocAsync((void**)&d, bytes, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d, bounds6, (size_t)6 * n * 4, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = build_qbvh_gpu(d, n, out, ctx->stream, pool);
    if (d) cudaFreeAsync(d, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) return;
    cudaGetLastError();
  }
  build_qbvh_host(bounds6, n, threads, out);
}

namespace {

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

template <class T>
tpt_status dev_upload(tpt_scene* s, const T* src, size_t count, const T** dst) {
  size_t bytes = std::max<size_t>(count * sizeof(T), 128);
  void* p = nullptr;
  tpt_status st = cuda_check(s->ctx, cudaMalloc(&p, bytes), "cudaMalloc(scene)");
  if (st) return st;
  s->allocations.push_back(p);
  s->device_bytes += bytes;
  if (count) {
    st = cuda_check(s->ctx, cudaMemcpy(p, src, count * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy(scene)");
    if (st) return st;
  }
  *dst = (const T*)p;
  return TPT_OK;
}

// Validates a QBVH against the primitive count so that no device access can
// leave its arrays; returns false with a reason.
bool validate_qbvh(const QbvhNodeHost* nodes, uint64_t num_nodes, const uint32_t* prims, uint64_t num_prims,
                   uint64_t prim_limit, std::string* why) {
  if (num_prims == 0) { *why = "empty primitive index list"; return false; }
  for (uint64_t i = 0; i < num_prims; ++i)
    if (prims[i] >= prim_limit) { *why = "primitive index out of range"; return false; }
  for (uint64_t i = 0; i < num_nodes; ++i)
    for (int s = 0; s < 4; ++s) {
      uint32_t w = nodes[i].children[s];
      if ((w >> 24) == 0x80u) continue;  // empty lane
      if (w & kLeafFlag) {
        uint64_t off = w & 0xFFFFFFu, cnt = (w >> 24) & 0x7Fu;
        if (off + cnt > num_prims) { *why = "leaf range out of range"; return false; }
      } else if (w >= num_nodes || w <= i) {
        *why = "interior child index out of range";
        return false;
      }
    }
  if (num_nodes == 0 && num_prims > 127) { *why = "root leaf with more than 127 primitives"; return false; }
  return true;
}

// Reference-layout node -> device node (empty lanes get the empty word).
DevNode to_dev(const QbvhNodeHost& h) {
  DevNode d;
  auto f4 = [&](int k) { return make_float4(h.b[k][0], h.b[k][1], h.b[k][2], h.b[k][3]); };
  d.lo_x = f4(0); d.lo_y = f4(1); d.lo_z = f4(2);
  d.hi_x = f4(3); d.hi_y = f4(4); d.hi_z = f4(5);
  uint32_t c[4];
  for (int s = 0; s < 4; ++s) c[s] = ((h.valid_mask >> s) & 1u) ? h.children[s] : kEmptyWord;
  d.child = make_uint4(c[0], c[1], c[2], c[3]);
  d.pad = make_uint4(0, 0, 0, 0);
  return d;
}

struct Vec3f {
  float x, y, z;
};

// glam Mat4::transform_point3 (column-major m[16]).
Vec3f xform_point(const float* m, Vec3f p) {
  float r[3];
  for (int i = 0; i < 3; ++i) r[i] = m[0 + i] * p.x;
  for (int i = 0; i < 3; ++i) r[i] = m[4 + i] * p.y + r[i];
  for (int i = 0; i < 3; ++i) r[i] = m[8 + i] * p.z + r[i];
  for (int i = 0; i < 3; ++i) r[i] = m[12 + i] + r[i];
  return Vec3f{r[0], r[1], r[2]};
}

}  // namespace

extern "C" {

const char* tpt_version(void) { return "tpt-b200 0.1 (sm_100a)"; }

const char* tpt_last_error(const tpt_context* ctx) {
  if (ctx) return ctx->last_error.c_str();
  std::lock_guard<std::mutex> g(g_err_mu);
  return g_global_error.c_str();
}

tpt_status tpt_context_create(int device, tpt_context** out) {
  if (!out) return set_error(nullptr, TPT_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return set_error(nullptr, TPT_ERR_CUDA, "no CUDA device available");
  if (device < 0 || device >= n) return set_error(nullptr, TPT_ERR_INVALID_ARG, "device index out of range");
  auto* ctx = new tpt_context();
  ctx->device = device;
  if ((e = cudaSetDevice(device)) != cudaSuccess) { delete ctx; return cuda_check(nullptr, e, "cudaSetDevice"); }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  if (prop.major < 10) {
    delete ctx;
    return set_error(nullptr, TPT_ERR_CUDA, "device is not sm_100 class (B200); this build targets sm_100a only");
  }
  ctx->num_sms = prop.multiProcessorCount;
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    delete ctx;
    return cuda_check(nullptr, e, "cudaStreamCreate");
  }
  if ((e = cudaMalloc(&ctx->d_err, 256)) != cudaSuccess) {
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return cuda_check(nullptr, e, "cudaMalloc(error word)");
  }
  cudaMemset(ctx->d_err, 0, 256);
  if ((e = cudaMalloc(&ctx->d_counters, kCounterSlots * sizeof(unsigned long long))) != cudaSuccess) {
    cudaFree(ctx->d_err);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return cuda_check(nullptr, e, "cudaMalloc(counters)");
  }
  *out = ctx;
  return TPT_OK;
}

tpt_status tpt_context_destroy(tpt_context* ctx) {
  if (!ctx) return TPT_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
  if (ctx->d_stage) cudaFree(ctx->d_stage);
  if (ctx->d_err) cudaFree(ctx->d_err);
  destroy_bounce_graphs(ctx);
  if (ctx->d_counters) cudaFree(ctx->d_counters);
  if (ctx->d_scratch) cudaFree(ctx->d_scratch);
  if (ctx->d_wf) cudaFree(ctx->d_wf);
  if (ctx->d_jobs) cudaFree(ctx->d_jobs);
  if (ctx->d_bd) cudaFree(ctx->d_bd);
  for (auto& kv : ctx->da_tables) cudaFree(kv.second);
  if (ctx->d_cec_e) cudaFree(ctx->d_cec_e);
  if (ctx->d_dec_e) cudaFree(ctx->d_dec_e);
  for (int k = 0; k < 2; ++k) {
    if (ctx->pipe[k]) cudaStreamDestroy(ctx->pipe[k]);
    if (ctx->ev_slot[k]) cudaEventDestroy(ctx->ev_slot[k]);
  }
  if (ctx->build_pool) cudaMemPoolDestroy(ctx->build_pool);
  if (ctx->copy_in) cudaStreamDestroy(ctx->copy_in);
  if (ctx->copy_out) cudaStreamDestroy(ctx->copy_out);
  for (cudaEvent_t e : ctx->ev_in) cudaEventDestroy(e);
  for (cudaEvent_t e : ctx->ev_done) cudaEventDestroy(e);
  if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return TPT_OK;
}

tpt_status tpt_context_check(tpt_context* ctx, void* stream) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  tpt_status st = set_device(ctx);
  if (st) return st;
  return check_device_errors(ctx, stream ? (cudaStream_t)stream : ctx->stream);
}

// ---- host QBVH builder -----------------------------------------------------
tpt_status tpt_qbvh_build(const float* bounds, uint64_t n, int threads, tpt_qbvh** out) {
  if (!out || (!bounds && n)) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  if (n == 0) return set_error(nullptr, TPT_ERR_INVALID_ARG, "no primitives (build_qbvh returns None)");
  if (n >= (1ull << 24)) return set_error(nullptr, TPT_ERR_CAPACITY, "more than 2^24 primitives in one QBVH");
  auto* q = new tpt_qbvh();
  build_qbvh_host(bounds, (uint32_t)n, host_threads(threads), &q->q);
  *out = q;
  return TPT_OK;
}

tpt_status tpt_qbvh_build_device(tpt_context* ctx, const float* d_bounds, uint64_t n, void* stream, tpt_qbvh** out) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  if (!out || (!d_bounds && n)) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  if (n == 0) return set_error(ctx, TPT_ERR_INVALID_ARG, "no primitives (build_qbvh returns None)");
  if (n >= (1ull << 24)) return set_error(ctx, TPT_ERR_CAPACITY, "more than 2^24 primitives in one QBVH");
  if (tpt_status st = set_device(ctx)) return st;
  auto* q = new tpt_qbvh();
  const cudaError_t e =
      build_qbvh_gpu(d_bounds, (uint32_t)n, &q->q, stream ? (cudaStream_t)stream : ctx->stream, build_pool(ctx));
  if (e != cudaSuccess) {
    delete q;
    if (e == cudaErrorLaunchOutOfResources)
      return set_error(ctx, TPT_ERR_CAPACITY, "GPU QBVH build exceeded its work-list capacity");
    return cuda_check(ctx, e, "GPU QBVH build");
  }
  *out = q;
  return TPT_OK;
}

tpt_status tpt_context_set_gpu_build(tpt_context* ctx, int enable) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  ctx->gpu_build = enable != 0;
  return TPT_OK;
}

tpt_status tpt_qbvh_view_of(const tpt_qbvh* q, tpt_qbvh_view* v) {
  if (!q || !v) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL argument");
  v->nodes = reinterpret_cast<const tpt_qbvh_node*>(q->q.nodes.data());
  v->num_nodes = q->q.nodes.size();
  v->primitive_indices = q->q.prim_indices.data();
  v->num_primitives = q->q.prim_indices.size();
  return TPT_OK;
}

tpt_status tpt_qbvh_free(tpt_qbvh* q) {
  delete q;
  return TPT_OK;
}

// ---- scene upload ----------------------------------------------------------
tpt_status tpt_scene_upload(tpt_context* ctx, const tpt_scene_desc* desc, tpt_scene** out) {
  if (!ctx || !desc || !out) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  if (desc->num_meshes && !desc->meshes) return set_error(ctx, TPT_ERR_INVALID_ARG, "meshes is NULL");
  if (desc->num_instances && !desc->instances) return set_error(ctx, TPT_ERR_INVALID_ARG, "instances is NULL");
  if (tpt_status st = set_device(ctx)) return st;
  const int threads = host_threads(0);

  std::vector<DevNode> nodes;
  std::vector<DevTri> tris;
  std::vector<uint32_t> mesh_node_base(desc->num_meshes), mesh_tri_base(desc->num_meshes),
      mesh_root(desc->num_meshes);
  std::vector<uint32_t> tri_counts(desc->num_meshes);
  std::vector<float> mesh_bounds(6 * (size_t)desc->num_meshes);

  for (uint32_t m = 0; m < desc->num_meshes; ++m) {
    const tpt_mesh_desc& md = desc->meshes[m];
    if (!md.positions || !md.indices || md.num_indices % 3 != 0 || md.num_vertices == 0)
      return set_error(ctx, TPT_ERR_INVALID_ARG, "mesh " + std::to_string(m) + ": bad vertex/index arrays");
    const uint64_t ntri = md.num_indices / 3;
    if (ntri == 0) return set_error(ctx, TPT_ERR_INVALID_ARG, "mesh " + std::to_string(m) + " has no triangles");
    if (ntri >= (1ull << 24)) return set_error(ctx, TPT_ERR_CAPACITY, "mesh with more than 2^24 triangles");
    for (uint64_t k = 0; k < md.num_indices; ++k)
      if (md.indices[k] >= md.num_vertices)
        return set_error(ctx, TPT_ERR_INVALID_ARG, "mesh " + std::to_string(m) + ": vertex index out of range");
    const float* P = md.positions;
    auto pos = [&](uint32_t vi) { return Vec3f{P[3 * (size_t)vi], P[3 * (size_t)vi + 1], P[3 * (size_t)vi + 2]}; };
    // mesh bounds (mesh.rs compute_bounds)
    float* mb = &mesh_bounds[6 * (size_t)m];
    mb[0] = mb[1] = mb[2] = INFINITY;
    mb[3] = mb[4] = mb[5] = -INFINITY;
    for (uint64_t v = 0; v < md.num_vertices; ++v)
      for (int k = 0; k < 3; ++k) {
        mb[k] = std::fmin(mb[k], P[3 * v + k]);
        mb[3 + k] = std::fmax(mb[3 + k], P[3 * v + k]);
      }
    // BLAS: caller's, or built here from triangle bounds (mesh.rs:105-119)
    QbvhHost built;
    const QbvhNodeHost* qn;
    uint64_t qnn;
    const uint32_t* qp;
    uint64_t qpn;
    if (md.qbvh.primitive_indices) {
      qn = reinterpret_cast<const QbvhNodeHost*>(md.qbvh.nodes);
      qnn = md.qbvh.num_nodes;
      qp = md.qbvh.primitive_indices;
      qpn = md.qbvh.num_primitives;
      if (qnn && !qn) return set_error(ctx, TPT_ERR_INVALID_ARG, "mesh QBVH nodes is NULL");
    } else {
      std::vector<float> tb(6 * ntri);
      for (uint64_t t = 0; t < ntri; ++t) {
        Vec3f v[3] = {pos(md.indices[3 * t]), pos(md.indices[3 * t + 1]), pos(md.indices[3 * t + 2])};
        float* b = &tb[6 * t];
        b[0] = std::fmin(std::fmin(v[0].x, v[1].x), v[2].x);
        b[1] = std::fmin(std::fmin(v[0].y, v[1].y), v[2].y);
        b[2] = std::fmin(std::fmin(v[0].z, v[1].z), v[2].z);
        b[3] = std::fmax(std::fmax(v[0].x, v[1].x), v[2].x);
        b[4] = std::fmax(std::fmax(v[0].y, v[1].y), v[2].y);
        b[5] = std::fmax(std::fmax(v[0].z, v[1].z), v[2].z);
      }
      build_qbvh_for(ctx, tb.data(), (uint32_t)ntri, threads, &built);
      qn = built.nodes.data();
      qnn = built.nodes.size();
      qp = built.prim_indices.data();
      qpn = built.prim_indices.size();
    }
    std::string why;
    if (qpn != ntri || !validate_qbvh(qn, qnn, qp, qpn, ntri, &why))
      return set_error(ctx, TPT_ERR_INVALID_ARG, "mesh " + std::to_string(m) + " QBVH invalid: " +
                                                     (qpn != ntri ? std::string("primitive count mismatch") : why));
    mesh_node_base[m] = (uint32_t)nodes.size();
    mesh_tri_base[m] = (uint32_t)tris.size();
    mesh_root[m] = qnn ? 0u : (kLeafFlag | ((uint32_t)qpn << 24));
    tri_counts[m] = (uint32_t)ntri;
    for (uint64_t i = 0; i < qnn; ++i) nodes.push_back(to_dev(qn[i]));
    for (uint64_t k = 0; k < qpn; ++k) {
      uint32_t t = qp[k];
      Vec3f a = pos(md.indices[3 * (size_t)t]), b = pos(md.indices[3 * (size_t)t + 1]),
            c = pos(md.indices[3 * (size_t)t + 2]);
      // ray.rs:114: (v2 - v0).cross(v1 - v0).length_squared() == 0
      float ux = c.x - a.x, uy = c.y - a.y, uz = c.z - a.z;
      float vx = b.x - a.x, vy = b.y - a.y, vz = b.z - a.z;
      float cx = uy * vz - vy * uz, cy = uz * vx - vz * ux, cz = ux * vy - vx * uy;
      float l2 = cx * cx + cy * cy + cz * cz;
      DevTri d;
      uint32_t tb = t;
      float tf;
      std::memcpy(&tf, &tb, 4);
      d.v0 = make_float4(a.x, a.y, a.z, tf);
      d.v1 = make_float4(b.x, b.y, b.z, l2 == 0.0f ? 1.0f : 0.0f);
      d.v2 = make_float4(c.x, c.y, c.z, 0.0f);
      tris.push_back(d);
    }
  }

  // instances + TLAS
  std::vector<DevInstance> insts(desc->num_instances);
  std::vector<float> inst_bounds(6 * (size_t)desc->num_instances);
  for (uint32_t i = 0; i < desc->num_instances; ++i) {
    const tpt_instance_desc& id = desc->instances[i];
    if (id.mesh_index >= desc->num_meshes)
      return set_error(ctx, TPT_ERR_INVALID_ARG, "instance " + std::to_string(i) + ": mesh index out of range");
    const float* w = id.world_to_local;
    DevInstance d;
    d.m0 = make_float4(w[0], w[1], w[2], w[4]);
    d.m1 = make_float4(w[5], w[6], w[8], w[9]);
    d.m2 = make_float4(w[10], w[12], w[13], w[14]);
    d.node_base = mesh_node_base[id.mesh_index];
    d.tri_base = mesh_tri_base[id.mesh_index];
    d.root_word = mesh_root[id.mesh_index];
    d.material = id.material_index;
    insts[i] = d;
    // scene/mod.rs:869-893 transform_bounds of the mesh bounds
    const float* mb = &mesh_bounds[6 * (size_t)id.mesh_index];
    float* ib = &inst_bounds[6 * (size_t)i];
    bool first = true;
    for (int c = 0; c < 8; ++c) {
      Vec3f corner{(c & 4) ? mb[3] : mb[0], (c & 2) ? mb[4] : mb[1], (c & 1) ? mb[5] : mb[2]};
      Vec3f p = xform_point(id.local_to_world, corner);
      if (first) {
        ib[0] = ib[3] = p.x; ib[1] = ib[4] = p.y; ib[2] = ib[5] = p.z;
        first = false;
      } else {
        ib[0] = std::fmin(ib[0], p.x); ib[1] = std::fmin(ib[1], p.y); ib[2] = std::fmin(ib[2], p.z);
        ib[3] = std::fmax(ib[3], p.x); ib[4] = std::fmax(ib[4], p.y); ib[5] = std::fmax(ib[5], p.z);
      }
    }
  }
  uint32_t tlas_base = (uint32_t)nodes.size();
  uint32_t tlas_root = kEmptyWord;
  std::vector<uint32_t> tlas_prims;
  if (desc->num_instances) {
    QbvhHost built;
    const QbvhNodeHost* qn;
    uint64_t qnn;
    const uint32_t* qp;
    uint64_t qpn;
    if (desc->tlas.primitive_indices) {
      qn = reinterpret_cast<const QbvhNodeHost*>(desc->tlas.nodes);
      qnn = desc->tlas.num_nodes;
      qp = desc->tlas.primitive_indices;
      qpn = desc->tlas.num_primitives;
      if (qnn && !qn) return set_error(ctx, TPT_ERR_INVALID_ARG, "TLAS nodes is NULL");
    } else {
      build_qbvh_for(ctx, inst_bounds.data(), desc->num_instances, threads, &built);
      qn = built.nodes.data();
      qnn = built.nodes.size();
      qp = built.prim_indices.data();
      qpn = built.prim_indices.size();
    }
    std::string why;
    if (qpn != desc->num_instances || !validate_qbvh(qn, qnn, qp, qpn, desc->num_instances, &why))
      return set_error(ctx, TPT_ERR_INVALID_ARG, "TLAS invalid: " + (why.empty() ? std::string("count mismatch") : why));
    for (uint64_t i = 0; i < qnn; ++i) nodes.push_back(to_dev(qn[i]));
    tlas_prims.assign(qp, qp + qpn);
    tlas_root = qnn ? 0u : (kLeafFlag | ((uint32_t)qpn << 24));
  }

  auto* s = new tpt_scene();
  s->ctx = ctx;
  s->num_meshes = desc->num_meshes;
  s->num_instances = desc->num_instances;
  s->mesh_tri_counts = tri_counts;
  tpt_status st = TPT_OK;
  if (!st) st = dev_upload(s, nodes.data(), nodes.size(), &s->geo.nodes);
  if (!st) st = dev_upload(s, tris.data(), tris.size(), &s->geo.tris);
  if (!st) st = dev_upload(s, insts.data(), insts.size(), &s->geo.instances);
  if (!st) st = dev_upload(s, tlas_prims.data(), tlas_prims.size(), &s->geo.tlas_prims);
  if (st) {
    tpt_scene_release(s);
    return st;
  }
  s->geo.tlas_node_base = tlas_base;
  s->geo.tlas_root_word = tlas_root;
  s->geo.num_instances = desc->num_instances;
  st = upload_render_data(s, desc);
  if (st) {
    tpt_scene_release(s);
    return st;
  }
  *out = s;
  return TPT_OK;
}

tpt_status tpt_scene_release(tpt_scene* s) {
  if (!s) return TPT_OK;
  if (s->ctx) cudaSetDevice(s->ctx->device);
  for (void* p : s->allocations) cudaFree(p);
  if (s->d_adj) cudaFree(s->d_adj);
  delete s;
  return TPT_OK;
}

tpt_status tpt_scene_light_tree(const tpt_scene* s, tpt_light_tree_view* v) {
  if (!s || !v) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL argument");
  v->nodes = reinterpret_cast<const tpt_light_node*>(s->light_tree.nodes.data());
  v->num_nodes = s->light_tree.nodes.size();
  v->root = s->light_tree.root;
  return TPT_OK;
}

tpt_status tpt_scene_device_bytes(const tpt_scene* s, uint64_t* bytes) {
  if (!s || !bytes) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL argument");
  *bytes = s->device_bytes;
  return TPT_OK;
}

// ---- ray queries ----------------------------------------------------------
tpt_status tpt_traverse_device(tpt_context* ctx, const tpt_scene* scene, const float* rays, uint64_t n, int mode,
                               int32_t* prim, float* t, int32_t* instance, float* bary, void* stream) {
  if (!ctx || !scene) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL context or scene");
  if (n && (!rays || !prim || !t)) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL ray or output buffer");
  if (mode != TPT_CLOSEST_HIT && mode != TPT_ANY_HIT) return set_error(ctx, TPT_ERR_INVALID_ARG, "bad mode");
  tpt_status st = set_device(ctx);
  if (st) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  note_device_call(ctx, "tpt_traverse_device");
  return cuda_check(ctx,
                    launch_traverse_strided(scene->geo, rays, n, n, mode, prim, t, instance, bary, n,
                                            next_counter(ctx), ctx->d_err, ctx->num_sms, s, nullptr, nullptr),
                    "traverse kernel launch");
}

tpt_status tpt_traverse_alpha_device(tpt_context* ctx, const tpt_scene* scene, const float* rays, uint64_t n,
                                     uint32_t* aux, int32_t* prim, float* t, int32_t* instance, float* bary,
                                     void* stream) {
  if (!ctx || !scene) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL context or scene");
  if (n && (!rays || !aux || !prim || !t)) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL ray, state or output buffer");
  tpt_status st = set_device(ctx);
  if (st) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  note_device_call(ctx, "tpt_traverse_alpha_device");
  return cuda_check(ctx,
                    launch_traverse_strided(scene->geo, rays, n, n, TPT_CLOSEST_HIT, prim, t, instance, bary, n,
                                            next_counter(ctx), ctx->d_err, ctx->num_sms, s, nullptr, nullptr,
                                            nullptr, nullptr, nullptr, nullptr, aux),
                    "traverse kernel launch");
}

tpt_status tpt_traverse_stats_device(tpt_context* ctx, const tpt_scene* scene, const float* rays, uint64_t n,
                                     int mode, int32_t* prim, float* t, uint32_t* node_tests, uint32_t* tri_tests,
                                     void* stream) {
  if (!ctx || !scene) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL context or scene");
  if (n && (!rays || !prim || !t || !node_tests || !tri_tests))
    return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL buffer");
  if (mode != TPT_CLOSEST_HIT && mode != TPT_ANY_HIT) return set_error(ctx, TPT_ERR_INVALID_ARG, "bad mode");
  tpt_status st = set_device(ctx);
  if (st) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  note_device_call(ctx, "tpt_traverse_stats_device");
  st = cuda_check(ctx,
                             launch_traverse_strided(scene->geo, rays, n, n, mode, prim, t, nullptr, nullptr, n,
                                                     next_counter(ctx), ctx->d_err, ctx->num_sms, s, node_tests,
                                                     tri_tests),
                             "traverse kernel launch");
  if (st) return st;
  return check_device_errors(ctx, s);
}

tpt_status tpt_traverse(tpt_context* ctx, const tpt_scene* scene, const float* rays, uint64_t n, int mode,
                        int32_t* prim, float* t, int32_t* instance, float* bary) {
  if (!ctx || !scene) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL context or scene");
  if (n == 0) return TPT_OK;
  if (!rays || !prim || !t) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL ray or output buffer");
  if (mode != TPT_CLOSEST_HIT && mode != TPT_ANY_HIT) return set_error(ctx, TPT_ERR_INVALID_ARG, "bad mode");
  tpt_status st = set_device(ctx);
  if (!st) st = ensure_pipeline(ctx);
  if (st) return st;
  // Device buffers for the whole batch: rays (7 planes) then outputs.
  const int n_out = 2 + (instance ? 1 : 0) + (bary ? 3 : 0);
  const size_t dev_bytes = (7 + (size_t)n_out) * n * 4;
  if ((st = ensure_device_staging(ctx, dev_bytes))) return st;
  float* d_rays = (float*)ctx->d_stage;
  int32_t* d_prim = (int32_t*)(d_rays + 7 * n);
  float* d_t = (float*)(d_prim + n);
  int32_t* d_inst = instance ? (int32_t*)(d_t + n) : nullptr;
  float* d_bary = bary ? (instance ? (float*)(d_inst + n) : (d_t + n)) : nullptr;

  // closest-hit queries start at t_max = +inf and never read the tmax plane: it is not copied
  const int in_planes = mode == TPT_CLOSEST_HIT ? 6 : 7;
  const bool in_pinned = is_pinned(rays);
  const bool out_pinned = is_pinned(prim) && is_pinned(t) && (!instance || is_pinned(instance)) &&
                          (!bary || is_pinned(bary));
  // Chunks of about 2M rays, at least 4 when the batch allows.
  uint64_t chunk = std::max<uint64_t>(1 << 16, std::min<uint64_t>(1 << 21, (n + 3) / 4));
  struct Out { void* host; const void* dev; size_t planes; };
  const Out outs[4] = {{prim, d_prim, 1}, {t, d_t, 1}, {instance, d_inst, 1}, {bary, d_bary, 3}};
  if (in_pinned && out_pinned) {
    // Pinned buffers: copies in on one stream, kernels alternating on two
    // streams, copies out on a third, ordered by per-chunk events, so the
    // host-to-device copies run back to back while earlier chunks traverse
    // and later ones drain.
    const std::vector<uint64_t> sizes = chunk_schedule(n, chunk);
    if ((st = ensure_copy_pipeline(ctx, sizes.size()))) return st;
    cudaEventRecord(ctx->ev_start, ctx->stream);
    cudaStreamWaitEvent(ctx->copy_in, ctx->ev_start, 0);
    for (int k = 0; k < 2; ++k) cudaStreamWaitEvent(ctx->pipe[k], ctx->ev_start, 0);
    uint64_t b = 0;
    for (size_t c = 0; c < sizes.size(); ++c) {
      const uint64_t m = sizes[c];
      for (int p = 0; p < in_planes; ++p)
        cudaMemcpyAsync(d_rays + p * n + b, rays + p * n + b, m * 4, cudaMemcpyHostToDevice, ctx->copy_in);
      cudaEventRecord(ctx->ev_in[c], ctx->copy_in);
      cudaStream_t s = ctx->pipe[c & 1];
      cudaStreamWaitEvent(s, ctx->ev_in[c], 0);
      cudaError_t e = launch_traverse_strided(scene->geo, d_rays + b, n, m, mode, d_prim + b, d_t + b,
                                              d_inst ? d_inst + b : nullptr, d_bary ? d_bary + b : nullptr, n,
                                              next_counter(ctx), ctx->d_err, ctx->num_sms, s, nullptr, nullptr);
      if ((st = cuda_check(ctx, e, "traverse kernel launch"))) return st;
      cudaEventRecord(ctx->ev_done[c], s);
      cudaStreamWaitEvent(ctx->copy_out, ctx->ev_done[c], 0);
      for (const Out& o : outs) {
        if (!o.host) continue;
        for (size_t p = 0; p < o.planes; ++p)
          cudaMemcpyAsync((char*)o.host + (p * n + b) * 4, (const char*)o.dev + (p * n + b) * 4, m * 4,
                          cudaMemcpyDeviceToHost, ctx->copy_out);
      }
      b += m;
    }
    cudaEventRecord(ctx->ev_slot[0], ctx->copy_out);
    cudaStreamWaitEvent(ctx->stream, ctx->ev_slot[0], 0);
    if ((st = cuda_check(ctx, cudaGetLastError(), "traverse pipeline"))) return st;
    return check_device_errors(ctx, ctx->stream);
  }
  // Pageable buffers: pinned staging slots, pipelined on two streams.
  const uint64_t n_chunks = (n + chunk - 1) / chunk;
  if (!in_pinned || !out_pinned) {
    const size_t per_slot = (7 + (size_t)n_out) * chunk * 4;
    if ((st = ensure_host_staging(ctx, 2 * per_slot))) return st;
  }
  cudaEventRecord(ctx->ev_start, ctx->stream);
  for (int k = 0; k < 2; ++k) cudaStreamWaitEvent(ctx->pipe[k], ctx->ev_start, 0);
  for (uint64_t c = 0; c < n_chunks; ++c) {
    const int k = (int)(c & 1);
    cudaStream_t s = ctx->pipe[k];
    const uint64_t b = c * chunk, m = std::min<uint64_t>(chunk, n - b);
    float* hslot = (float*)((char*)ctx->h_stage + k * ((7 + (size_t)n_out) * chunk * 4));
    if (!in_pinned || !out_pinned) {
      // the slot is reused every other chunk: wait until its last copy-out is done
      cudaEventSynchronize(ctx->ev_slot[k]);
    }
    if (in_pinned) {
      for (int p = 0; p < in_planes; ++p)
        cudaMemcpyAsync(d_rays + p * n + b, rays + p * n + b, m * 4, cudaMemcpyHostToDevice, s);
    } else {
      for (int p = 0; p < in_planes; ++p) std::memcpy(hslot + p * m, rays + p * n + b, m * 4);
      for (int p = 0; p < in_planes; ++p)
        cudaMemcpyAsync(d_rays + p * n + b, hslot + p * m, m * 4, cudaMemcpyHostToDevice, s);
    }
    // the kernel reads plane p of the chunk at d_rays + p*n + b: pass a view with stride n
    cudaError_t e = launch_traverse_strided(scene->geo, d_rays + b, n, m, mode, d_prim + b, d_t + b,
                                            d_inst ? d_inst + b : nullptr, d_bary ? d_bary + b : nullptr, n,
                                            next_counter(ctx), ctx->d_err, ctx->num_sms, s, nullptr, nullptr);
    if ((st = cuda_check(ctx, e, "traverse kernel launch"))) return st;
    float* hout = hslot + 7 * m;
    size_t ho = 0;
    for (const Out& o : outs) {
      if (!o.host) continue;
      for (size_t p = 0; p < o.planes; ++p) {
        const char* src = (const char*)o.dev + (p * n + b) * 4;
        if (out_pinned) {
          cudaMemcpyAsync((char*)o.host + (p * n + b) * 4, src, m * 4, cudaMemcpyDeviceToHost, s);
        } else {
          cudaMemcpyAsync(hout + ho * m, src, m * 4, cudaMemcpyDeviceToHost, s);
          ++ho;
        }
      }
    }
    if (!out_pinned) {
      // drain the slot before it is reused (two chunks later)
      cudaStreamSynchronize(s);
      size_t h2 = 0;
      for (const Out& o : outs) {
        if (!o.host) continue;
        for (size_t p = 0; p < o.planes; ++p, ++h2)
          std::memcpy((char*)o.host + (p * n + b) * 4, hout + h2 * m, m * 4);
      }
    }
    cudaEventRecord(ctx->ev_slot[k], s);
  }
  for (int k = 0; k < 2; ++k) {
    cudaEventRecord(ctx->ev_slot[k], ctx->pipe[k]);
    cudaStreamWaitEvent(ctx->stream, ctx->ev_slot[k], 0);
  }
  if ((st = cuda_check(ctx, cudaGetLastError(), "traverse pipeline"))) return st;
  return check_device_errors(ctx, ctx->stream);
}

}  // extern "C"
