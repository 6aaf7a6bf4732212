// BDPT as a wavefront (integrator/bdpt.rs:70-131 split into stages), per chunk
// of samples:
//
//   bd_init      : per sample, the camera ray and the light endpoint
//   bd_step x max_depth, each after a traversal of the subpath ray queue:
//                  one iteration of the camera loop (depth = step) or of the
//                  light loop (depth = step + 1) per queued ray, vertices into
//                  HBM, camera-side emission into L0, next rays into the other
//                  queue (the same step functions the one-kernel BDPT runs).
//                  A queue holds the camera rays in its first half and the
//                  light rays in its second (sample_capacity slots each, own
//                  counters), so every warp of bd_step runs one of the two
//                  loops and the two halves are traversed as two launches;
//                  in scenes with point, spot, directional or environment
//                  lights, the camera vertices' light samples queue a shadow
//                  ray, traversed after the step, and bd_nee_resolve adds the
//                  unoccluded ones to L0 before the next step
//   bd_pairs     : per sample, its nl * nc connection slots allocated
//                  contiguously in the pair queue (one atomic per warp)
//   bd_connect   : per pair, bdpt_connect_prepare; non-zero contributions
//                  append their visibility ray to the shadow queue
//   traverse     : the persistent traversal kernel over the shadow queue
//   bd_resolve   : per visible connection, the MIS weight (bdpt_mis) times the
//                  contribution, into the pair's slot
//   bd_finalize  : per sample, L0 plus the pair slots in the reference's
//                  (light, camera) order
//
// Every connection does the arithmetic of the one-kernel BDPT in the same
// order (the sums per sample too), so both executions give the same samples
// bit for bit.  The connections, the bulk of the work, thus run as uniform
// kernels over compacted queues instead of inside each sample's thread.
#include "../api/internal.h"
#include "../device/bdpt.cuh"

namespace tpt {

constexpr int kBdWfBlock = 128;
#ifndef TPT_BD_STEP_MINB
// bd_step's minimum resident blocks per SM: 4 caps it at 128 registers (from
// 168, a few hundred bytes of spills), 16 warps per SM instead of 12: 6 % less
// BDPT time on the large scene
#define TPT_BD_STEP_MINB 4
#endif

// Warp-exclusive prefix sum of `v` (all lanes call); returns the lane's offset
// and the warp total in `total`.
__device__ __forceinline__ uint32_t warp_exclusive_scan(uint32_t v, uint32_t& total) {
  const unsigned lane = threadIdx.x & 31u;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if ((int)lane >= o) x += y;
  }
  total = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}

__device__ __forceinline__ uint32_t warp_append1(uint32_t* counter, bool pred) {
  const unsigned act = __activemask();
  const unsigned m = __ballot_sync(act, pred);
  const unsigned lane = threadIdx.x & 31u;
  const int leader = __ffs(act) - 1;
  uint32_t base = 0;
  if ((int)lane == leader && m) base = atomicAdd(counter, (uint32_t)__popc(m));
  base = __shfl_sync(act, base, leader);
  return base + (uint32_t)__popc(m & ((1u << lane) - 1u));
}

// Queue halves: camera rays at [0, sample_capacity) counted in counts[2 + q],
// light rays at [sample_capacity, 2 * sample_capacity) in counts[4 + q].
__device__ __forceinline__ void push_ray(const BdWfBuffers& B, int q, uint32_t slot, V3 o, V3 d, uint32_t tag) {
  const uint32_t Q = 2 * B.sample_capacity;
  float* r = B.q_ray[q];
  r[slot] = o.x;
  r[Q + slot] = o.y;
  r[2 * Q + slot] = o.z;
  r[3 * Q + slot] = d.x;
  r[4 * Q + slot] = d.y;
  r[5 * Q + slot] = d.z;
  r[6 * Q + slot] = __int_as_float(0x7f800000);
  B.q_tag[q][slot] = tag;
}

__device__ __forceinline__ PathSamplerDev sampler_of(const RenderLaunch& P, uint64_t path, uint32_t& px,
                                                     uint32_t& py) {
  const uint32_t pixel = (uint32_t)(path / P.spp), sample = (uint32_t)(path % P.spp);
  px = pixel % P.width;
  py = pixel / P.width;
  PathSamplerDev ps;
  ps.init(px, py, sample, P.log2_spp, P.n_base4_digits, P.seed);
  return ps;
}

constexpr uint32_t kLightTag = 0x80000000u;

// Per sample: the camera ray and the light endpoint (bdpt.rs:96-110, 264-300);
// both first rays into queue 0.
__global__ void __launch_bounds__(kBdWfBlock) bd_init(const __grid_constant__ DevRender S,
                                                  const __grid_constant__ RenderLaunch P, BdWfBuffers B,
                                                      uint64_t first_path, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t px, py;
  const PathSamplerDev ps = sampler_of(P, first_path + i, px, py);
  float c0, c1;
  ps.sample_2d(kDimCamera, c0, c1);
  const float fx = ((float)px + 0.5f) + 0.5f * tent(c0);
  const float fy = ((float)py + 0.5f) + 0.5f * tent(c1);
  const V3 d = camera_dir(P.cam, P.width, P.height, fx, fy);
  const V3 o = V3{P.cam.eye[0], P.cam.eye[1], P.cam.eye[2]};
  BdCamState c;
  camera_state_init(c, P.max_depth > 0);
  BdVertex* lig = B.verts + (size_t)i * 2 * B.max_vertices + B.max_vertices;
  V3 lo, ld;
  BdLightState l;
  l.pending_pdf = 0.0f;
  l.lock = -1.0f;
  l.alive = bdpt_light_endpoint(S, P, ps, lig, lo, ld, l.beta, l.pending_from, l.pending_pdf);
  l.n = l.alive ? 1u : 0u;
  B.cam_state[i] = c;
  B.light_state[i] = l;
  B.L0[3 * (size_t)i] = 0.0f;
  B.L0[3 * (size_t)i + 1] = 0.0f;
  B.L0[3 * (size_t)i + 2] = 0.0f;
  const bool cam_ray = c.alive;
  const bool light_ray = l.alive && P.max_depth > 1;
  const uint32_t qc = warp_append1(&B.counts[2], cam_ray);
  if (cam_ray) push_ray(B, 0, qc, o, d, i);
  const uint32_t ql = warp_append1(&B.counts[4], light_ray);
  if (light_ray) push_ray(B, 0, B.sample_capacity + ql, lo, ld, i | kLightTag);
}

// Step `step` of both loops: camera rays of depth `step`, light rays of depth
// step + 1, traced into the hit arrays; the next rays into queue cur ^ 1.
__global__ void __launch_bounds__(kBdWfBlock, TPT_BD_STEP_MINB) bd_step(const __grid_constant__ DevRender S,
                                                  const __grid_constant__ RenderLaunch P, BdWfBuffers B,
                                                      uint64_t first_path, uint32_t step, int cur) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t S_cap = B.sample_capacity, Q = 2 * S_cap;
  if (j < S_cap ? j >= B.counts[2 + cur] : j - S_cap >= B.counts[4 + cur]) return;
  const uint32_t tag = B.q_tag[cur][j];
  const uint32_t i = tag & ~kLightTag;
  const bool light = (tag & kLightTag) != 0;
  uint32_t px, py;
  const PathSamplerDev ps = sampler_of(P, first_path + i, px, py);
  TraceResult h;
  h.tri = B.h_tri[j];
  h.inst = B.h_inst[j];
  h.t = B.h_t[j];
  h.b0 = B.h_bary[j];
  h.b1 = B.h_bary[Q + j];
  h.b2 = B.h_bary[2 * Q + j];
  const float* r = B.q_ray[cur];
  V3 ro = V3{r[j], r[Q + j], r[2 * Q + j]};
  V3 rd = V3{r[3 * Q + j], r[4 * Q + j], r[5 * Q + j]};
  BdVertex* cam = B.verts + (size_t)i * 2 * B.max_vertices;
  bool next = false;
  bool nee = false;
  DirectPrep dp;
  if (!light) {
    BdCamState c = B.cam_state[i];
    V3 L = V3{B.L0[3 * (size_t)i], B.L0[3 * (size_t)i + 1], B.L0[3 * (size_t)i + 2]};
    camera_step<int>(S, P, ps, step, h, ro, rd, cam, c, L, nee, dp);
    B.cam_state[i] = c;
    B.L0[3 * (size_t)i] = L.x;
    B.L0[3 * (size_t)i + 1] = L.y;
    B.L0[3 * (size_t)i + 2] = L.z;
    next = c.alive && step + 1 < P.max_depth;
  } else {
    BdLightState l = B.light_state[i];
    light_step<int>(S, ps, step + 1, h, ro, rd, cam + B.max_vertices, l);
    B.light_state[i] = l;
    next = l.alive && step + 2 < P.max_depth;
  }
  const uint32_t q = warp_append1(&B.counts[(light ? 4 : 2) + (cur ^ 1)], next);
  if (next) push_ray(B, cur ^ 1, light ? S_cap + q : q, ro, rd, tag);
  // a camera vertex's light sample: its shadow ray into the visibility queue
  // (free until the connection stage), contribution and light distance beside it
  const uint32_t qs = warp_append1(&B.counts[1], nee);
  if (!nee) return;
  const uint32_t C = B.pair_capacity;
  float* sr = B.s_ray;
  sr[qs] = dp.so.x;
  sr[C + qs] = dp.so.y;
  sr[2 * C + qs] = dp.so.z;
  sr[3 * C + qs] = dp.wi.x;
  sr[4 * C + qs] = dp.wi.y;
  sr[5 * C + qs] = dp.wi.z;
  sr[6 * C + qs] = __int_as_float(0x7f800000);
  B.s_pair[qs] = i;
  B.c[3 * (size_t)qs] = dp.contrib.x;
  B.c[3 * (size_t)qs + 1] = dp.contrib.y;
  B.c[3 * (size_t)qs + 2] = dp.contrib.z;
  B.dist[qs] = dp.dist;
}

// The camera vertices' light samples of one step whose shadow rays are
// unoccluded (unoccluded_ray, integrator/mod.rs:239-265; point, spot,
// directional and environment lights have no target triangle) into L0.
__global__ void __launch_bounds__(kBdWfBlock) bd_nee_resolve(BdWfBuffers B) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= B.counts[1]) return;
  if (!shadow_visible(B.s_tri[e], B.s_inst[e], B.s_t[e], 0xFFFFFFFFu, 0xFFFFFFFFu, B.dist[e])) return;
  const uint32_t i = B.s_pair[e];
  B.L0[3 * (size_t)i] = B.L0[3 * (size_t)i] + B.c[3 * (size_t)e];
  B.L0[3 * (size_t)i + 1] = B.L0[3 * (size_t)i + 1] + B.c[3 * (size_t)e + 1];
  B.L0[3 * (size_t)i + 2] = B.L0[3 * (size_t)i + 2] + B.c[3 * (size_t)e + 2];
}

// Per sample: subpath lengths and the nl * nc connection slots, contiguous
// per sample (one atomic per warp).
__global__ void __launch_bounds__(kBdWfBlock) bd_pairs(BdWfBuffers B, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t nc = valid ? B.cam_state[i].n : 0u;
  const uint32_t nl = valid ? B.light_state[i].n : 0u;
  const uint32_t np = nl * nc;
  uint32_t total;
  const uint32_t off = warp_exclusive_scan(np, total);
  uint32_t pbase = 0;
  if (lane == 31 && total) pbase = atomicAdd(B.counts, total);
  pbase = __shfl_sync(0xffffffffu, pbase, 31) + off;
  if (!valid) return;
  B.nc[i] = nc;
  B.nl[i] = nl;
  B.pair_base[i] = pbase;
  for (uint32_t k = 0; k < np; ++k) B.pair_sample[pbase + k] = i;
}

__global__ void __launch_bounds__(kBdWfBlock) bd_connect(const __grid_constant__ DevRender S, BdWfBuffers B) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= B.counts[0]) return;
  const uint32_t MD = B.max_vertices;
  const uint32_t i = B.pair_sample[j];
  const uint32_t k = j - B.pair_base[i];
  const uint32_t nc = B.nc[i];
  const uint32_t li = k / nc, ci = k - (k / nc) * nc;
  const BdVertex* cam = B.verts + (size_t)i * 2 * MD;
  const BdVertex& lv = cam[MD + li];
  const BdVertex& cv = cam[ci];
  BdConnection cn;
  bool want = false;
  if ((lv.flags & kBdConnectible) && (cv.flags & kBdConnectible)) want = bdpt_connect_prepare(S, lv, cv, cn) == 2;
  B.contrib[3 * (size_t)j] = 0.0f;
  B.contrib[3 * (size_t)j + 1] = 0.0f;
  B.contrib[3 * (size_t)j + 2] = 0.0f;
  const uint32_t q = warp_append1(&B.counts[1], want);
  if (!want) return;
  const uint32_t C = B.pair_capacity;
  float* r = B.s_ray;
  r[q] = cn.origin.x;
  r[C + q] = cn.origin.y;
  r[2 * C + q] = cn.origin.z;
  r[3 * C + q] = cn.dir.x;
  r[4 * C + q] = cn.dir.y;
  r[5 * C + q] = cn.dir.z;
  r[6 * C + q] = __int_as_float(0x7f800000);
  B.s_pair[q] = j;
  B.c[3 * (size_t)j] = cn.c.x;
  B.c[3 * (size_t)j + 1] = cn.c.y;
  B.c[3 * (size_t)j + 2] = cn.c.z;
  B.dist[j] = cn.dist;
}

__global__ void __launch_bounds__(kBdWfBlock) bd_resolve(const __grid_constant__ DevRender S, BdWfBuffers B) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= B.counts[1]) return;
  const uint32_t MD = B.max_vertices;
  const uint32_t j = B.s_pair[e];
  const uint32_t i = B.pair_sample[j];
  const uint32_t k = j - B.pair_base[i];
  const uint32_t nc = B.nc[i];
  const uint32_t li = k / nc, ci = k - (k / nc) * nc;
  const BdVertex* cam = B.verts + (size_t)i * 2 * MD;
  // visible_between (bdpt.rs:577-602)
  const int32_t tri = B.s_tri[e];
  if (tri >= 0) {
    const bool target = (uint32_t)B.s_inst[e] == cam[ci].v.inst && (uint32_t)tri == cam[ci].v.tri;
    if (!target && !(B.s_t[e] >= B.dist[j] * (1.0f - kShadowTolerance))) return;
  }
  const float w = bdpt_mis(S, cam + MD, li + 1, cam, ci + 1);
  const V3 c = V3{B.c[3 * (size_t)j], B.c[3 * (size_t)j + 1], B.c[3 * (size_t)j + 2]};
  const V3 wc = w * c;
  B.contrib[3 * (size_t)j] = wc.x;
  B.contrib[3 * (size_t)j + 1] = wc.y;
  B.contrib[3 * (size_t)j + 2] = wc.z;
}

__global__ void __launch_bounds__(kBdWfBlock) bd_finalize(BdWfBuffers B, uint32_t n, float* __restrict__ samples) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  V3 L = V3{B.L0[3 * (size_t)i], B.L0[3 * (size_t)i + 1], B.L0[3 * (size_t)i + 2]};
  const uint32_t np = B.nl[i] * B.nc[i];
  const float* c = B.contrib + 3 * (size_t)B.pair_base[i];
  for (uint32_t k = 0; k < np; ++k) {
    const V3 wc = V3{c[3 * k], c[3 * k + 1], c[3 * k + 2]};
    if (wc.x == 0.0f && wc.y == 0.0f && wc.z == 0.0f) continue;  // a zero connection adds exactly zero
    L = L + wc;
  }
  samples[3 * (size_t)i] = L.x;
  samples[3 * (size_t)i + 1] = L.y;
  samples[3 * (size_t)i + 2] = L.z;
}

static inline unsigned grid_of(uint64_t n) { return (unsigned)((n + kBdWfBlock - 1) / kBdWfBlock); }

cudaError_t launch_bdpt_wavefront(const DevGeometry& geo, const DevRenderData& rd, const RenderLaunch& P,
                                  const BdWfBuffers& B, uint64_t first_path, uint32_t n, float* samples,
                                  unsigned long long* counter, uint32_t* err, int num_sms, cudaStream_t s,
                                  unsigned long long* totals, unsigned long long* counter2, cudaStream_t side,
                                  cudaEvent_t fork, cudaEvent_t join) {
  if (n == 0) return cudaSuccess;
  if (!counter2 || !fork || !join) side = nullptr;
  DevRender S{geo, rd};
  cudaError_t e = cudaMemsetAsync(B.counts, 0, 6 * sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  const uint32_t S_cap = B.sample_capacity, Q = 2 * S_cap;
  bd_init<<<grid_of(n), kBdWfBlock, 0, s>>>(S, P, B, first_path, n);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const bool lights = rd.num_extra_lights > 0;
  for (uint32_t step = 0; step < P.max_depth; ++step) {
    const int cur = (int)(step & 1u);
    if ((e = cudaMemsetAsync(B.counts + 2 + (cur ^ 1), 0, sizeof(uint32_t), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(B.counts + 4 + (cur ^ 1), 0, sizeof(uint32_t), s)) != cudaSuccess) return e;
    // the camera half and the light half of the queue (hits at the rays' slots,
    // disjoint halves): with a side stream the light half runs beside the
    // camera half, which matters in late steps, where each launch lasts as long
    // as its longest ray's chain of node loads however few rays it holds
    if (side) {
      if ((e = cudaEventRecord(fork, s)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(side, fork, 0)) != cudaSuccess) return e;
    }
    e = launch_traverse_strided(geo, B.q_ray[cur], Q, S_cap, TPT_CLOSEST_HIT, B.h_tri, B.h_t, B.h_inst, B.h_bary, Q,
                                counter, err, num_sms, s, nullptr, nullptr, B.counts + 2 + cur, nullptr, nullptr,
                                totals);
    if (e == cudaSuccess)
      e = launch_traverse_strided(geo, B.q_ray[cur] + S_cap, Q, S_cap, TPT_CLOSEST_HIT, B.h_tri + S_cap,
                                  B.h_t + S_cap, B.h_inst + S_cap, B.h_bary + S_cap, Q, side ? counter2 : counter, err,
                                  num_sms, side ? side : s, nullptr, nullptr, B.counts + 4 + cur, nullptr, nullptr,
                                  totals);
    if (side) {  // join even after an error: no branch is left open on the caller's stream
      const cudaError_t ej = cudaEventRecord(join, side);
      const cudaError_t ew = ej == cudaSuccess ? cudaStreamWaitEvent(s, join, 0) : ej;
      if (e == cudaSuccess) e = ew;
    }
    if (e != cudaSuccess) return e;
    bd_step<<<grid_of(Q), kBdWfBlock, 0, s>>>(S, P, B, first_path, step, cur);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (lights) {  // at most one light sample per sample and step: n <= sample_capacity <= pair_capacity
      e = launch_traverse_strided(geo, B.s_ray, B.pair_capacity, B.pair_capacity, TPT_CLOSEST_HIT, B.s_tri, B.s_t,
                                  B.s_inst, nullptr, B.pair_capacity, counter, err, num_sms, s, nullptr, nullptr,
                                  B.counts + 1, nullptr, nullptr, totals ? totals + 4 : nullptr);
      if (e != cudaSuccess) return e;
      bd_nee_resolve<<<grid_of(B.sample_capacity), kBdWfBlock, 0, s>>>(B);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      if ((e = cudaMemsetAsync(B.counts + 1, 0, sizeof(uint32_t), s)) != cudaSuccess) return e;
    }
  }
  bd_pairs<<<grid_of(n), kBdWfBlock, 0, s>>>(B, n);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  bd_connect<<<grid_of(B.pair_capacity), kBdWfBlock, 0, s>>>(S, B);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  e = launch_traverse_strided(geo, B.s_ray, B.pair_capacity, B.pair_capacity, TPT_CLOSEST_HIT, B.s_tri, B.s_t,
                              B.s_inst, nullptr, B.pair_capacity, counter, err, num_sms, s, nullptr, nullptr,
                              B.counts + 1, nullptr, nullptr, totals ? totals + 4 : nullptr);
  if (e != cudaSuccess) return e;
  bd_resolve<<<grid_of(B.pair_capacity), kBdWfBlock, 0, s>>>(S, B);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  bd_finalize<<<grid_of(n), kBdWfBlock, 0, s>>>(B, n, samples);
  return cudaGetLastError();
}

}  // namespace tpt
