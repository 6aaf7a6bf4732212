// Wavefront path tracing: the MIS integrator of integrator/mis.rs split into
// stage kernels over compacted queues of path slots,
//
//   generate -> [ traverse(closest) -> shade -> traverse(shadow) -> resolve ]
//               x (max_depth + 1) -> finalize -> accumulate
//
// Traversal runs in the persistent-warp kernel of traverse_kernels.cu; shade
// handles one path vertex (emission with MIS against the previous vertex, NEE
// preparation, BSDF sampling, Russian roulette) and appends the next ray and
// the shadow ray with warp-aggregated atomics; resolve adds the NEE
// contribution of visible shadow rays.  Each path's radiance is updated in the
// reference's order (emission of vertex d, then NEE of vertex d, then emission
// of vertex d + 1), so the result equals the megakernel's bit for bit.
// Stage launch shapes do not depend on queue lengths (those live on the
// device), so one bounce is a fixed launch sequence that a CUDA graph replays.
//
// The batched instantiation (BATCH = true) runs many jobs (scenes, cameras,
// resolutions, spp, depths) through one launch sequence: slot i of a chunk is
// global path first_path + i of the batch, whose job is found by binary search
// over the jobs' path bases; every slot, queued ray and shadow ray carries its
// job index, and each stage reads the job's scene and launch record from the
// DevJob array instead of its kernel parameters.
//
// The adjoint instantiation (ADJ = true) replays the same paths with the
// radiance planes holding R, the part of the path's radiance still to come:
// generate starts R at the path's radiance from the forward pass, shade and
// resolve subtract what each vertex collects, and shade adds, at every rough
// OpenPBR vertex, dLoss/dL * R * (df/dtheta) / f to the per-material gradients.
// A light sample C at an OpenPBR vertex (directional lights) is only known to
// count once its shadow ray is resolved, while shade has already used R with C
// still in it; shade therefore queues, with the shadow ray, the change
// dLoss/dL * C * [(df/dtheta) / f at the light direction - the same at the
// sampled direction], which resolve adds when the ray is unoccluded.
#include "../api/internal.h"
#include "../device/adjoint.cuh"
#include "../device/render.cuh"

namespace tpt {

constexpr int kWfBlock = 256;
// Blocks per SM the shade kernel's register budget is sized for: 512 threads
// per SM (128 registers, 16 warps) for rendering, which the forward variants
// reach without spilling; the adjoint variant (~200 registers) is not capped.
template <bool ADJ, int BS>
constexpr int shade_min_blocks() {
  return ADJ ? 1 : 512 / BS;
}

__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool pred) {
  const unsigned act = __activemask();
  const unsigned m = __ballot_sync(act, pred);
  const unsigned lane = threadIdx.x & 31u;
  const int leader = __ffs(act) - 1;
  uint32_t base = 0;
  if ((int)lane == leader && m) base = atomicAdd(counter, (uint32_t)__popc(m));
  base = __shfl_sync(act, base, leader);
  return base + (uint32_t)__popc(m & ((1u << lane) - 1u));
}

// Job of global path g: the last job whose path_base <= g (jobs sorted by path_base).
__device__ __forceinline__ uint32_t job_of_path(const DevJob* __restrict__ jobs, uint32_t n_jobs, uint64_t g) {
  uint32_t lo = 0, hi = n_jobs;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (jobs[mid].path_base <= g) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <bool ADJ, bool BATCH>
__global__ void __launch_bounds__(kWfBlock) wf_generate(const __grid_constant__ DevRender S0,
                                                                 const __grid_constant__ RenderLaunch P0, WfBuffers B,
                                                        uint64_t first_path, uint32_t n_paths,
                                                        const float* __restrict__ primal,
                                                        const DevJob* __restrict__ jobs, uint32_t n_jobs) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    B.counts[0] = n_paths;
    B.counts[1] = 0;
    B.counts[2] = 0;
    // the chunk's first path, for the later stages (which a graph replays
    // unchanged from chunk to chunk)
    B.counts[4] = (uint32_t)first_path;
    B.counts[5] = (uint32_t)(first_path >> 32);
  }
  if (i >= n_paths) return;
  const uint32_t C = B.capacity;
  const uint32_t jb = BATCH ? job_of_path(jobs, n_jobs, first_path + i) : 0u;
  const RenderLaunch& P = BATCH ? jobs[jb].P : P0;
  const uint64_t path = first_path + i - (BATCH ? jobs[jb].path_base : 0ull);
  const uint32_t pixel = (uint32_t)(path / P.spp), sample = (uint32_t)(path % P.spp);
  const uint32_t px = pixel % P.width, py = pixel / P.width;
  PathSamplerDev ps;
  ps.init(px, py, sample, P.log2_spp, P.n_base4_digits, P.seed);
  float c0, c1;
  ps.sample_2d(kDimCamera, c0, c1);
  const float fx = ((float)px + 0.5f) + 0.5f * tent(c0);
  const float fy = ((float)py + 0.5f) + 0.5f * tent(c1);
  const V3 d = camera_dir(P.cam, P.width, P.height, fx, fy);
  float* q = B.q_ray[0];
  q[i] = P.cam.eye[0];
  q[C + i] = P.cam.eye[1];
  q[2 * C + i] = P.cam.eye[2];
  q[3 * C + i] = d.x;
  q[4 * C + i] = d.y;
  q[5 * C + i] = d.z;
  q[6 * C + i] = __int_as_float(0x7f800000);
  B.q_slot[0][i] = i;
  if (BATCH) {
    B.job[i] = jb;
    B.q_job[0][i] = jb;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    B.beta[k * C + i] = 1.0f;
    B.L[k * C + i] = ADJ ? primal[3 * (uint64_t)i + k] : 0.0f;
  }
  B.depth[i] = 0;
  B.lock[i] = -1.0f;
  // alpha tests: the camera ray's AuxRng (mis.rs: the initial seed; nee.rs /
  // pt.rs: depth 0's seed)
  if (B.q_aux && (BATCH ? jobs[jb].render.geo.inst_alpha : S0.geo.inst_alpha) != nullptr)
    B.q_aux[i] = aux_from_seed(ps, P.integrator == kIntegMis ? -1 : 0);
}

// One vertex per queue entry of queue `cur`; appends to queue `cur ^ 1` and the shadow queue.
// LIGHTS: the scene (any scene of a batch) has point, spot or directional
// lights (prepare_direct's specialisation).
template <bool ADJ, bool BATCH, int BS, bool LIGHTS>
__global__ void __launch_bounds__(BS, shade_min_blocks<ADJ, BS>()) wf_shade(const __grid_constant__ DevRender S0,
                                                               const __grid_constant__ RenderLaunch P0,
                                                               WfBuffers B, int cur,
                                                               const __grid_constant__ DevAdjoint A,
                                                               const DevJob* __restrict__ jobs) {
  __shared__ float grad_sh[ADJ ? BS * kGradParams : 1];
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= B.counts[cur]) return;
  const uint64_t first_path = (uint64_t)B.counts[4] | ((uint64_t)B.counts[5] << 32);
  const float sgn = ADJ ? -1.0f : 1.0f;  // the adjoint takes collected radiance off R
  uint32_t grad_key = 0xFFFFFFFFu, s_key = 0xFFFFFFFFu;
  float grad_v[ADJ ? kGradParams : 1], s_grad[ADJ ? kGradParams : 1];
  const uint32_t C = B.capacity;
  const uint32_t slot = B.q_slot[cur][j];
  const uint32_t jb = BATCH ? B.job[slot] : 0u;
  const DevRender& S = BATCH ? jobs[jb].render : S0;
  const RenderLaunch& P = BATCH ? jobs[jb].P : P0;
  const uint32_t d = B.depth[slot];
  bool push_next = false, push_shadow = false;
  V3 next_o, next_d;
  DirectPrep dp;
  V3 beta = V3{B.beta[slot], B.beta[C + slot], B.beta[2 * C + slot]};
  V3 L = V3{B.L[slot], B.L[C + slot], B.L[2 * C + slot]};
  // alpha tests (integrator order, see render_kernels.cu): the shadow ray's
  // AuxRng start, the bounce ray's, and whether the bounce continues from the
  // shadow ray's final state (MIS; the resolve stage copies it over)
  const bool alpha = B.q_aux != nullptr && S.geo.inst_alpha != nullptr;
  uint32_t sh_aux = 0, nx_aux = 0, aux_cont = 0;
  const int32_t tri = B.h_tri[j];
  if (tri >= 0) {
    TraceResult h;
    h.tri = tri;
    h.inst = B.h_inst[j];
    h.b0 = B.h_bary[j];
    h.b1 = B.h_bary[C + j];
    h.b2 = B.h_bary[2 * C + j];
    const float* qr = B.q_ray[cur];
    const V3 rd = V3{qr[3 * C + j], qr[4 * C + j], qr[5 * C + j]};
    Vertex v = shade_hit<int>(S, h, rd);
    v.thr = beta;  // the path state of the vertex (mis.rs:54-55)
    v.lock = B.lock[slot];
    const uint32_t mi = __ldg(&S.d.inst[v.inst].material);
    const DevMaterialRec m = S.d.mats[mi];
    // emission of this vertex (mis.rs:45-47 for the camera vertex, 101-117
    // after a bounce; PT counts every hit in full, NEE only from the camera
    // and after delta samples)
    V3 le;
    if (may_emit(m) && material_le(S, m, v, le)) {
      if (d == 0) {
        L = L + sgn * le;
      } else {
        const uint32_t pm = B.prev_mat[slot];
        if ((pm >> 31) || P.integrator == kIntegPt) {
          L = L + sgn * (beta * le);
        } else if (P.integrator == kIntegMis) {
          Vertex pv;
          pv.p = V3{B.prev[slot], B.prev[C + slot], B.prev[2 * C + slot]};
          pv.ns = V3{B.prev[3 * C + slot], B.prev[4 * C + slot], B.prev[5 * C + slot]};
          const float lp = light_pdf_for_hit(S, S.d.mats[pm & 0x7FFFFFFFu], pv, v);
          L = L + sgn * (beta * le * balance_heuristic(B.prev[6 * C + slot], lp));
        }
      }
    }
    if (d < P.max_depth && m.kind != kDevEmissive) {
      const uint64_t path = first_path + slot - (BATCH ? jobs[jb].path_base : 0ull);
      V3 dl = V3{0.0f, 0.0f, 0.0f};
      if (ADJ) {
        const uint64_t di = 3ull * ((uint32_t)(path / P.spp) - A.pixel_base);
        dl = V3{A.d_image[di], A.d_image[di + 1], A.d_image[di + 2]} * A.scale;
      }
      const uint32_t pixel = (uint32_t)(path / P.spp), sample = (uint32_t)(path % P.spp);
      PathSamplerDev ps;
      ps.init(pixel % P.width, pixel / P.width, sample, P.log2_spp, P.n_base4_digits, P.seed);
      if (alpha) {
        if (P.integrator == kIntegMis) {
          sh_aux = nx_aux = aux_from_seed(ps, (int)d);
          aux_cont = 1u;
        } else {
          sh_aux = B.q_aux[slot];  // NEE: after the arriving ray's draws
          nx_aux = aux_from_seed(ps, (int)d + 1);
        }
      }
      float us0, us1;
      ps.sample_2d(vertex_dim(d, kOffSurface), us0, us1);
      const float u_tree = ps.sample_1d(vertex_dim(d, kOffTree));
      // one light-sampler category takes any u: skip drawing it
      const float u_cat = LIGHTS && S.d.num_cat > 1 ? ps.sample_1d(vertex_dim(d, kOffCategory)) : 0.0f;
      // (PT: BSDF sampling only)
      if (P.integrator != kIntegPt &&
          prepare_direct<LIGHTS>(S, m, v, u_cat, u_tree, us0, us1, dp, P.integrator == kIntegNee)) {
        dp.contrib = beta * dp.contrib;
        push_shadow = true;
      }
      BsdfSampleOut s;
      bool sampled_grads = false;
      float sens_s[ADJ ? 3 * kGradGroups : 1];
      if (material_sample(S, m, v, ps, d, s)) {
        beta = beta * s.weight;
        if (s.lock >= 0.0f) B.lock[slot] = s.lock;
        bool alive = true;
        if (d + 1 >= 4) {
          const float q = clampf(max_element(beta), 0.05f, 1.0f);
          if (ps.sample_1d(vertex_dim(d, kOffRr)) > q) alive = false;
          else beta = beta / q;
        }
        if (alive) {
          push_next = true;
          if (ADJ && m.kind == kDevOpenPbr && !s.delta) {
            // R (= L here) still holds this vertex's light sample, if any:
            // resolve corrects for it once the shadow ray is known unoccluded
            openpbr_vertex_sens(S, A, m.openpbr, v, s.wi, sens_s);
            grads_from_sens(sens_s, dl * L, grad_v);
            grad_key = mi;
            sampled_grads = true;
          }
          next_o = offset_origin(v.p, v.ng, s.wi);
          next_d = s.wi;
          B.prev[slot] = v.p.x;
          B.prev[C + slot] = v.p.y;
          B.prev[2 * C + slot] = v.p.z;
          B.prev[3 * C + slot] = v.ns.x;
          B.prev[4 * C + slot] = v.ns.y;
          B.prev[5 * C + slot] = v.ns.z;
          B.prev[6 * C + slot] = s.pdf;
          B.prev_mat[slot] = mi | (s.delta ? 0x80000000u : 0u);
          B.depth[slot] = d + 1;
        }
      }
      if (ADJ && push_shadow && A.s_gkey) {
        s_key = 0xFFFFFFFFu;
        if (m.kind == kDevOpenPbr) {
          float sens_l[3 * kGradGroups], t[kGradParams];
          openpbr_vertex_sens(S, A, m.openpbr, v, dp.wi, sens_l);
          const V3 w = dl * dp.contrib;
          grads_from_sens(sens_l, w, s_grad);
          if (sampled_grads) {
            grads_from_sens(sens_s, w, t);
#pragma unroll
            for (int k = 0; k < (int)kGradParams; ++k) s_grad[k] -= t[k];
          }
          s_key = mi;
        }
      }
    }
  }
  if (LIGHTS && tri < 0 && S.d.has_env) {
    // the ray left the scene: the environment's radiance (mis.rs:33-35,
    // 127-135; PT in full, pt.rs:36-39; NEE from the camera and after delta
    // samples only, nee.rs:37-42)
    const uint32_t pm = d == 0 ? 0u : B.prev_mat[slot];
    const bool full = d == 0 || (pm >> 31) != 0 || P.integrator == kIntegPt;
    if (full || P.integrator == kIntegMis) {
      const float* qr = B.q_ray[cur];
      const V3 rd = V3{qr[3 * C + j], qr[4 * C + j], qr[5 * C + j]};
      const V3 le = env_escape(S.d, rd, full, false, full ? 0.0f : B.prev[6 * C + slot]);
      L = L + sgn * (d == 0 ? le : beta * le);
    }
  }
  B.L[slot] = L.x;
  B.L[C + slot] = L.y;
  B.L[2 * C + slot] = L.z;
  B.beta[slot] = beta.x;
  B.beta[C + slot] = beta.y;
  B.beta[2 * C + slot] = beta.z;
  const int nxt = cur ^ 1;
  const uint32_t qn = warp_append(&B.counts[nxt], push_next);
  const uint32_t qs = warp_append(&B.counts[2], push_shadow);
  if (push_next) {
    float* q = B.q_ray[nxt];
    q[qn] = next_o.x;
    q[C + qn] = next_o.y;
    q[2 * C + qn] = next_o.z;
    q[3 * C + qn] = next_d.x;
    q[4 * C + qn] = next_d.y;
    q[5 * C + qn] = next_d.z;
    q[6 * C + qn] = __int_as_float(0x7f800000);
    B.q_slot[nxt][qn] = slot;
    if (BATCH) B.q_job[nxt][qn] = jb;
    if (alpha) B.q_aux[slot] = nx_aux;
  }
  if (push_shadow) {
    float* q = B.s_ray;
    q[qs] = dp.so.x;
    q[C + qs] = dp.so.y;
    q[2 * C + qs] = dp.so.z;
    q[3 * C + qs] = dp.wi.x;
    q[4 * C + qs] = dp.wi.y;
    q[5 * C + qs] = dp.wi.z;
    q[6 * C + qs] = __int_as_float(0x7f800000);
    B.s_slot[qs] = slot;
    if (BATCH) B.s_job[qs] = jb;
    if (alpha) {
      B.s_aux[qs] = sh_aux;
      B.s_aux_cont[qs] = aux_cont;
    } else if (B.s_aux_cont) {
      B.s_aux_cont[qs] = 0u;  // a batch mixes scenes with and without alpha tests
    }
    B.s_target[qs] = dp.inst;
    B.s_target[C + qs] = dp.tri;
    if (LIGHTS) B.s_dist[qs] = dp.dist;
    B.s_contrib[qs] = dp.contrib.x;
    B.s_contrib[C + qs] = dp.contrib.y;
    B.s_contrib[2 * C + qs] = dp.contrib.z;
    if (ADJ && A.s_gkey) {
      A.s_gkey[qs] = s_key;
      if (s_key != 0xFFFFFFFFu) {
#pragma unroll
        for (int k = 0; k < (int)kGradParams; ++k) A.s_grad[(size_t)k * C + qs] = s_grad[k];
      }
    }
  }
  if (ADJ) warp_accumulate_grads(A.grad, grad_key, grad_v, grad_sh + (threadIdx.x & ~31u) * kGradParams);
}

// unoccluded_ray (integrator/mod.rs:239-265): visible when nothing is hit, the
// first hit is the sampled emitter triangle, or (point and spot lights) the
// first hit lies beyond the light.
template <bool ADJ>
__global__ void __launch_bounds__(kWfBlock) wf_resolve(WfBuffers B, const __grid_constant__ DevAdjoint A) {
  __shared__ float grad_sh[ADJ ? kWfBlock * kGradParams : 1];
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= B.counts[2]) return;
  const uint32_t C = B.capacity;
  // MIS with alpha tests: the bounce ray continues the shadow ray's AuxRng
  if (B.s_aux_cont && B.s_aux_cont[j]) B.q_aux[B.s_slot[j]] = B.s_aux[j];
  const uint32_t tgt_inst = B.s_target[j];
  // the distance plane is written for delta-light shadow rays only
  const bool visible = shadow_visible(B.s_tri[j], B.s_inst[j], B.s_t[j], tgt_inst, B.s_target[C + j],
                                      tgt_inst == 0xFFFFFFFFu ? B.s_dist[j] : 0.0f);
  if (visible) {
    const uint32_t slot = B.s_slot[j];
    const float sgn = ADJ ? -1.0f : 1.0f;
    B.L[slot] = B.L[slot] + sgn * B.s_contrib[j];
    B.L[C + slot] = B.L[C + slot] + sgn * B.s_contrib[C + j];
    B.L[2 * C + slot] = B.L[2 * C + slot] + sgn * B.s_contrib[2 * C + j];
  }
  if (ADJ && A.s_gkey) {
    const uint32_t key = visible ? A.s_gkey[j] : 0xFFFFFFFFu;
    float vals[kGradParams];
#pragma unroll
    for (int k = 0; k < (int)kGradParams; ++k) vals[k] = key != 0xFFFFFFFFu ? A.s_grad[(size_t)k * C + j] : 0.0f;
    warp_accumulate_grads(A.grad, key, vals, grad_sh + (threadIdx.x & ~31u) * kGradParams);
  }
}

__global__ void __launch_bounds__(kWfBlock) wf_finalize(WfBuffers B, uint32_t n_paths, float* samples) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_paths) return;
  const uint32_t C = B.capacity;
  samples[3 * (uint64_t)i] = B.L[i];
  samples[3 * (uint64_t)i + 1] = B.L[C + i];
  samples[3 * (uint64_t)i + 2] = B.L[2 * C + i];
}

static inline unsigned grid_for(uint32_t n) { return (n + kWfBlock - 1) / kWfBlock; }

cudaError_t launch_wf_generate(const DevGeometry& geo, const DevRenderData& rd, const RenderLaunch& P,
                               const WfBuffers& B, uint64_t first_path, uint32_t n_paths, cudaStream_t s,
                               const float* primal) {
  DevRender S{geo, rd};
  if (primal)
    wf_generate<true, false><<<grid_for(std::max(n_paths, 1u)), kWfBlock, 0, s>>>(S, P, B, first_path, n_paths,
                                                                                  primal, nullptr, 0);
  else
    wf_generate<false, false><<<grid_for(std::max(n_paths, 1u)), kWfBlock, 0, s>>>(S, P, B, first_path, n_paths,
                                                                                   nullptr, nullptr, 0);
  return cudaGetLastError();
}

static inline unsigned grid_for_block(uint32_t n, int bs) { return (n + bs - 1) / bs; }

cudaError_t launch_wf_shade(const DevGeometry& geo, const DevRenderData& rd, const RenderLaunch& P,
                            const WfBuffers& B, int cur, cudaStream_t s, const DevAdjoint* A, int block) {
  DevRender S{geo, rd};
  const bool lights = rd.num_extra_lights > 0;
  const DevAdjoint none{};
  if (A)  // one instantiation for the adjoint, with the delta-light paths
    wf_shade<true, false, kWfBlock, true><<<grid_for(B.capacity), kWfBlock, 0, s>>>(S, P, B, cur, *A, nullptr);
  else if (block == 128 && lights)
    wf_shade<false, false, 128, true><<<grid_for_block(B.capacity, 128), 128, 0, s>>>(S, P, B, cur, none, nullptr);
  else if (block == 128)
    wf_shade<false, false, 128, false><<<grid_for_block(B.capacity, 128), 128, 0, s>>>(S, P, B, cur, none, nullptr);
  else if (lights)
    wf_shade<false, false, kWfBlock, true><<<grid_for(B.capacity), kWfBlock, 0, s>>>(S, P, B, cur, none, nullptr);
  else
    wf_shade<false, false, kWfBlock, false><<<grid_for(B.capacity), kWfBlock, 0, s>>>(S, P, B, cur, none, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_wf_generate_batch(const DevJob* jobs, uint32_t n_jobs, const WfBuffers& B, uint64_t first_path,
                                     uint32_t n_paths, cudaStream_t s) {
  wf_generate<false, true><<<grid_for(std::max(n_paths, 1u)), kWfBlock, 0, s>>>(
      DevRender{}, RenderLaunch{}, B, first_path, n_paths, nullptr, jobs, n_jobs);
  return cudaGetLastError();
}

cudaError_t launch_wf_shade_batch(const DevJob* jobs, const WfBuffers& B, int cur, cudaStream_t s, int block,
                                  bool lights) {
  const DevRender S{};
  const RenderLaunch P{};
  const DevAdjoint none{};
  if (block == 128 && lights)
    wf_shade<false, true, 128, true><<<grid_for_block(B.capacity, 128), 128, 0, s>>>(S, P, B, cur, none, jobs);
  else if (block == 128)
    wf_shade<false, true, 128, false><<<grid_for_block(B.capacity, 128), 128, 0, s>>>(S, P, B, cur, none, jobs);
  else if (lights)
    wf_shade<false, true, kWfBlock, true><<<grid_for(B.capacity), kWfBlock, 0, s>>>(S, P, B, cur, none, jobs);
  else
    wf_shade<false, true, kWfBlock, false><<<grid_for(B.capacity), kWfBlock, 0, s>>>(S, P, B, cur, none, jobs);
  return cudaGetLastError();
}

cudaError_t launch_wf_resolve(const WfBuffers& B, cudaStream_t s, const DevAdjoint* A) {
  if (A) wf_resolve<true><<<grid_for(B.capacity), kWfBlock, 0, s>>>(B, *A);
  else wf_resolve<false><<<grid_for(B.capacity), kWfBlock, 0, s>>>(B, DevAdjoint{});
  return cudaGetLastError();
}

cudaError_t launch_wf_finalize(const WfBuffers& B, uint32_t n_paths, float* samples, cudaStream_t s) {
  wf_finalize<<<grid_for(std::max(n_paths, 1u)), kWfBlock, 0, s>>>(B, n_paths, samples);
  return cudaGetLastError();
}

}  // namespace tpt
