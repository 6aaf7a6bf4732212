// Path-tracing megakernel: one thread carries one (pixel, sample) path at a
// time through the MIS integrator (integrator/mis.rs), then an in-order
// per-pixel running mean (main.rs:107-123) so the accumulated image rounds
// exactly like the reference.
//
// The kernel is persistent and phase-synchronous: every iteration of its loop
// traces exactly one ray per lane (the camera ray, a bounce ray or an NEE
// shadow ray) at a single traversal call site, then advances each lane's path
// by one step; a lane whose path ends writes its radiance and takes the next
// path from a global counter (one warp-aggregated atomic).  Lanes of a warp
// thus run the same code region at the same time whatever their path depth,
// which keeps the instruction cache warm and the SIMT lanes busy.  Radiance is
// accumulated in the reference's order (emission of vertex d, its NEE, then
// emission of vertex d + 1), so results equal the wavefront execution's bit
// for bit.
//
// Alpha tests draw from the path's AuxRng in the order of the integrator
// (mis.rs: the camera ray from the initial seed, then per vertex its seed for
// the light sample's shadow ray and the bounce ray after it; nee.rs / pt.rs:
// each depth's seed for the ray arriving there and, NEE, the light sample of
// that vertex).
#include "../api/internal.h"
#include "../device/render.cuh"

namespace tpt {

constexpr int kRenderBlock = 128;
constexpr int kRenderShStack = 32;
#ifndef TPT_MK_MINB
#define TPT_MK_MINB 4  // 128 registers: 4 blocks (16 warps) per SM, a few bytes of spill
#endif

namespace {
enum : uint32_t { kRayNone = 0, kRayBounce = 1, kRayShadow = 2 };
}

// LIGHTS: the scene has point, spot or directional lights (prepare_direct's specialisation).
template <bool LIGHTS>
__global__ void __launch_bounds__(kRenderBlock, TPT_MK_MINB) render_mis_kernel(const __grid_constant__ DevRender S,
                                                                  const __grid_constant__ RenderLaunch P,
                                                                  float* __restrict__ samples, uint64_t first_path,
                                                                  uint64_t n_paths,
                                                                  unsigned long long* __restrict__ counter,
                                                                  uint32_t* err) {
  __shared__ uint32_t stack_sh[kRenderShStack * kRenderBlock];
  SplitStack<kRenderShStack> st;
  st.sh = stack_sh + threadIdx.x;
  const unsigned lane = threadIdx.x & 31u;
  int64_t k = -1;  // path (relative to first_path); -1: needs one, -2: none left
  uint32_t kind = kRayNone, depth = 0;
  V3 ro, rd;                   // the ray to trace next
  V3 bo, bd;                   // bounce ray waiting behind a shadow ray
  bool bounce_pending = false;
  V3 L, beta, contrib;         // contrib: NEE radiance counted if the shadow ray is clear
  uint32_t tgt_inst = 0, tgt_tri = 0;
  float tgt_dist = 0.0f;
  V3 prev_p, prev_ns;          // previous vertex (emission MIS after a BSDF sample)
  float prev_pdf = 0.0f;
  uint32_t prev_mat = 0;       // material index, bit 31: delta sample
  float lock = -1.0f;          // the path's wavelength lock (< 0: none)
  uint32_t aux = 0, bounce_aux = 0;  // AuxRng state; the state the pending bounce ray starts from (NEE, PT)
  const bool alpha = S.geo.inst_alpha != nullptr;
  PathSamplerDev ps;
  for (;;) {
    const unsigned need = __ballot_sync(0xffffffffu, k == -1);
    if (need) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if ((int)lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (k == -1) {
        const uint64_t i = base + __popc(need & ((1u << lane) - 1u));
        if (i < n_paths) {
          k = (int64_t)i;
          const uint64_t path = first_path + i;
          const uint32_t pixel = (uint32_t)(path / P.spp), sample = (uint32_t)(path % P.spp);
          const uint32_t px = pixel % P.width, py = pixel / P.width;
          ps.init(px, py, sample, P.log2_spp, P.n_base4_digits, P.seed);
          float c0, c1;
          ps.sample_2d(kDimCamera, c0, c1);
          // PinholeCamera::generate_ray_differential (camera.rs:48-73), primary direction only
          const float fx = ((float)px + 0.5f) + 0.5f * tent(c0);
          const float fy = ((float)py + 0.5f) + 0.5f * tent(c1);
          rd = camera_dir(P.cam, P.width, P.height, fx, fy);
          ro = V3{P.cam.eye[0], P.cam.eye[1], P.cam.eye[2]};
          kind = kRayBounce;
          depth = 0;
          L = V3{0.0f, 0.0f, 0.0f};
          beta = V3{1.0f, 1.0f, 1.0f};
          lock = -1.0f;
          if (alpha) aux = aux_from_seed(ps, P.integrator == kIntegMis ? -1 : 0);
          bounce_pending = false;
        } else {
          k = -2;
        }
      }
    }
    if (__all_sync(0xffffffffu, k == -2)) break;
    const unsigned act = __ballot_sync(0xffffffffu, k >= 0);
    if (k < 0) continue;
    TraceResult h;
    trace_ray_ww<0>(S.geo, st, act, ro.x, ro.y, ro.z, rd.x, rd.y, rd.z, __int_as_float(0x7f800000), h, err,
                    alpha ? &aux : nullptr);
    bool done = false;
    if (kind == kRayShadow) {
      // unoccluded_ray (integrator/mod.rs:239-265)
      if (shadow_visible(h.tri, h.inst, h.t, tgt_inst, tgt_tri, tgt_dist)) L = L + contrib;
      if (bounce_pending) {
        ro = bo;
        rd = bd;
        if (alpha && P.integrator != kIntegMis) aux = bounce_aux;  // MIS continues after the shadow ray
        kind = kRayBounce;
        bounce_pending = false;
      } else {
        done = true;
      }
    } else if (h.tri < 0) {
      // the ray left the scene: the environment's radiance (mis.rs:33-35, 127-135)
      // (PT in full, NEE from the camera and after delta samples only)
      const bool full = depth == 0 || (prev_mat >> 31) != 0 || P.integrator == kIntegPt;
      if (LIGHTS && S.d.has_env && (full || P.integrator == kIntegMis)) {
        const V3 le = env_escape(S.d, rd, full, false, full ? 0.0f : prev_pdf);
        L = L + (depth == 0 ? le : beta * le);
      }
      done = true;
    } else {
      Vertex v = shade_hit<int>(S, h, rd);
      v.thr = beta;  // the path state of the vertex (mis.rs:54-55)
      v.lock = lock;
      const uint32_t mi = __ldg(&S.d.inst[v.inst].material);
      const DevMaterialRec m = S.d.mats[mi];
      V3 le;
      if (may_emit(m) && material_le(S, m, v, le)) {
        if (depth == 0) {
          L = L + le;
        } else if ((prev_mat >> 31) || P.integrator == kIntegPt) {
          L = L + beta * le;
        } else if (P.integrator == kIntegMis) {
          Vertex pv;
          pv.p = prev_p;
          pv.ns = prev_ns;
          const float lp = light_pdf_for_hit(S, S.d.mats[prev_mat & 0x7FFFFFFFu], pv, v);
          L = L + beta * le * balance_heuristic(prev_pdf, lp);
        }
      }
      if (depth >= P.max_depth || m.kind == kDevEmissive) {
        done = true;  // pure emitter: no NEE, and sample() is None
      } else {
        if (alpha && P.integrator == kIntegMis) aux = aux_from_seed(ps, (int)depth);
        float us0, us1;
        ps.sample_2d(vertex_dim(depth, kOffSurface), us0, us1);
        const float u_tree = ps.sample_1d(vertex_dim(depth, kOffTree));
        const float u_cat = LIGHTS && S.d.num_cat > 1 ? ps.sample_1d(vertex_dim(depth, kOffCategory)) : 0.0f;
        DirectPrep dp;
        const bool nee = P.integrator != kIntegPt &&  // PT: BSDF sampling only
                         prepare_direct<LIGHTS>(S, m, v, u_cat, u_tree, us0, us1, dp, P.integrator == kIntegNee);
        if (nee) {
          contrib = beta * dp.contrib;
          tgt_inst = dp.inst;
          tgt_tri = dp.tri;
          if (LIGHTS) tgt_dist = dp.dist;
        }
        bool alive = false;
        BsdfSampleOut s;
        if (material_sample(S, m, v, ps, depth, s)) {
          beta = beta * s.weight;
          if (s.lock >= 0.0f) lock = s.lock;
          alive = true;
          if (depth + 1 >= 4) {
            const float q = clampf(max_element(beta), 0.05f, 1.0f);
            if (ps.sample_1d(vertex_dim(depth, kOffRr)) > q) alive = false;
            else beta = beta / q;
          }
          if (alive) {
            bo = offset_origin(v.p, v.ng, s.wi);
            bd = s.wi;
            prev_p = v.p;
            prev_ns = v.ns;
            prev_pdf = s.pdf;
            prev_mat = mi | (s.delta ? 0x80000000u : 0u);
            depth = depth + 1;
            if (alpha && P.integrator != kIntegMis) bounce_aux = aux_from_seed(ps, (int)depth);
          }
        }
        if (nee) {
          ro = dp.so;
          rd = dp.wi;
          kind = kRayShadow;
          bounce_pending = alive;
        } else if (alive) {
          ro = bo;
          rd = bd;
          kind = kRayBounce;
          if (alpha && P.integrator != kIntegMis) aux = bounce_aux;
        } else {
          done = true;
        }
      }
    }
    if (done) {
      samples[3 * k + 0] = L.x;
      samples[3 * k + 1] = L.y;
      samples[3 * k + 2] = L.z;
      k = -1;
    }
  }
}

// color += (sample - color) / (i + 1), in sample order; then * exposure.
__global__ void accumulate_kernel(const float* __restrict__ samples, uint32_t spp, uint32_t first_pixel,
                                  uint32_t n_pixels, float exposure, float* __restrict__ image) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_pixels) return;
  const float* s = samples + 3ull * spp * i;
  float r = 0.0f, g = 0.0f, b = 0.0f;
  for (uint32_t k = 0; k < spp; ++k) {
    const float n = (float)(k + 1);
    r = r + (s[3 * k + 0] - r) / n;
    g = g + (s[3 * k + 1] - g) / n;
    b = b + (s[3 * k + 2] - b) / n;
  }
  float* o = image + 3ull * (first_pixel + i);
  o[0] = r * exposure;
  o[1] = g * exposure;
  o[2] = b * exposure;
}

cudaError_t launch_render(const DevGeometry& geo, const DevRenderData& rd, const RenderLaunch& P, float* samples,
                          uint64_t first_path, uint64_t n_paths, uint32_t* err, int num_sms, cudaStream_t s,
                          unsigned long long* counter) {
  if (n_paths == 0) return cudaSuccess;
  if (P.integrator == TPT_INTEGRATOR_BDPT)
    return launch_render_bdpt(geo, rd, P, samples, first_path, n_paths, err, num_sms, s);
  DevRender S;
  S.geo = geo;
  S.d = rd;
  const bool lights = rd.num_extra_lights > 0;
  static int blocks_per_sm[2] = {0, 0};
  int& bps = blocks_per_sm[lights ? 1 : 0];
  if (bps == 0) {
    const cudaError_t q =
        lights ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, render_mis_kernel<true>, kRenderBlock, 0)
               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, render_mis_kernel<false>, kRenderBlock, 0);
    if (q != cudaSuccess || bps <= 0) bps = 2;
  }
  uint64_t blocks = (n_paths + kRenderBlock - 1) / kRenderBlock;
  const uint64_t cap = (uint64_t)num_sms * bps;  // persistent: one wave
  if (blocks > cap) blocks = cap;
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  if (lights)
    render_mis_kernel<true><<<(unsigned)blocks, kRenderBlock, 0, s>>>(S, P, samples, first_path, n_paths, counter,
                                                                      err);
  else
    render_mis_kernel<false><<<(unsigned)blocks, kRenderBlock, 0, s>>>(S, P, samples, first_path, n_paths, counter,
                                                                       err);
  return cudaGetLastError();
}

cudaError_t launch_accumulate(const float* samples, uint32_t spp, uint32_t first_pixel, uint32_t n_pixels,
                              float exposure, float* image, cudaStream_t s) {
  if (n_pixels == 0) return cudaSuccess;
  accumulate_kernel<<<(n_pixels + 255) / 256, 256, 0, s>>>(samples, spp, first_pixel, n_pixels, exposure, image);
  return cudaGetLastError();
}

}  // namespace tpt
