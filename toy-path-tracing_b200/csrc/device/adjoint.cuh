// Path-replay adjoint on the device: the per-vertex gradient of the OpenPBR
// BSDF value with respect to the material parameters, and the warp-aggregated
// FP64 accumulation into per-material gradients.
//
// No counterpart in the reference (its renderer is not differentiable).  With
// detached sampling the sample weight f cos / pdf of vertex i changes only
// through f, so dL/dtheta = sum_i R_i * (df_i/dtheta) / f_i, R_i being the
// radiance the path collects after vertex i.  df/dtheta is a central
// difference of the closed-form BSDF at the fixed (wo, wi) pair between two
// host-lowered copies of the material (theta - h, theta + h, clipped to the
// parameter range; the divisor is the clipped span).  The three base-colour
// channels are perturbed together: channel c of f depends on base_color[c]
// only, so one pair of evaluations gives all three partials.
#pragma once
#include "openpbr.cuh"
#include "render.cuh"

namespace tpt {

// f of material `rec` at the pair (wo_l, wi_l) of `base`'s vertex.  Base colour
// and metalness only enter the layer weights (evaluated inside eval_pdf), so
// for those groups the per-vertex state of the unperturbed material is reused
// when the lowering flags agree and the coat darkening (which reads the base
// albedo) is off; every other case rebuilds the state.
__device__ __forceinline__ V3 perturbed_f(const opbr::OpbrVertex& base, const DevOpenPbr* rec, bool reuse_state,
                                          V3 wo_l, V3 wi_l, bool front) {
  opbr::OpbrVertex s;
  if (reuse_state && rec->flags == base.m->flags && !(rec->flags & kOpbrDarkening)) {
    s = base;
    s.m = rec;
  } else {
    opbr::init_vertex(s, rec, base.cec_e, base.dec_e, wo_l, front, base.dk_cos);
  }
  V3 f;
  float pdf;
  opbr::eval_pdf(s, s, wi_l, f, pdf, false);
  return f;
}

// Gradient contributions of one rough OpenPBR vertex: w = dLoss/dL (per
// channel) * R, out[kGradParams] (zeros where the group is masked off).
static __device__ __noinline__ void openpbr_vertex_grads(const DevRender& S, const DevAdjoint& A,
                                                          uint32_t opbr_index, const Vertex& v, V3 wi, V3 w,
                                                          float* out) {
#pragma unroll
  for (int k = 0; k < (int)kGradParams; ++k) out[k] = 0.0f;
  const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
  const V3 wi_l = normalize_or_zero(to_local(v.frame, wi));
  opbr::OpbrVertex base;
  opbr::init_vertex(base, S.d.openpbr + opbr_index, S.d.cec_e, S.d.dec_e, wo_l, v.front, fabsf(wo_l.z));
  V3 f0;
  float pdf0;
  opbr::eval_pdf(base, base, wi_l, f0, pdf0, false);
  const float f0c[3] = {f0.x, f0.y, f0.z};
  const float wc[3] = {w.x, w.y, w.z};
  const int slot[kGradGroups] = {0, 3, 4, 5, 6};
  for (int g = 0; g < (int)kGradGroups; ++g) {
    if (!(A.mask & (1u << g))) continue;
    const DevOpenPbr* lo = A.pert + ((size_t)opbr_index * kGradGroups + g) * 2;
    const float* span = A.span + ((size_t)opbr_index * kGradGroups + g) * 3;
    const bool reuse = (g == 0 || g == 2);
    const V3 fp = perturbed_f(base, lo + 1, reuse, wo_l, wi_l, v.front);
    const V3 fm = perturbed_f(base, lo, reuse, wo_l, wi_l, v.front);
    const float df[3] = {fp.x - fm.x, fp.y - fm.y, fp.z - fm.z};
    if (g == 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (f0c[c] > 0.0f && span[c] > 0.0f) out[c] = wc[c] * (df[c] / span[c]) / f0c[c];
    } else if (span[0] > 0.0f) {
      float acc = 0.0f;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (f0c[c] > 0.0f) acc += wc[c] * (df[c] / span[0]) / f0c[c];
      out[slot[g]] = acc;
    }
  }
}

// Adds each lane's kGradParams values to grad[key * kGradParams + k] in FP64:
// lanes with the same key are summed by their lowest lane, which issues one
// atomic per non-zero parameter.  Every lane of the warp that is still running
// must call this (key 0xFFFFFFFF = nothing to add); `sh` is this warp's
// 32 x kGradParams scratch in shared memory.
__device__ __forceinline__ void warp_accumulate_grads(double* grad, uint32_t key, const float* vals, float* sh) {
  const unsigned act = __activemask();
  const unsigned lane = threadIdx.x & 31u;
  const unsigned peers = __match_any_sync(act, key);
#pragma unroll
  for (int k = 0; k < (int)kGradParams; ++k) sh[lane * kGradParams + k] = vals[k];
  __syncwarp(act);
  if (key != 0xFFFFFFFFu && (int)lane == __ffs(peers) - 1) {
#pragma unroll 1
    for (int k = 0; k < (int)kGradParams; ++k) {
      double acc = 0.0;
      for (unsigned m = peers; m; m &= m - 1) acc += (double)sh[(__ffs(m) - 1) * kGradParams + k];
      if (acc != 0.0) atomicAdd(grad + (size_t)key * kGradParams + k, acc);
    }
  }
  __syncwarp(act);
}

}  // namespace tpt
