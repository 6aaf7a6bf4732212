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

// Per-channel sensitivities of one rough OpenPBR vertex at the pair (wo, wi):
// sens[3 * g + c] = (df_c / dtheta_g) / f_c for parameter group g (for the
// base colour, channel c's own parameter), zero where the group is masked off
// or f_c = 0.  A contribution C that scales with f_c adds C_c * sens[3g + c]
// to the group's gradient.
static __device__ __noinline__ void openpbr_vertex_sens(const DevRender& S, const DevAdjoint& A,
                                                         uint32_t opbr_index, const Vertex& v, V3 wi,
                                                         float* sens) {
#pragma unroll
  for (int k = 0; k < 3 * (int)kGradGroups; ++k) sens[k] = 0.0f;
  const V3 wo_l = normalize_or_zero(to_local(v.frame, v.wo));
  const V3 wi_l = normalize_or_zero(to_local(v.frame, wi));
  opbr::OpbrVertex base;
  opbr::init_vertex(base, S.d.openpbr + opbr_index, S.d.cec_e, S.d.dec_e, wo_l, v.front, fabsf(wo_l.z));
  V3 f0;
  float pdf0;
  opbr::eval_pdf(base, base, wi_l, f0, pdf0, false);
  const float f0c[3] = {f0.x, f0.y, f0.z};
  for (int g = 0; g < (int)kGradGroups; ++g) {
    if (!(A.mask & (1u << g))) continue;
    const DevOpenPbr* lo = A.pert + ((size_t)opbr_index * kGradGroups + g) * 2;
    const float* span = A.span + ((size_t)opbr_index * kGradGroups + g) * 3;
    const bool reuse = (g == 0 || g == 2);
    const V3 fp = perturbed_f(base, lo + 1, reuse, wo_l, wi_l, v.front);
    const V3 fm = perturbed_f(base, lo, reuse, wo_l, wi_l, v.front);
    const float df[3] = {fp.x - fm.x, fp.y - fm.y, fp.z - fm.z};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float sp = g == 0 ? span[c] : span[0];
      if (f0c[c] > 0.0f && sp > 0.0f) sens[3 * g + c] = (df[c] / sp) / f0c[c];
    }
  }
}

// Gradient slots of a contribution w (per channel, dLoss/dL already applied)
// with sensitivities sens: out[kGradParams] = base colour r, g, b, then one
// slot per further group.
__device__ __forceinline__ void grads_from_sens(const float* sens, V3 w, float* out) {
  const float wc[3] = {w.x, w.y, w.z};
#pragma unroll
  for (int c = 0; c < 3; ++c) out[c] = wc[c] * sens[c];
#pragma unroll
  for (int g = 1; g < (int)kGradGroups; ++g) out[g + 2] = wc[0] * sens[3 * g] + wc[1] * sens[3 * g + 1] +
                                                         wc[2] * sens[3 * g + 2];
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
