// Batched OpenPBR BSDF queries of one material of an uploaded scene, in the
// shading frame: eval + pdf for direction pairs, and sample.  They expose the
// device BSDF the renderers use to unit-level parity tests and benchmarks.
#include "../api/internal.h"
#include "../device/openpbr.cuh"

namespace tpt {

namespace {
constexpr int kQueryBlock = 128;

__global__ void __launch_bounds__(kQueryBlock) bsdf_eval_kernel(const __grid_constant__ DevRenderData rd, uint32_t material, uint64_t n,
                                                                const float* __restrict__ wo,
                                                                const float* __restrict__ wi,
                                                                const uint32_t* __restrict__ front, uint32_t mode,
                                                                const float* __restrict__ state,
                                                                float* __restrict__ f, float* __restrict__ pdf) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DevOpenPbr* m = rd.openpbr + rd.mats[material].openpbr;
  opbr::OpbrVertex s;
  const V3 o = V3{wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]};
  const V3 w = V3{wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]};
  opbr::init_vertex(s, m, rd.cec_e, rd.dec_e, o, front[i] != 0, fabsf(o.z));
  if (state) {  // path throughput and wavelength lock (NaN: none)
    s.thr = V3{state[4 * i], state[4 * i + 1], state[4 * i + 2]};
    s.lock = isnan(state[4 * i + 3]) ? -1.0f : state[4 * i + 3];
  }
  V3 fv;
  float p;
  if (mode == 1) {  // importance transport: layer weights at wi
    opbr::OpbrVertex lay;
    opbr::init_vertex(lay, m, rd.cec_e, rd.dec_e, w, front[i] != 0, fabsf(o.z));
    lay.thr = s.thr;
    lay.lock = s.lock;
    opbr::eval_pdf(s, lay, w, fv, p, true, true);
  } else {
    opbr::eval_pdf(s, s, w, fv, p);
  }
  f[3 * i] = fv.x;
  f[3 * i + 1] = fv.y;
  f[3 * i + 2] = fv.z;
  pdf[i] = p;
}

__global__ void __launch_bounds__(kQueryBlock) bsdf_sample_kernel(const __grid_constant__ DevRenderData rd, uint32_t material, uint64_t n,
                                                                  const float* __restrict__ wo,
                                                                  const float* __restrict__ u,
                                                                  const uint32_t* __restrict__ front, uint32_t mode,
                                                                  const float* __restrict__ state,
                                                                  float* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DevOpenPbr* m = rd.openpbr + rd.mats[material].openpbr;
  opbr::OpbrVertex s;
  const V3 w = V3{wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]};
  opbr::init_vertex(s, m, rd.cec_e, rd.dec_e, w, front[i] != 0, fabsf(w.z));
  // with a path state: u holds 7 values (u_lobe, u_dir, u_extra0..3) and the
  // record 10 (the sampled wavelength lock last, NaN: none)
  const int nu = state ? 7 : 3, no = state ? 10 : 9;
  float ux[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  if (state) {
    s.thr = V3{state[4 * i], state[4 * i + 1], state[4 * i + 2]};
    s.lock = isnan(state[4 * i + 3]) ? -1.0f : state[4 * i + 3];
    for (int k = 0; k < 4; ++k) ux[k] = u[nu * i + 3 + k];
  }
  opbr::Sample smp;
  float* o = out + no * i;
  if (!opbr::sample(s, u[nu * i], u[nu * i + 1], u[nu * i + 2], smp, mode == 1, true, ux)) {
    for (int k = 0; k < no; ++k) o[k] = 0.0f;
    return;
  }
  if (state) o[9] = smp.lock >= 0.0f ? smp.lock : __int_as_float(0x7fc00000);
  o[0] = smp.weight.x;
  o[1] = smp.weight.y;
  o[2] = smp.weight.z;
  o[3] = smp.wi.x;
  o[4] = smp.wi.y;
  o[5] = smp.wi.z;
  o[6] = smp.pdf;
  o[7] = smp.pdf_rev;
  o[8] = __uint_as_float(smp.flags);
}
}  // namespace

cudaError_t launch_bsdf_eval(const DevRenderData& rd, uint32_t material, uint64_t n, const float* wo, const float* wi,
                             const uint32_t* front, uint32_t mode, const float* state, float* f, float* pdf,
                             cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  bsdf_eval_kernel<<<(unsigned)((n + kQueryBlock - 1) / kQueryBlock), kQueryBlock, 0, s>>>(rd, material, n, wo, wi,
                                                                                          front, mode, state, f, pdf);
  return cudaGetLastError();
}

cudaError_t launch_bsdf_sample(const DevRenderData& rd, uint32_t material, uint64_t n, const float* wo,
                               const float* u, const uint32_t* front, uint32_t mode, const float* state, float* out,
                               cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  bsdf_sample_kernel<<<(unsigned)((n + kQueryBlock - 1) / kQueryBlock), kQueryBlock, 0, s>>>(rd, material, n, wo, u,
                                                                                            front, mode, state, out);
  return cudaGetLastError();
}

}  // namespace tpt
