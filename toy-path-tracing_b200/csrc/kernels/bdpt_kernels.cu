// BDPT kernel: one thread per (pixel, sample), integrator/bdpt.rs, the lanes of
// a warp stepping through their subpaths and connections together (see
// trace_bdpt).  The per-pixel running mean is the shared accumulate kernel.
#include "../api/internal.h"
#include "../device/bdpt.cuh"

namespace tpt {

constexpr int kBdptBlock = 128;
constexpr int kBdptShStack = 32;

__global__ void __launch_bounds__(kBdptBlock) render_bdpt_kernel(const __grid_constant__ DevRender S,
                                                            const __grid_constant__ RenderLaunch P,
                                                                 float* __restrict__ samples, uint64_t first_path,
                                                                 uint64_t n_paths, uint32_t* err) {
  __shared__ uint32_t stack_sh[kBdptShStack * kBdptBlock];
  SplitStack<kBdptShStack> st;
  st.sh = stack_sh + threadIdx.x;
  // warp-uniform loop: the lanes of a warp take consecutive samples together
  // (trace_bdpt is warp-synchronous); lanes past the end carry no sample
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const unsigned lane = threadIdx.x & 31u;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x - lane); base < n_paths; base += stride) {
    const uint64_t k = base + lane;
    const bool valid = k < n_paths;
    const uint64_t path = first_path + (valid ? k : 0);
    const uint32_t pixel = (uint32_t)(path / P.spp);
    const uint32_t sample = (uint32_t)(path % P.spp);
    const uint32_t px = pixel % P.width, py = pixel / P.width;
    PathSamplerDev ps;
    ps.init(px, py, sample, P.log2_spp, P.n_base4_digits, P.seed);
    float c0, c1;
    ps.sample_2d(kDimCamera, c0, c1);
    const float fx = ((float)px + 0.5f) + 0.5f * tent(c0);
    const float fy = ((float)py + 0.5f) + 0.5f * tent(c1);
    const V3 d = camera_dir(P.cam, P.width, P.height, fx, fy);
    const V3 o = V3{P.cam.eye[0], P.cam.eye[1], P.cam.eye[2]};
    const V3 L = trace_bdpt(S, st, valid, P, ps, o, d, err);
    if (valid) {
      samples[3 * k + 0] = L.x;
      samples[3 * k + 1] = L.y;
      samples[3 * k + 2] = L.z;
    }
  }
}

cudaError_t launch_render_bdpt(const DevGeometry& geo, const DevRenderData& rd, const RenderLaunch& P, float* samples,
                               uint64_t first_path, uint64_t n_paths, uint32_t* err, int num_sms, cudaStream_t s) {
  if (n_paths == 0) return cudaSuccess;
  DevRender S;
  S.geo = geo;
  S.d = rd;
  static int blocks_per_sm = 0;
  if (blocks_per_sm == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, render_bdpt_kernel, kBdptBlock, 0) !=
            cudaSuccess ||
        blocks_per_sm <= 0)
      blocks_per_sm = 2;
  }
  uint64_t blocks = (n_paths + kBdptBlock - 1) / kBdptBlock;
  const uint64_t cap = (uint64_t)num_sms * blocks_per_sm * 8;
  if (blocks > cap) blocks = cap;
  render_bdpt_kernel<<<(unsigned)blocks, kBdptBlock, 0, s>>>(S, P, samples, first_path, n_paths, err);
  return cudaGetLastError();
}

}  // namespace tpt
