// Path-tracing megakernel: one thread per (pixel, sample) path, MIS
// integrator (integrator/mis.rs), then an in-order per-pixel running mean
// (main.rs:107-123) so the accumulated image rounds exactly like the reference.
#include "../api/internal.h"
#include "../device/render.cuh"

namespace tpt {

constexpr int kRenderBlock = 128;
constexpr int kRenderShStack = 32;

__global__ void __launch_bounds__(kRenderBlock) render_mis_kernel(DevRender S, RenderLaunch P,
                                                                  float* __restrict__ samples, uint64_t first_path,
                                                                  uint64_t n_paths, uint32_t* err) {
  __shared__ uint32_t stack_sh[kRenderShStack * kRenderBlock];
  SplitStack<kRenderShStack> st;
  st.sh = stack_sh + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n_paths; k += stride) {
    const uint64_t path = first_path + k;
    const uint32_t pixel = (uint32_t)(path / P.spp);
    const uint32_t sample = (uint32_t)(path % P.spp);
    const uint32_t px = pixel % P.width, py = pixel / P.width;
    PathSamplerDev ps;
    ps.init(px, py, sample, P.log2_spp, P.n_base4_digits);
    float c0, c1;
    ps.sample_2d(kDimCamera, c0, c1);
    // PinholeCamera::generate_ray_differential (camera.rs:48-73), primary direction only
    const float fx = ((float)px + 0.5f) + 0.5f * tent(c0);
    const float fy = ((float)py + 0.5f) + 0.5f * tent(c1);
    const V3 d = camera_dir(P.cam, P.width, P.height, fx, fy);
    const V3 o = V3{P.cam.eye[0], P.cam.eye[1], P.cam.eye[2]};
    const V3 L = trace_mis(S, st, P, ps, o, d, err);
    samples[3 * k + 0] = L.x;
    samples[3 * k + 1] = L.y;
    samples[3 * k + 2] = L.z;
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
                          uint64_t first_path, uint64_t n_paths, uint32_t* err, int num_sms, cudaStream_t s) {
  if (n_paths == 0) return cudaSuccess;
  if (P.integrator == TPT_INTEGRATOR_BDPT)
    return launch_render_bdpt(geo, rd, P, samples, first_path, n_paths, err, num_sms, s);
  DevRender S;
  S.geo = geo;
  S.d = rd;
  static int blocks_per_sm = 0;
  if (blocks_per_sm == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, render_mis_kernel, kRenderBlock, 0) !=
            cudaSuccess ||
        blocks_per_sm <= 0)
      blocks_per_sm = 2;
  }
  uint64_t blocks = (n_paths + kRenderBlock - 1) / kRenderBlock;
  const uint64_t cap = (uint64_t)num_sms * blocks_per_sm * 8;
  if (blocks > cap) blocks = cap;
  render_mis_kernel<<<(unsigned)blocks, kRenderBlock, 0, s>>>(S, P, samples, first_path, n_paths, err);
  return cudaGetLastError();
}

cudaError_t launch_accumulate(const float* samples, uint32_t spp, uint32_t first_pixel, uint32_t n_pixels,
                              float exposure, float* image, cudaStream_t s) {
  if (n_pixels == 0) return cudaSuccess;
  accumulate_kernel<<<(n_pixels + 255) / 256, 256, 0, s>>>(samples, spp, first_pixel, n_pixels, exposure, image);
  return cudaGetLastError();
}

}  // namespace tpt
