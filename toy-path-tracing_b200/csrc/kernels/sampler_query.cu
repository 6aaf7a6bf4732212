// tpt_sampler_values_device: the device's per-pixel sample streams, value for
// value, so that the integer-exact restatement of sampler/{zsobol,pcg,
// path_sampler}.rs that every render kernel uses can be compared with the
// reference's directly rather than through rendered radiance.
//
// One thread per query (px, py, sample, depth): PathSampler::new
// (path_sampler.rs:81-95) with the image's IndexSampler (zsobol.rs:213-224),
// then camera_sample (dimension 0), initial_aux_rng_seed (dimension
// 0x80000000) and path_vertex_randoms(depth) (path_sampler.rs:97-118: the 11
// values at 2 + 16 depth + {0..13} and the aux seed at + 14) -- the same
// PathSamplerDev calls, with the same dimension numbers, that the render
// kernels make.
#include <algorithm>

#include "../api/internal.h"
#include "../device/sampler.cuh"

namespace tpt {
namespace {

constexpr int kQueryBlock = 256;

__global__ void sampler_values_kernel(uint32_t log2_spp, uint32_t n_digits, uint64_t n,
                                      const uint4* __restrict__ queries, float* __restrict__ out,
                                      uint32_t* __restrict__ seeds) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint4 q = queries[i];  // px, py, sample, depth
  PathSamplerDev ps;
  ps.init(q.x, q.y, q.z, log2_spp, n_digits);
  float v[16];
  ps.sample_2d(kDimCamera, v[0], v[1]);
  const uint32_t d = q.w;
  v[2] = ps.sample_1d(vertex_dim(d, kOffCategory));
  v[3] = ps.sample_1d(vertex_dim(d, kOffTree));
  v[4] = ps.sample_1d(vertex_dim(d, kOffLightAux));
  ps.sample_2d(vertex_dim(d, kOffSurface), v[5], v[6]);
  v[7] = ps.sample_1d(vertex_dim(d, kOffLobe));
  v[8] = ps.sample_1d(vertex_dim(d, kOffLayer));
  ps.sample_2d(vertex_dim(d, kOffDir), v[9], v[10]);
  v[11] = ps.sample_1d(vertex_dim(d, kOffExtra0));
  v[12] = ps.sample_1d(vertex_dim(d, kOffExtra1));
  v[13] = ps.sample_1d(vertex_dim(d, kOffExtra2));
  v[14] = ps.sample_1d(vertex_dim(d, kOffExtra3));
  v[15] = ps.sample_1d(vertex_dim(d, kOffRr));
#pragma unroll
  for (int k = 0; k < 16; ++k) out[16 * i + k] = v[k];
  seeds[2 * i] = ps.aux_rng_seed(0x80000000u);
  seeds[2 * i + 1] = ps.aux_rng_seed(vertex_dim(d, kOffAuxSeed));
}

uint32_t pow2_at_least(uint32_t v) {
  uint32_t p = 1;
  while (p < v && p < 0x80000000u) p <<= 1;
  return p;
}
uint32_t log2_of(uint32_t p) {
  uint32_t k = 0;
  while ((1u << k) < p) ++k;
  return k;
}

}  // namespace
}  // namespace tpt

using namespace tpt;

extern "C" tpt_status tpt_sampler_values_device(tpt_context* ctx, uint32_t width, uint32_t height, uint32_t spp,
                                                uint64_t n, const uint32_t* queries, float* out, uint32_t* seeds,
                                                void* stream) {
  if (!ctx) return set_error(nullptr, TPT_ERR_INVALID_ARG, "NULL context");
  if (width == 0 || height == 0 || spp == 0) return set_error(ctx, TPT_ERR_INVALID_ARG, "empty image or spp 0");
  if (spp > (1u << 24)) return set_error(ctx, TPT_ERR_INVALID_ARG, "spp above 2^24");
  if (n && (!queries || !out || !seeds)) return set_error(ctx, TPT_ERR_INVALID_ARG, "NULL buffer");
  if ((uintptr_t)queries % 16) return set_error(ctx, TPT_ERR_INVALID_ARG, "queries must be 16-byte aligned");
  // IndexSampler::new (zsobol.rs:213-224), as the render launches derive it
  const uint32_t log2_spp = log2_of(pow2_at_least(spp));
  const uint32_t n_digits = log2_of(pow2_at_least(std::max(width, height))) + (log2_spp + 1) / 2;
  if (2 * n_digits + 2 > 64) return set_error(ctx, TPT_ERR_CAPACITY, "resolution x spp beyond 64-bit Morton index");
  tpt_status st = set_device(ctx);
  if (st || n == 0) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  const uint64_t blocks = (n + kQueryBlock - 1) / kQueryBlock;
  if (blocks > 0x7FFFFFFFull) return set_error(ctx, TPT_ERR_INVALID_ARG, "too many queries");
  sampler_values_kernel<<<(unsigned)blocks, kQueryBlock, 0, s>>>(log2_spp, n_digits, n, (const uint4*)queries, out,
                                                                  seeds);
  return cuda_check(ctx, cudaGetLastError(), "sampler query launch");
}
