// Batch ray-query kernels: `Scene::closest_hit` over a structure-of-arrays
// ray batch (scene/mod.rs:340-395), plus the any-hit occlusion variant.
#include "../api/internal.h"
#include "../device/trace.cuh"

namespace tpt {

template <int MODE, bool STATS, bool BARY>
__global__ void __launch_bounds__(128) traverse_kernel(DevGeometry geo, const float* __restrict__ rays, uint64_t rs, uint64_t n,
                                                       uint64_t bs, int32_t* __restrict__ prim, float* __restrict__ tout,
                                                       int32_t* __restrict__ inst, float* __restrict__ bary,
                                                       uint32_t* __restrict__ node_tests,
                                                       uint32_t* __restrict__ tri_tests, uint32_t* err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    // plane p of ray i at rays[p * rs + i]
    const float ox = __ldcs(rays + i), oy = __ldcs(rays + rs + i), oz = __ldcs(rays + 2 * rs + i);
    const float dx = __ldcs(rays + 3 * rs + i), dy = __ldcs(rays + 4 * rs + i), dz = __ldcs(rays + 5 * rs + i);
    const float tmax = MODE == 0 ? __int_as_float(0x7f800000) : __ldcs(rays + 6 * rs + i);
    TraceResult r;
    TraceCounters c;
    trace_ray<MODE, STATS>(geo, ox, oy, oz, dx, dy, dz, tmax, r, c, err);
    __stcs(prim + i, r.tri);
    __stcs(tout + i, r.t);
    if (inst) __stcs(inst + i, r.inst);
    if (BARY) {
      __stcs(bary + i, r.b0);
      __stcs(bary + bs + i, r.b1);
      __stcs(bary + 2 * bs + i, r.b2);
    }
    if (STATS) {
      node_tests[i] = c.nodes;
      tri_tests[i] = c.tris;
    }
  }
}

template <int MODE, bool STATS, bool BARY>
static cudaError_t launch_t(const DevGeometry& geo, const float* rays, uint64_t rs, uint64_t n, uint64_t bs,
                            int32_t* prim, float* t, int32_t* inst, float* bary, uint32_t* nt, uint32_t* tt,
                            uint32_t* err, int num_sms, cudaStream_t s) {
  const int block = 128;
  uint64_t blocks = (n + block - 1) / block;
  const uint64_t cap = (uint64_t)num_sms * 64;  // grid-stride beyond ~64 blocks per SM
  if (blocks > cap) blocks = cap;
  if (blocks == 0) return cudaSuccess;
  traverse_kernel<MODE, STATS, BARY><<<(unsigned)blocks, block, 0, s>>>(geo, rays, rs, n, bs, prim, t, inst, bary, nt, tt, err);
  return cudaGetLastError();
}

cudaError_t launch_traverse_strided(const DevGeometry& geo, const float* rays, uint64_t rs, uint64_t n, int mode,
                                    int32_t* prim, float* t, int32_t* inst, float* bary, uint64_t bs,
                                    uint32_t* err, int num_sms, cudaStream_t s, uint32_t* nt, uint32_t* tt) {
  const bool stats = nt != nullptr;
  const bool b = bary != nullptr;
#define TPT_L(M, S, B) launch_t<M, S, B>(geo, rays, rs, n, bs, prim, t, inst, bary, nt, tt, err, num_sms, s)
  if (mode == 0) {
    if (stats) return TPT_L(0, true, false);
    if (b) return TPT_L(0, false, true);
    return TPT_L(0, false, false);
  }
  if (stats) return TPT_L(1, true, false);
  if (b) return TPT_L(1, false, true);
  return TPT_L(1, false, false);
#undef TPT_L
}

cudaError_t launch_traverse_strided(const DevGeometry& geo, const float* rays, uint64_t rs, uint64_t n, int mode,
                                    int32_t* prim, float* t, int32_t* inst, float* bary, uint64_t bs,
                                    uint32_t* err, int num_sms, cudaStream_t s) {
  return launch_traverse_strided(geo, rays, rs, n, mode, prim, t, inst, bary, bs, err, num_sms, s, nullptr, nullptr);
}

cudaError_t launch_traverse(const DevGeometry& geo, const float* rays, uint64_t n, int mode, int32_t* prim, float* t,
                            int32_t* inst, float* bary, uint32_t* nt, uint32_t* tt, uint32_t* err, int num_sms,
                            cudaStream_t s) {
  return launch_traverse_strided(geo, rays, n, n, mode, prim, t, inst, bary, n, err, num_sms, s, nt, tt);
}

}  // namespace tpt
