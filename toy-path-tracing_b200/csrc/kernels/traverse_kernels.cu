// Batch ray-query kernels: `Scene::closest_hit` over a structure-of-arrays
// ray batch (scene/mod.rs:340-395), plus the any-hit occlusion variant.
//
// Persistent warps, "while-while" order: each warp keeps 32 rays in flight;
// lanes step through interior nodes together until every lane faces a leaf
// (or enough lanes have finished to be worth a refill), then all leaves are
// tested together, then finished lanes get new rays from a global counter by
// one warp-aggregated atomic.  Batching keeps the warp on one code path at a
// time without changing any ray's own visit order.
// Traversal stacks: 32 entries per thread in shared memory, spilling to local
// memory beyond that (total depth 128, as the reference).
// Counting (STATS): per-ray node and triangle test counts into node_tests /
// tri_tests when given, and, when `totals` is given, the launch's sums added
// to totals[0..3] = rays, 4-wide node tests, triangle tests, hits (one atomic
// per warp at the end) -- the algorithmic-bytes account of renders.
// The batched instantiation (BATCH) serves rays of many scenes in one launch:
// ray i belongs to job ray_job[i], and a lane loads that job's geometry record
// when it takes the ray.
#include "../api/internal.h"
#include "../device/trace.cuh"

namespace tpt {

constexpr int kBlock = 128;
constexpr int kShStack = 32;
#ifndef TPT_TRAV_MINB
#define TPT_TRAV_MINB 8
#endif
#ifndef TPT_REFILL_MIN
#define TPT_REFILL_MIN 12  // finished lanes that end the node phase early for a refill
#endif

template <int MODE, bool STATS, bool BARY, bool BATCH>
__global__ void __launch_bounds__(kBlock, TPT_TRAV_MINB)
    traverse_kernel(DevGeometry geo, const float* __restrict__ rays, uint64_t rs, uint64_t n, uint64_t bs,
                    int32_t* __restrict__ prim, float* __restrict__ tout, int32_t* __restrict__ inst,
                    float* __restrict__ bary, uint32_t* __restrict__ node_tests, uint32_t* __restrict__ tri_tests,
                    unsigned long long* __restrict__ counter, const uint32_t* __restrict__ n_dev, uint32_t* err,
                    const DevJob* __restrict__ jobs, const uint32_t* __restrict__ ray_job,
                    unsigned long long* __restrict__ totals, uint32_t* __restrict__ aux,
                    const uint32_t* __restrict__ aux_index) {
  if (n_dev) n = *n_dev;  // queue length produced on the device (wavefront stages)
  DevGeometry lane_geo;  // BATCH: the scene of this lane's ray
  const DevGeometry& G = BATCH ? lane_geo : geo;
  __shared__ uint32_t stack_sh[kShStack * kBlock];
  SplitStack<kShStack> st;
  st.sh = stack_sh + threadIdx.x;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  TravState s;
  TraceCounters c;
  int64_t ray = -1;  // -1: needs a ray, -2: no rays left, >= 0: active ray index
  int stalled = 0;   // consecutive iterations in which no lane of the warp advanced
  uint32_t sum_rays = 0, sum_hits = 0;  // STATS with totals: this lane's finished rays
  unsigned long long sum_nodes = 0, sum_tris = 0;
  for (;;) {
    bool moved = false;
    // refill finished lanes: one warp-aggregated atomic, converged ray setup
    const unsigned need = __ballot_sync(0xffffffffu, ray == -1);
    if (need) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if ((int)lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (ray == -1) {
        const uint64_t i = base + __popc(need & lt_mask);
        moved = true;
        if (i < n) {
          ray = (int64_t)i;
          // plane p of ray i at rays[p * rs + i]
          const float ox = __ldcs(rays + i), oy = __ldcs(rays + rs + i), oz = __ldcs(rays + 2 * rs + i);
          const float dx = __ldcs(rays + 3 * rs + i), dy = __ldcs(rays + 4 * rs + i), dz = __ldcs(rays + 5 * rs + i);
          const float tmax = MODE == 0 ? __int_as_float(0x7f800000) : __ldcs(rays + 6 * rs + i);
          if (BATCH) lane_geo = jobs[__ldg(ray_job + i)].render.geo;
          trav_init(G, s, ox, oy, oz, dx, dy, dz, tmax, aux ? aux + (aux_index ? aux_index[i] : i) : nullptr);
          if (STATS) { c.nodes = 0; c.tris = 0; }
        } else {
          ray = -2;
        }
      }
    }
    if (__all_sync(0xffffffffu, ray == -2)) break;
    const bool active = ray >= 0;
    // phase A: interior nodes until every active lane faces a leaf, or until
    // enough lanes have finished their ray to be worth a refill (lanes with no
    // ray left do not count: they can never be refilled)
    for (;;) {
      const bool want = active && !(s.next & kLeafBit);
      if (!__any_sync(0xffffffffu, want)) break;
      if (__popc(__ballot_sync(0xffffffffu, active && s.next == kNone)) >= TPT_REFILL_MIN) break;
      if (want) {
        node_step<STATS>(G, s, st, c, err);
        moved = true;
      }
    }
    // phase B: one leaf / instance entry per lane
    if (active && s.next != kNone && (s.next & kLeafBit)) {
      leaf_step<MODE, STATS>(G, s, st, c, err);
      moved = true;
    }
    if (active && s.next == kNone) {
      moved = true;
      const uint64_t i = (uint64_t)ray;
      __stcs(prim + i, s.res.tri);
      __stcs(tout + i, s.res.t);
      if (aux) aux[aux_index ? aux_index[i] : i] = s.aux;
      if (inst) __stcs(inst + i, s.res.inst);
      if (BARY) {
        __stcs(bary + i, s.res.b0);
        __stcs(bary + bs + i, s.res.b1);
        __stcs(bary + 2 * bs + i, s.res.b2);
      }
      if (STATS) {
        if (node_tests) {
          node_tests[i] = c.nodes;
          tri_tests[i] = c.tris;
        }
        sum_rays += 1;
        sum_hits += s.res.tri >= 0 ? 1 : 0;
        sum_nodes += c.nodes;
        sum_tris += c.tris;
      }
      ray = -1;
    }
    // watchdog: every iteration must advance some lane; if none does for a
    // long run, flag the launch and stop instead of spinning
    if (__any_sync(0xffffffffu, moved)) {
      stalled = 0;
    } else if (++stalled > 64) {
      if (lane == 0) atomicOr(err, kDevErrTimeout);
      break;
    }
  }
  if (STATS && totals) {  // the loop ends converged (every exit is warp-uniform)
    unsigned long long r = sum_rays, h = sum_hits, nn = sum_nodes, tt = sum_tris;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      r += __shfl_down_sync(0xffffffffu, r, o);
      h += __shfl_down_sync(0xffffffffu, h, o);
      nn += __shfl_down_sync(0xffffffffu, nn, o);
      tt += __shfl_down_sync(0xffffffffu, tt, o);
    }
    if (lane == 0 && r) {
      atomicAdd(totals, r);
      atomicAdd(totals + 1, nn);
      atomicAdd(totals + 2, tt);
      atomicAdd(totals + 3, h);
    }
  }
}

template <int MODE, bool STATS, bool BARY, bool BATCH>
static cudaError_t launch_t(const DevGeometry& geo, const float* rays, uint64_t rs, uint64_t n, uint64_t bs,
                            int32_t* prim, float* t, int32_t* inst, float* bary, uint32_t* nt, uint32_t* tt,
                            unsigned long long* counter, const uint32_t* n_dev, uint32_t* err, int num_sms,
                            cudaStream_t s, const DevJob* jobs, const uint32_t* ray_job, unsigned long long* totals,
                            uint32_t* aux, const uint32_t* aux_index) {
  if (n == 0) return cudaSuccess;
  static int blocks_per_sm = 0;
  if (blocks_per_sm == 0) {
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &blocks_per_sm, traverse_kernel<MODE, STATS, BARY, BATCH>, kBlock, 0);
    if (e != cudaSuccess || blocks_per_sm <= 0) blocks_per_sm = 4;
  }
  uint64_t blocks = (uint64_t)num_sms * blocks_per_sm;
  const uint64_t need = (n + kBlock - 1) / kBlock;  // n is an upper bound when n_dev is given
  if (blocks > need) blocks = need;
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  traverse_kernel<MODE, STATS, BARY, BATCH><<<(unsigned)blocks, kBlock, 0, s>>>(
      geo, rays, rs, n, bs, prim, t, inst, bary, nt, tt, counter, n_dev, err, jobs, ray_job, totals, aux, aux_index);
  return cudaGetLastError();
}

cudaError_t launch_traverse_strided(const DevGeometry& geo, const float* rays, uint64_t rs, uint64_t n, int mode,
                                    int32_t* prim, float* t, int32_t* inst, float* bary, uint64_t bs,
                                    unsigned long long* counter, uint32_t* err, int num_sms, cudaStream_t s,
                                    uint32_t* nt, uint32_t* tt, const uint32_t* n_dev, const DevJob* jobs,
                                    const uint32_t* ray_job, unsigned long long* totals, uint32_t* aux,
                                    const uint32_t* aux_index) {
  const bool stats = nt != nullptr || totals != nullptr;
  const bool b = bary != nullptr;
#define TPT_L(M, S, B, J) \
  launch_t<M, S, B, J>(geo, rays, rs, n, bs, prim, t, inst, bary, nt, tt, counter, n_dev, err, num_sms, s, jobs, \
                       ray_job, totals, aux, aux_index)
  if (jobs) {  // batched wavefront: closest hit, with or without barycentrics
    if (mode != 0 || stats) return cudaErrorInvalidValue;
    if (b) return TPT_L(0, false, true, true);
    return TPT_L(0, false, false, true);
  }
  if (mode == 0) {
    if (stats && b) return TPT_L(0, true, true, false);
    if (stats) return TPT_L(0, true, false, false);
    if (b) return TPT_L(0, false, true, false);
    return TPT_L(0, false, false, false);
  }
  if (stats) return TPT_L(1, true, false, false);
  if (b) return TPT_L(1, false, true, false);
  return TPT_L(1, false, false, false);
#undef TPT_L
}

}  // namespace tpt
