// The 4-wide BVH builder on the GPU: build_qbvh (crates/renderer/src/qbvh.rs:
// 144-516) -- binned SAH over 16 bins per axis, leaf target 4, forced median
// split above 16 primitives, each node taking up to two children from each
// side of its binary split -- producing the same node array and primitive
// order as the host builder (host/qbvh_build.cpp).
//
// Large ranges (>= kSeqMax primitives) are processed level by level, all
// ranges of a level at once, element-parallel:
//   bounds     per position: atomic min/max into its range's box and
//              centroid box (warp- or block-aggregated)
//   binning    per position and axis: its bin, atomic bounds and counts
//              (block-aggregated in shared memory when a block lies in one range)
//   decision   per range: the SAH sweep, in the host builder's order
//   partition  the reference's in-place swap partition reproduced exactly
//              from prefix counts: with mid = #left, the F region [0, mid)
//              keeps its left elements; its k-th right element goes to the top
//              of the k-th run of the B region [mid, n) (runs read downwards,
//              each ending at a left element), right elements of a run shift
//              down by one, the run's left element takes the F element's
//              place, and the tail below the last run rotates down by one
//   emit       the next level's ranges, node ids and child links
// The forced median split of a large range (no usable binned split: rare)
// sorts the range on the host.  Ranges below kSeqMax are built whole by one
// thread each, with the host builder's recursion on an explicit stack.
//
// The node records are then flattened in pre-order on the host, as the
// reference's flatten_recursive does.  Bounds are min/max reductions and
// therefore order-independent, except that the host's fmin/fmax keep whichever
// of +0.0 and -0.0 they meet first: inputs are canonicalised to +0.0 here, so
// a box face at zero may carry +0.0 where the host builder would keep -0.0
// (the same value; traversal results do not change).
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <thread>
#include <vector>

#include "../api/internal.h"
#include "../host/host_types.h"

namespace tpt {

namespace {

constexpr int kBinsG = 16;
constexpr uint32_t kLeafTargetG = 4, kLeafMaxG = 16;
constexpr uint32_t kSeqMax = 64;  // ranges below this size are built whole by one thread
constexpr uint32_t kNoneG = 0xFFFFFFFFu;
constexpr int kBlk = 256;
constexpr int kSeqStack = 96;

enum : uint32_t { kRoleNode = 0, kRoleSide = 1 };
enum : uint32_t { kActSplit = 1, kActMedian = 2, kActSingle = 3 };

struct GNode {
  float lo[3], hi[3];
  uint32_t begin, count;
  uint32_t kid[2][2];  // [side][k]: node ids of the children taken from each side
  uint32_t nkid[2];    // 0 on both sides: a leaf
};

struct Task {
  uint32_t begin, count, role, node, side;
  uint32_t action, axis, bin, mid;
  float cmin, scale;
  uint32_t next[2];  // next-level task ids of the two halves (or of the whole range)
};

// accumulators of one large range
struct TaskAcc {
  float box[6], cbox[6];
  float bin_box[3][kBinsG][6];
  uint32_t bin_cnt[3][kBinsG];
  float axis_cmin[3], axis_scale[3];
  uint32_t axis_ok;
};
constexpr int kAccFloats = 12 + 3 * kBinsG * 6;

struct Counters {
  uint32_t next_tasks, seq_tasks, nodes, medians;
};

struct BuildBuffers {
  float* box;  // 6 planes: lo x y z, hi x y z
  float* cen;  // 3 planes
  uint32_t* order;
  uint32_t* order_tmp;
  uint32_t* seg;     // task of each position at the current level (kNoneG: none)
  uint32_t* flag;    // n + 1 left flags, then their exclusive scan
  uint32_t* scan;
  uint32_t* rpos;    // per split range: position of its k-th right element in F
  uint32_t* ypos;    // per split range: position of its j-th left element in B, from the top
  GNode* nodes;
  Counters* cnt;
  uint32_t n;
};

__device__ __forceinline__ void atomic_min_f(float* a, float v) {
  if (v >= 0.0f) atomicMin((int*)a, __float_as_int(v));
  else atomicMax((unsigned*)a, __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_f(float* a, float v) {
  if (v >= 0.0f) atomicMax((int*)a, __float_as_int(v));
  else atomicMin((unsigned*)a, __float_as_uint(v));
}

__device__ __forceinline__ uint32_t bin_of_g(float c, float cmin, float scale) {
  float raw = (c - cmin) * scale;
  if (isnan(raw)) return 0;
  if (raw < 0.0f) raw = 0.0f;
  if (raw > (float)(kBinsG - 1)) raw = (float)(kBinsG - 1);
  return (uint32_t)raw;
}

__device__ __forceinline__ float area6(const float* b) {
  const float ex = fmaxf(b[3] - b[0], 0.0f), ey = fmaxf(b[4] - b[1], 0.0f), ez = fmaxf(b[5] - b[2], 0.0f);
  return 2.0f * (ex * ey + ex * ez + ey * ez);
}
__device__ __forceinline__ void empty6(float* b) {
  b[0] = b[1] = b[2] = __int_as_float(0x7f800000);
  b[3] = b[4] = b[5] = -__int_as_float(0x7f800000);
}
__device__ __forceinline__ void grow6(float* a, const float* b) {
  for (int k = 0; k < 3; ++k) {
    a[k] = fminf(a[k], b[k]);
    a[3 + k] = fmaxf(a[3 + k], b[3 + k]);
  }
}

// The SAH sweep of one axis over its 16 bins (host best_split): the best bin
// and cost, or -1.
__device__ int sweep_bins(const float (*bin_box)[6], const uint32_t* bin_cnt, float parent_area, float* best_cost) {
  float suffix[kBinsG][6];
  float acc[6];
  empty6(acc);
  for (int i = kBinsG - 1; i >= 0; --i) {
    grow6(acc, bin_box[i]);
    for (int k = 0; k < 6; ++k) suffix[i][k] = acc[k];
  }
  uint32_t total = 0;
  for (int i = 0; i < kBinsG; ++i) total += bin_cnt[i];
  if (total <= 1) return -1;
  float pre[6];
  empty6(pre);
  uint32_t left = 0;
  float best = __int_as_float(0x7f800000);
  int best_bin = -1;
  for (int s = 0; s < kBinsG - 1; ++s) {
    grow6(pre, bin_box[s]);
    left += bin_cnt[s];
    const uint32_t right = total - left;
    if (left == 0 || right == 0) continue;
    const float cost = 1.0f + 1.0f * (area6(pre) * (float)left + area6(suffix[s + 1]) * (float)right) / parent_area;
    if (cost < best) {
      best = cost;
      best_bin = s;
    }
  }
  *best_cost = best;
  return best_bin;
}

// ---- preparation -----------------------------------------------------------------

__global__ void k_prep(const float* __restrict__ bounds6, uint32_t n, BuildBuffers B) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float b[6];
  for (int k = 0; k < 6; ++k) b[k] = bounds6[6 * (size_t)i + k] + 0.0f;  // -0.0 -> +0.0
  for (int k = 0; k < 6; ++k) B.box[(size_t)k * n + i] = b[k];
  for (int k = 0; k < 3; ++k) B.cen[(size_t)k * n + i] = 0.5f * (b[k] + b[3 + k]);
  B.order[i] = i;
  B.seg[i] = 0;
}

// ---- the level kernels (large ranges) ------------------------------------------

__global__ void k_acc_init(const Task* __restrict__ T, uint32_t m, TaskAcc* acc) {
  const uint64_t gid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t t = (uint32_t)(gid / (kAccFloats + 3 * kBinsG + 1));
  const uint32_t k = (uint32_t)(gid % (kAccFloats + 3 * kBinsG + 1));
  if (t >= m) return;
  TaskAcc& a = acc[t];
  if (k < kAccFloats) {
    float* f = &a.box[0];
    // box, cbox, then the bins: lo faces start at +inf, hi faces at -inf
    const uint32_t face = k < 12 ? k % 6 : (k - 12) % 6;
    f[k] = face < 3 ? __int_as_float(0x7f800000) : -__int_as_float(0x7f800000);
  } else if (k < kAccFloats + 3 * kBinsG) {
    (&a.bin_cnt[0][0])[k - kAccFloats] = 0;
  } else {
    a.axis_ok = 0;
  }
}

__global__ void __launch_bounds__(kBlk) k_bounds(BuildBuffers B, TaskAcc* acc) {
  const uint32_t n = B.n;
  const unsigned lane = threadIdx.x & 31u;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p - lane < n; p += gridDim.x * blockDim.x) {
    const bool in = p < n;
    const uint32_t t = in ? B.seg[p] : kNoneG;
    float v[12];
    if (t != kNoneG) {
      const uint32_t q = B.order[p];
      for (int k = 0; k < 6; ++k) v[k] = B.box[(size_t)k * n + q];
      for (int k = 0; k < 3; ++k) v[6 + k] = v[9 + k] = B.cen[(size_t)k * n + q];
    }
    const uint32_t t0 = __shfl_sync(0xffffffffu, t, 0);
    const bool uniform = __all_sync(0xffffffffu, t == t0) && t0 != kNoneG;
    if (uniform) {
      for (int o = 16; o > 0; o >>= 1) {
        for (int k = 0; k < 3; ++k) {
          v[k] = fminf(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
          v[3 + k] = fmaxf(v[3 + k], __shfl_xor_sync(0xffffffffu, v[3 + k], o));
          v[6 + k] = fminf(v[6 + k], __shfl_xor_sync(0xffffffffu, v[6 + k], o));
          v[9 + k] = fmaxf(v[9 + k], __shfl_xor_sync(0xffffffffu, v[9 + k], o));
        }
      }
      if (lane == 0) {
        TaskAcc& a = acc[t0];
        for (int k = 0; k < 3; ++k) {
          atomic_min_f(&a.box[k], v[k]);
          atomic_max_f(&a.box[3 + k], v[3 + k]);
          atomic_min_f(&a.cbox[k], v[6 + k]);
          atomic_max_f(&a.cbox[3 + k], v[9 + k]);
        }
      }
    } else if (t != kNoneG) {
      TaskAcc& a = acc[t];
      for (int k = 0; k < 3; ++k) {
        atomic_min_f(&a.box[k], v[k]);
        atomic_max_f(&a.box[3 + k], v[3 + k]);
        atomic_min_f(&a.cbox[k], v[6 + k]);
        atomic_max_f(&a.cbox[3 + k], v[9 + k]);
      }
    }
  }
}

// per range: the binning frame of each axis (host best_split: an axis whose
// centroid extent is not positive is skipped)
__global__ void k_split_prep(const Task* __restrict__ T, uint32_t m, TaskAcc* acc) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  TaskAcc& a = acc[t];
  uint32_t ok = 0;
  for (int ax = 0; ax < 3; ++ax) {
    const float cmin = a.cbox[ax], cmax = a.cbox[3 + ax];
    a.axis_cmin[ax] = cmin;
    a.axis_scale[ax] = (float)kBinsG / fmaxf(cmax - cmin, 1.0e-30f);
    if (cmax - cmin > 0.0f) ok |= 1u << ax;
  }
  a.axis_ok = ok;
}

__global__ void __launch_bounds__(kBlk) k_bin(BuildBuffers B, TaskAcc* acc, uint32_t chunk) {
  __shared__ float sh_box[3][kBinsG][6];
  __shared__ uint32_t sh_cnt[3][kBinsG];
  const uint32_t n = B.n;
  const uint32_t b0 = blockIdx.x * chunk;
  if (b0 >= n) return;
  const uint32_t b1 = min(n, b0 + chunk);
  const uint32_t tf = B.seg[b0], tl = B.seg[b1 - 1];
  const bool uniform = tf == tl && tf != kNoneG;  // ranges are contiguous
  if (uniform) {
    for (int k = threadIdx.x; k < 3 * kBinsG * 6; k += blockDim.x)
      (&sh_box[0][0][0])[k] = (k % 6) < 3 ? __int_as_float(0x7f800000) : -__int_as_float(0x7f800000);
    for (int k = threadIdx.x; k < 3 * kBinsG; k += blockDim.x) (&sh_cnt[0][0])[k] = 0;
    __syncthreads();
  }
  for (uint32_t p = b0 + threadIdx.x; p < b1; p += blockDim.x) {
    const uint32_t t = uniform ? tf : B.seg[p];
    if (t == kNoneG) continue;
    const TaskAcc& a = acc[t];
    const uint32_t ok = a.axis_ok;
    if (!ok) continue;
    const uint32_t q = B.order[p];
    float bx[6];
    for (int k = 0; k < 6; ++k) bx[k] = B.box[(size_t)k * n + q];
    for (int ax = 0; ax < 3; ++ax) {
      if (!(ok & (1u << ax))) continue;
      const uint32_t k = bin_of_g(B.cen[(size_t)ax * n + q], a.axis_cmin[ax], a.axis_scale[ax]);
      float* bb = uniform ? sh_box[ax][k] : acc[t].bin_box[ax][k];
      for (int f = 0; f < 3; ++f) {
        atomic_min_f(bb + f, bx[f]);
        atomic_max_f(bb + 3 + f, bx[3 + f]);
      }
      atomicAdd(uniform ? &sh_cnt[ax][k] : &acc[t].bin_cnt[ax][k], 1u);
    }
  }
  if (uniform) {
    __syncthreads();
    TaskAcc& a = acc[tf];
    for (int k = threadIdx.x; k < 3 * kBinsG * 6; k += blockDim.x) {
      const float v = (&sh_box[0][0][0])[k];
      float* dst = &a.bin_box[0][0][0] + k;
      if ((k % 6) < 3) {
        if (v != __int_as_float(0x7f800000)) atomic_min_f(dst, v);
      } else if (v != -__int_as_float(0x7f800000)) {
        atomic_max_f(dst, v);
      }
    }
    for (int k = threadIdx.x; k < 3 * kBinsG; k += blockDim.x) {
      const uint32_t c = (&sh_cnt[0][0])[k];
      if (c) atomicAdd(&a.bin_cnt[0][0] + k, c);
    }
  }
}

// per range: the decision (node_task / expand_side on a range of >= kSeqMax > 16
// primitives, so neither the leaf-size tests nor the SAH leaf test apply)
__global__ void k_decide(Task* T, uint32_t m, const TaskAcc* __restrict__ acc, GNode* nodes) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  Task& tk = T[t];
  const TaskAcc& a = acc[t];
  if (tk.role == kRoleNode) {
    GNode& g = nodes[tk.node];
    for (int k = 0; k < 3; ++k) {
      g.lo[k] = a.box[k];
      g.hi[k] = a.box[3 + k];
    }
    g.begin = tk.begin;
    g.count = tk.count;
  }
  const float parent_area = fmaxf(area6(a.box), 1.0e-30f);
  bool found = false;
  float best_cost = 0.0f;
  for (int ax = 0; ax < 3; ++ax) {
    if (!(a.axis_ok & (1u << ax))) continue;
    float cost;
    const int bin = sweep_bins(a.bin_box[ax], a.bin_cnt[ax], parent_area, &cost);
    if (bin < 0) continue;
    if (!found || cost < best_cost) {
      found = true;
      best_cost = cost;
      tk.axis = ax;
      tk.bin = (uint32_t)bin;
      tk.cmin = a.axis_cmin[ax];
      tk.scale = a.axis_scale[ax];
    }
  }
  tk.action = found ? kActSplit : (tk.role == kRoleNode ? kActMedian : kActSingle);
  tk.mid = 0;
}

__global__ void __launch_bounds__(kBlk) k_flag(BuildBuffers B, const Task* __restrict__ T) {
  const uint32_t n = B.n;
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > n) return;
  uint32_t f = 0;
  if (p < n) {
    const uint32_t t = B.seg[p];
    if (t != kNoneG && T[t].action == kActSplit) {
      const Task& tk = T[t];
      f = bin_of_g(B.cen[(size_t)tk.axis * n + B.order[p]], tk.cmin, tk.scale) <= tk.bin ? 1u : 0u;
    }
  }
  B.flag[p] = f;
}

__global__ void k_mid(Task* T, uint32_t m, BuildBuffers B) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  Task& tk = T[t];
  if (tk.action != kActSplit) return;
  tk.mid = B.scan[tk.begin + tk.count] - B.scan[tk.begin];
}

// per position of a split range: record its place in the F/B run structure
__global__ void __launch_bounds__(kBlk) k_rpos(BuildBuffers B, const Task* __restrict__ T) {
  const uint32_t n = B.n;
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const uint32_t t = B.seg[p];
  if (t == kNoneG || T[t].action != kActSplit) return;
  const Task& tk = T[t];
  const uint32_t b = tk.begin, rel = p - b, mid = tk.mid;
  const uint32_t lbefore = B.scan[p] - B.scan[b];
  const bool is_l = B.flag[p] != 0;
  if (rel < mid && !is_l) B.rpos[b + (rel - lbefore)] = rel;             // k-th right element of F
  else if (rel >= mid && is_l) B.ypos[b + (mid - lbefore - 1)] = rel;   // j-th left element of B, from the top
}

__global__ void __launch_bounds__(kBlk) k_perm(BuildBuffers B, const Task* __restrict__ T) {
  const uint32_t n = B.n;
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const uint32_t t = B.seg[p];
  if (t == kNoneG || T[t].action != kActSplit) return;
  const Task& tk = T[t];
  const uint32_t b = tk.begin, cnt = tk.count, rel = p - b, mid = tk.mid;
  const uint32_t lbefore = B.scan[p] - B.scan[b];
  const bool is_l = B.flag[p] != 0;
  const uint32_t l_in_f = B.scan[b + mid] - B.scan[b];
  const uint32_t K = mid - l_in_f;  // right elements in F = left elements in B
  const uint32_t yk = K ? B.ypos[b + K - 1] : cnt;  // lowest left element of B (or the range end)
  uint32_t np;
  if (rel < mid) {
    if (is_l) {
      np = rel;
    } else {
      const uint32_t k = rel - lbefore;
      np = (k == 0 ? cnt : B.ypos[b + k - 1]) - 1;  // top of run k
    }
  } else if (is_l) {
    np = B.rpos[b + (mid - lbefore - 1)];
  } else if (rel > yk || rel != mid) {
    np = rel - 1;  // shifts down within its run or the tail
  } else {
    np = yk - 1;  // the tail's first element rotates to its top
  }
  B.order_tmp[b + np] = B.order[p];
}

__global__ void __launch_bounds__(kBlk) k_copyback(BuildBuffers B, const Task* __restrict__ T) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= B.n) return;
  const uint32_t t = B.seg[p];
  if (t == kNoneG || T[t].action != kActSplit) return;
  B.order[p] = B.order_tmp[p];
}

__device__ __forceinline__ uint32_t push_task(Task* list, uint32_t* counter, uint32_t cap, uint32_t* overflow,
                                              uint32_t begin, uint32_t count, uint32_t role, uint32_t node,
                                              uint32_t side) {
  const uint32_t i = atomicAdd(counter, 1u);
  if (i >= cap) {
    atomicExch(overflow, 1u);
    return kNoneG;
  }
  Task& t = list[i];
  t.begin = begin;
  t.count = count;
  t.role = role;
  t.node = node;
  t.side = side;
  t.action = 0;
  t.mid = 0;
  t.next[0] = t.next[1] = kNoneG;
  return i;
}

struct Lists {
  Task* next;
  Task* seq;
  uint32_t next_cap, seq_cap, node_cap;
  uint32_t* overflow;
};

__device__ __forceinline__ uint32_t alloc_nodes(BuildBuffers& B, const Lists& Ls, uint32_t k) {
  const uint32_t id = atomicAdd(&B.cnt->nodes, k);
  if (id + k > Ls.node_cap) {
    atomicExch(Ls.overflow, 1u);
    return kNoneG;
  }
  return id;
}

// Ranges that need the forced median split (make_leaf_or_force_split on a
// large range): listed for the host, which sorts them before k_emit.
__global__ void k_median_mark(const Task* __restrict__ T, uint32_t m, uint32_t* list, BuildBuffers B) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  const Task& tk = T[t];
  if (tk.role != kRoleNode) return;
  if (tk.action == kActSplit && tk.mid != 0 && tk.mid != tk.count) return;
  list[atomicAdd(&B.cnt->medians, 1u)] = t;
}

// Next-level ranges: large ones into Ls.next, small ones into Ls.seq (built
// whole by k_seq); next[] of each current range names the next-level task of
// each half (kNoneG when it went to the small list).
__global__ void k_emit(Task* T, uint32_t m, BuildBuffers B, Lists Ls) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  Task& tk = T[t];
  const uint32_t b = tk.begin, n = tk.count;
  auto emit = [&](uint32_t begin, uint32_t count, uint32_t role, uint32_t node, uint32_t side) -> uint32_t {
    if (count >= kSeqMax)
      return push_task(Ls.next, &B.cnt->next_tasks, Ls.next_cap, Ls.overflow, begin, count, role, node, side);
    push_task(Ls.seq, &B.cnt->seq_tasks, Ls.seq_cap, Ls.overflow, begin, count, role, node, side);
    return kNoneG;
  };
  const bool split = tk.action == kActSplit && tk.mid != 0 && tk.mid != n;
  if (tk.role == kRoleNode) {
    // build_qbvh_node: both sides of the split (or of the forced median split,
    // whose range the host sorted) go to split_into_children
    const uint32_t mid = split ? tk.mid : n / 2;
    tk.mid = mid;
    tk.next[0] = emit(b, mid, kRoleSide, tk.node, 0);
    tk.next[1] = emit(b + mid, n - mid, kRoleSide, tk.node, 1);
  } else if (split) {
    // split_into_children: two children, one per half
    const uint32_t id = alloc_nodes(B, Ls, 2);
    if (id == kNoneG) return;
    GNode& parent = B.nodes[tk.node];
    parent.kid[tk.side][0] = id;
    parent.kid[tk.side][1] = id + 1;
    parent.nkid[tk.side] = 2;
    tk.next[0] = emit(b, tk.mid, kRoleNode, id, 0);
    tk.next[1] = emit(b + tk.mid, n - tk.mid, kRoleNode, id + 1, 0);
  } else {
    // split_into_children: one child built on the whole range
    const uint32_t id = alloc_nodes(B, Ls, 1);
    if (id == kNoneG) return;
    GNode& parent = B.nodes[tk.node];
    parent.kid[tk.side][0] = id;
    parent.nkid[tk.side] = 1;
    tk.mid = n;
    tk.next[0] = emit(b, n, kRoleNode, id, 0);
  }
}

__global__ void __launch_bounds__(kBlk) k_seg(BuildBuffers B, const Task* __restrict__ T) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= B.n) return;
  const uint32_t t = B.seg[p];
  if (t == kNoneG) return;
  const Task& tk = T[t];
  B.seg[p] = (p - tk.begin) < tk.mid ? tk.next[0] : tk.next[1];
}

// ---- small ranges: the host builder's recursion, one thread per range -------------

__device__ void seq_range_box(const BuildBuffers& B, uint32_t b, uint32_t n, float* box) {
  empty6(box);
  for (uint32_t i = b; i < b + n; ++i) {
    const uint32_t q = B.order[i];
    for (int k = 0; k < 3; ++k) {
      box[k] = fminf(box[k], B.box[(size_t)k * B.n + q]);
      box[3 + k] = fmaxf(box[3 + k], B.box[(size_t)(3 + k) * B.n + q]);
    }
  }
}

struct SeqSplit {
  uint32_t axis, bin;
  float cmin, scale, cost;
};

__device__ bool seq_best_split(const BuildBuffers& B, uint32_t b, uint32_t n, const float* parent, SeqSplit* out) {
  if (n <= 1) return false;
  float cb[6];
  empty6(cb);
  for (uint32_t i = b; i < b + n; ++i) {
    const uint32_t q = B.order[i];
    for (int k = 0; k < 3; ++k) {
      const float c = B.cen[(size_t)k * B.n + q];
      cb[k] = fminf(cb[k], c);
      cb[3 + k] = fmaxf(cb[3 + k], c);
    }
  }
  const float parent_area = fmaxf(area6(parent), 1.0e-30f);
  bool found = false;
  for (int ax = 0; ax < 3; ++ax) {
    const float cmin = cb[ax], cmax = cb[3 + ax];
    if (cmax - cmin <= 0.0f) continue;
    const float scale = (float)kBinsG / fmaxf(cmax - cmin, 1.0e-30f);
    float bin_box[kBinsG][6];
    uint32_t bin_cnt[kBinsG];
    for (int i = 0; i < kBinsG; ++i) {
      empty6(bin_box[i]);
      bin_cnt[i] = 0;
    }
    for (uint32_t i = b; i < b + n; ++i) {
      const uint32_t q = B.order[i];
      const uint32_t k = bin_of_g(B.cen[(size_t)ax * B.n + q], cmin, scale);
      for (int f = 0; f < 3; ++f) {
        bin_box[k][f] = fminf(bin_box[k][f], B.box[(size_t)f * B.n + q]);
        bin_box[k][3 + f] = fmaxf(bin_box[k][3 + f], B.box[(size_t)(3 + f) * B.n + q]);
      }
      bin_cnt[k] += 1;
    }
    float cost;
    const int bin = sweep_bins(bin_box, bin_cnt, parent_area, &cost);
    if (bin < 0) continue;
    if (!found || cost < out->cost) {
      out->axis = ax;
      out->bin = (uint32_t)bin;
      out->cmin = cmin;
      out->scale = scale;
      out->cost = cost;
      found = true;
    }
  }
  return found;
}

// the reference's in-place swap partition (qbvh.rs:460-482)
__device__ uint32_t seq_partition(const BuildBuffers& B, uint32_t b, uint32_t n, const SeqSplit& s) {
  uint32_t l = b, r = b + n;
  while (l < r) {
    const uint32_t k = bin_of_g(B.cen[(size_t)s.axis * B.n + B.order[l]], s.cmin, s.scale);
    if (k <= s.bin) {
      ++l;
    } else {
      --r;
      const uint32_t x = B.order[l];
      B.order[l] = B.order[r];
      B.order[r] = x;
    }
  }
  return l - b;
}

// forced median order: ascending centroid on `axis`, ties by primitive index
// (heap sort; the order is total, so any correct sort gives the same result)
__device__ __forceinline__ bool seq_less(const BuildBuffers& B, int axis, uint32_t x, uint32_t y) {
  const float cx = B.cen[(size_t)axis * B.n + x], cy = B.cen[(size_t)axis * B.n + y];
  if (cx < cy) return true;
  if (cy < cx) return false;
  return x < y;
}
__device__ void seq_sort(const BuildBuffers& B, uint32_t b, uint32_t n, int axis) {
  uint32_t* a = B.order + b;
  auto sift = [&](uint32_t root, uint32_t end) {
    for (;;) {
      uint32_t child = 2 * root + 1;
      if (child >= end) return;
      if (child + 1 < end && seq_less(B, axis, a[child], a[child + 1])) ++child;
      if (!seq_less(B, axis, a[root], a[child])) return;
      const uint32_t x = a[root];
      a[root] = a[child];
      a[child] = x;
      root = child;
    }
  };
  for (uint32_t i = n / 2; i-- > 0;) sift(i, n);
  for (uint32_t end = n; end-- > 1;) {
    const uint32_t x = a[0];
    a[0] = a[end];
    a[end] = x;
    sift(0, end);
  }
}

struct SeqEntry {
  uint32_t role, b, n, node, side;
};

__global__ void __launch_bounds__(128) k_seq(const Task* __restrict__ tasks, uint32_t count, BuildBuffers B, Lists Ls) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  SeqEntry st[kSeqStack];
  int sp = 0;
  st[sp++] = SeqEntry{tasks[t].role, tasks[t].begin, tasks[t].count, tasks[t].node, tasks[t].side};
  while (sp > 0) {
    const SeqEntry e = st[--sp];
    float box[6];
    seq_range_box(B, e.b, e.n, box);
    if (e.role == kRoleNode) {
      // build_qbvh_node
      GNode& g = B.nodes[e.node];
      for (int k = 0; k < 3; ++k) {
        g.lo[k] = box[k];
        g.hi[k] = box[3 + k];
      }
      g.begin = e.b;
      g.count = e.n;
      if (e.n <= kLeafTargetG) continue;
      SeqSplit s;
      bool median = false;
      uint32_t mid = 0;
      if (!seq_best_split(B, e.b, e.n, box, &s)) {
        median = true;
      } else if (s.cost >= 1.0f * (float)e.n && e.n <= kLeafMaxG) {
        continue;  // leaf
      } else {
        mid = seq_partition(B, e.b, e.n, s);
        if (mid == 0 || mid == e.n) median = true;
      }
      if (median) {
        // make_leaf_or_force_split
        if (e.n <= kLeafMaxG) continue;
        const float ex = box[3] - box[0], ey = box[4] - box[1], ez = box[5] - box[2];
        const int axis = (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
        seq_sort(B, e.b, e.n, axis);
        mid = e.n / 2;
      }
      if (sp + 2 > kSeqStack) {
        atomicExch(Ls.overflow, 2u);
        return;
      }
      // the larger half is pushed first (popped last), which bounds the stack
      // by the depth of a balanced split; disjoint ranges make the order free
      const SeqEntry lo{kRoleSide, e.b, mid, e.node, 0}, hi{kRoleSide, e.b + mid, e.n - mid, e.node, 1};
      st[sp++] = mid >= e.n - mid ? lo : hi;
      st[sp++] = mid >= e.n - mid ? hi : lo;
    } else {
      // split_into_children
      GNode& parent = B.nodes[e.node];
      SeqSplit s;
      uint32_t mid = 0;
      bool single = e.n <= kLeafTargetG || !seq_best_split(B, e.b, e.n, box, &s) ||
                    (s.cost >= 1.0f * (float)e.n && e.n <= kLeafMaxG);
      if (!single) {
        mid = seq_partition(B, e.b, e.n, s);
        single = mid == 0 || mid == e.n;
      }
      if (sp + 2 > kSeqStack) {
        atomicExch(Ls.overflow, 2u);
        return;
      }
      if (single) {
        const uint32_t id = alloc_nodes(B, Ls, 1);
        if (id == kNoneG) return;
        parent.kid[e.side][0] = id;
        parent.nkid[e.side] = 1;
        st[sp++] = SeqEntry{kRoleNode, e.b, e.n, id, 0};
      } else {
        const uint32_t id = alloc_nodes(B, Ls, 2);
        if (id == kNoneG) return;
        parent.kid[e.side][0] = id;
        parent.kid[e.side][1] = id + 1;
        parent.nkid[e.side] = 2;
        const SeqEntry lo{kRoleNode, e.b, mid, id, 0}, hi{kRoleNode, e.b + mid, e.n - mid, id + 1, 0};
        st[sp++] = mid >= e.n - mid ? lo : hi;
        st[sp++] = mid >= e.n - mid ? hi : lo;
      }
    }
  }
}

inline unsigned grid1(uint64_t n, int blk = kBlk) { return (unsigned)((n + blk - 1) / blk); }

// pre-order flattening (qbvh.rs:491-516).  The interior nodes below a GNode
// are counted first, so each child subtree knows where its pre-order range
// starts, and the top two levels hand their subtrees to separate threads
// (the output is the same as one depth-first pass).
inline uint32_t kids_of(const GNode& nd, uint32_t* kids) {
  uint32_t nk = 0;
  for (int side = 0; side < 2; ++side)
    for (uint32_t k = 0; k < nd.nkid[side]; ++k) kids[nk++] = nd.kid[side][k];
  return nk;
}

uint32_t count_interior(const std::vector<GNode>& g, uint32_t id, std::vector<uint32_t>& cnt, int par_depth) {
  uint32_t kids[4];
  const uint32_t nk = kids_of(g[id], kids);
  uint32_t c = nk ? 1 : 0;
  if (par_depth > 0 && nk > 1) {
    // a child whose thread cannot be started (thread limit, memory) is counted
    // on this thread instead: the counts do not depend on who computes them
    std::vector<std::thread> th;
    bool serial[4] = {false, false, false, false};
    for (uint32_t i = 1; i < nk; ++i) {
      try {
        th.emplace_back([&, i] { count_interior(g, kids[i], cnt, par_depth - 1); });
      } catch (const std::exception&) {
        serial[i] = true;
      }
    }
    count_interior(g, kids[0], cnt, par_depth - 1);
    for (uint32_t i = 1; i < nk; ++i)
      if (serial[i]) count_interior(g, kids[i], cnt, 0);
    for (auto& t : th) t.join();
    for (uint32_t i = 0; i < nk; ++i) c += cnt[kids[i]];
  } else {
    for (uint32_t i = 0; i < nk; ++i) c += count_interior(g, kids[i], cnt, 0);
  }
  cnt[id] = c;
  return c;
}

// Writes the subtree of GNode `id` with its root at out[idx]; returns the
// child reference (node index, or the leaf's flagged primitive range).
uint32_t flatten(const std::vector<GNode>& g, uint32_t id, const std::vector<uint32_t>& cnt, QbvhNodeHost* out,
                 uint32_t idx, int par_depth) {
  const GNode& nd = g[id];
  uint32_t kids[4];
  const uint32_t nk = kids_of(nd, kids);
  if (nk == 0) return kLeafFlag | (nd.count << 24) | nd.begin;
  uint32_t at[4], refs[4];
  at[0] = idx + 1;
  for (uint32_t i = 1; i < nk; ++i) at[i] = at[i - 1] + cnt[kids[i - 1]];
  if (par_depth > 0 && nk > 1) {
    // as in count_interior: a subtree whose thread cannot start is flattened
    // here; every subtree owns its pre-order range, so the tree is the same
    std::vector<std::thread> th;
    bool serial[4] = {false, false, false, false};
    for (uint32_t i = 1; i < nk; ++i) {
      try {
        th.emplace_back([&, i] { refs[i] = flatten(g, kids[i], cnt, out, at[i], par_depth - 1); });
      } catch (const std::exception&) {
        serial[i] = true;
      }
    }
    refs[0] = flatten(g, kids[0], cnt, out, at[0], par_depth - 1);
    for (uint32_t i = 1; i < nk; ++i)
      if (serial[i]) refs[i] = flatten(g, kids[i], cnt, out, at[i], 0);
    for (auto& t : th) t.join();
  } else {
    for (uint32_t i = 0; i < nk; ++i) refs[i] = flatten(g, kids[i], cnt, out, at[i], 0);
  }
  QbvhNodeHost nn;
  for (int s = 0; s < 4; ++s) {
    for (int k = 0; k < 3; ++k) {
      nn.b[k][s] = INFINITY;
      nn.b[3 + k][s] = -INFINITY;
    }
    nn.children[s] = kLeafFlag;
  }
  nn.valid_mask = 0;
  nn.reserved[0] = nn.reserved[1] = nn.reserved[2] = 0;
  for (uint32_t i = 0; i < nk; ++i) {
    const GNode& c = g[kids[i]];
    for (int k = 0; k < 3; ++k) {
      nn.b[k][i] = c.lo[k];
      nn.b[3 + k][i] = c.hi[k];
    }
    nn.children[i] = refs[i];
    nn.valid_mask |= 1u << i;
  }
  out[idx] = nn;
  return idx;
}

}  // namespace

// Builds the QBVH of n primitive boxes (device array, n x 6 floats: min xyz,
// max xyz) on the device; the result (nodes and primitive order) in `out`.
// Returns cudaErrorMemoryAllocation / cudaErrorInvalidValue on failure;
// capacity overflows (never expected) return cudaErrorLaunchOutOfResources.
cudaError_t build_qbvh_gpu(const float* d_bounds6, uint32_t n, QbvhHost* out, cudaStream_t s, cudaMemPool_t pool) {
  out->nodes.clear();
  out->prim_indices.clear();
  if (n == 0) return cudaErrorInvalidValue;
  const uint32_t large_cap = n / (kSeqMax / 2) + 16;
  const uint32_t seq_cap = n / 4 + 64;
  const uint32_t node_cap = 2 * n + 16;
  std::vector<void*> allocs;
  // stream-ordered allocations: with a pool that keeps its memory mapped,
  // later builds take them without mapping or synchronising
  auto take = [&](size_t bytes) -> void* {
    void* p = nullptr;
    const size_t b = std::max<size_t>(bytes, 16);
    if ((pool ? cudaMallocFromPoolAsync(&p, b, pool, s) : cudaMallocAsync(&p, b, s)) != cudaSuccess) return nullptr;
    allocs.push_back(p);
    return p;
  };
  auto release = [&]() {
    for (void* p : allocs) cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
  };
  BuildBuffers B{};
  B.n = n;
  B.box = (float*)take((size_t)6 * n * 4);
  B.cen = (float*)take((size_t)3 * n * 4);
  B.order = (uint32_t*)take((size_t)n * 4);
  B.order_tmp = (uint32_t*)take((size_t)n * 4);
  B.seg = (uint32_t*)take((size_t)n * 4);
  B.flag = (uint32_t*)take((size_t)(n + 1) * 4);
  B.scan = (uint32_t*)take((size_t)(n + 1) * 4);
  B.rpos = (uint32_t*)take((size_t)n * 4);
  B.ypos = (uint32_t*)take((size_t)n * 4);
  B.nodes = (GNode*)take((size_t)node_cap * sizeof(GNode));
  B.cnt = (Counters*)take(sizeof(Counters) + 16);
  Task* lists[2] = {(Task*)take((size_t)large_cap * sizeof(Task)), (Task*)take((size_t)large_cap * sizeof(Task))};
  Task* seq = (Task*)take((size_t)seq_cap * sizeof(Task));
  TaskAcc* acc = (TaskAcc*)take((size_t)large_cap * sizeof(TaskAcc));
  uint32_t* medians = (uint32_t*)take((size_t)large_cap * 4);
  uint32_t* overflow = (uint32_t*)take(16);
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, B.flag, B.scan, (int)(n + 1), s);
  void* scan_tmp = take(scan_bytes);
  for (void* p : allocs)
    if (!p) {
      release();
      return cudaErrorMemoryAllocation;
    }
  cudaError_t e = cudaSuccess;
  e = cudaMemsetAsync(B.nodes, 0, (size_t)node_cap * sizeof(GNode), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(overflow, 0, 16, s);
  k_prep<<<grid1(n), kBlk, 0, s>>>(d_bounds6, n, B);
  // the root: node 0 over the whole range
  Counters c0{0, 0, 1, 0};
  Task root{};
  root.begin = 0;
  root.count = n;
  root.role = kRoleNode;
  root.node = 0;
  root.next[0] = root.next[1] = kNoneG;
  uint32_t m = 0;
  if (n >= kSeqMax) {
    m = 1;
    if (e == cudaSuccess) e = cudaMemcpyAsync(lists[0], &root, sizeof root, cudaMemcpyHostToDevice, s);
  } else {
    c0.seq_tasks = 1;
    if (e == cudaSuccess) e = cudaMemcpyAsync(seq, &root, sizeof root, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(B.seg, 0xFF, (size_t)n * 4, s);  // no level ranges
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(B.cnt, &c0, sizeof c0, cudaMemcpyHostToDevice, s);
  Lists Ls{};
  Ls.seq = seq;
  Ls.next_cap = large_cap;
  Ls.seq_cap = seq_cap;
  Ls.node_cap = node_cap;
  Ls.overflow = overflow;
  std::vector<float> h_cen;
  int cur = 0;
  const uint32_t bin_chunk = 2048;
  while (e == cudaSuccess && m > 0) {
    Task* T = lists[cur];
    Ls.next = lists[cur ^ 1];
    const uint32_t acc_words = kAccFloats + 3 * kBinsG + 1;
    k_acc_init<<<grid1((uint64_t)m * acc_words), kBlk, 0, s>>>(T, m, acc);
    k_bounds<<<std::max(1u, std::min(grid1(n), 148u * 16u)), kBlk, 0, s>>>(B, acc);
    k_split_prep<<<grid1(m), kBlk, 0, s>>>(T, m, acc);
    k_bin<<<(n + bin_chunk - 1) / bin_chunk, kBlk, 0, s>>>(B, acc, bin_chunk);
    k_decide<<<grid1(m), kBlk, 0, s>>>(T, m, acc, B.nodes);
    k_flag<<<grid1((uint64_t)n + 1), kBlk, 0, s>>>(B, T);
    e = cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, B.flag, B.scan, (int)(n + 1), s);
    if (e != cudaSuccess) break;
    k_mid<<<grid1(m), kBlk, 0, s>>>(T, m, B);
    k_rpos<<<grid1(n), kBlk, 0, s>>>(B, T);
    k_perm<<<grid1(n), kBlk, 0, s>>>(B, T);
    k_copyback<<<grid1(n), kBlk, 0, s>>>(B, T);
    k_median_mark<<<grid1(m), kBlk, 0, s>>>(T, m, medians, B);
    Counters hc{};
    e = cudaMemcpyAsync(&hc, B.cnt, sizeof hc, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) break;
    if (hc.medians) {
      // make_leaf_or_force_split on large ranges (rare): sorted here
      std::vector<uint32_t> idx(hc.medians);
      std::vector<Task> ht(m);
      e = cudaMemcpyAsync(idx.data(), medians, hc.medians * 4, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(ht.data(), T, (size_t)m * sizeof(Task), cudaMemcpyDeviceToHost, s);
      if (h_cen.empty() && e == cudaSuccess) {
        h_cen.resize((size_t)3 * n);
        e = cudaMemcpyAsync(h_cen.data(), B.cen, (size_t)3 * n * 4, cudaMemcpyDeviceToHost, s);
      }
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      for (uint32_t k = 0; e == cudaSuccess && k < hc.medians; ++k) {
        const Task& tk = ht[idx[k]];
        GNode g;
        e = cudaMemcpyAsync(&g, B.nodes + tk.node, sizeof g, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) break;
        const float ex = g.hi[0] - g.lo[0], ey = g.hi[1] - g.lo[1], ez = g.hi[2] - g.lo[2];
        const int axis = (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
        std::vector<uint32_t> ord(tk.count);
        e = cudaMemcpyAsync(ord.data(), B.order + tk.begin, (size_t)tk.count * 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) break;
        const float* cn = h_cen.data() + (size_t)axis * n;
        std::sort(ord.begin(), ord.end(), [cn](uint32_t x, uint32_t y) {
          if (cn[x] < cn[y]) return true;
          if (cn[y] < cn[x]) return false;
          return x < y;
        });
        e = cudaMemcpyAsync(B.order + tk.begin, ord.data(), (size_t)tk.count * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      }
      if (e != cudaSuccess) break;
    }
    k_emit<<<grid1(m), kBlk, 0, s>>>(T, m, B, Ls);
    k_seg<<<grid1(n), kBlk, 0, s>>>(B, T);
    uint32_t ov = 0;
    e = cudaMemcpyAsync(&hc, B.cnt, sizeof hc, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ov, overflow, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && ov) e = cudaErrorLaunchOutOfResources;
    if (e != cudaSuccess) break;
    m = hc.next_tasks;
    hc.next_tasks = 0;
    hc.medians = 0;
    e = cudaMemcpyAsync(B.cnt, &hc, sizeof hc, cudaMemcpyHostToDevice, s);
    cur ^= 1;
  }
  Counters hc{};
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hc, B.cnt, sizeof hc, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && hc.seq_tasks > seq_cap) e = cudaErrorLaunchOutOfResources;
  if (e == cudaSuccess && hc.seq_tasks) {
    Ls.next = lists[cur];
    k_seq<<<grid1(hc.seq_tasks, 128), 128, 0, s>>>(seq, hc.seq_tasks, B, Ls);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hc, B.cnt, sizeof hc, cudaMemcpyDeviceToHost, s);
  uint32_t ov = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&ov, overflow, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && (ov || hc.nodes > node_cap)) e = cudaErrorLaunchOutOfResources;
  std::vector<GNode> g;
  if (e == cudaSuccess) {
    g.resize(hc.nodes);
    out->prim_indices.resize(n);
    e = cudaMemcpyAsync(g.data(), B.nodes, (size_t)hc.nodes * sizeof(GNode), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out->prim_indices.data(), B.order, (size_t)n * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  release();
  if (e != cudaSuccess) {
    out->prim_indices.clear();
    return e;
  }
  // two threaded levels (up to 16 subtrees) once the tree is large enough to gain
  const int par_depth = g.size() >= (1u << 16) ? 2 : 0;
  std::vector<uint32_t> cnt(g.size());
  out->nodes.resize(count_interior(g, 0, cnt, par_depth));
  flatten(g, 0, cnt, out->nodes.data(), 0, par_depth);
  return cudaSuccess;
}

}  // namespace tpt
