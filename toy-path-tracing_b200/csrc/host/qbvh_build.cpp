// Host-side 4-wide BVH builder (binned SAH, 16 bins, leaf target 4 / max 16).
//
// Produces exactly the node array and primitive order of the reference
// builder `build_qbvh` (crates/renderer/src/qbvh.rs:144-516): same binning
// arithmetic, same split rules, same pre-order flattening.  The reference
// parallelises subtrees with rayon; this builder runs independent subtrees on
// a pool of std::threads, which does not change the result because every
// subtree is built from its own disjoint primitive range.  The forced median
// split (qbvh.rs:265-301) orders equal centroids by primitive index.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "host_types.h"

namespace tpt {
namespace {

constexpr int kBins = 16;
constexpr uint32_t kLeafTarget = 4;
constexpr uint32_t kLeafMax = 16;
constexpr uint32_t kParallelMin = 4096;

struct Box {
  float lo[3], hi[3];
};

inline float minnum(float a, float b) { return std::fmin(a, b); }
inline float maxnum(float a, float b) { return std::fmax(a, b); }

inline Box box_empty() {
  const float inf = INFINITY;
  return Box{{inf, inf, inf}, {-inf, -inf, -inf}};
}
inline void box_grow(Box& a, const Box& b) {
  for (int k = 0; k < 3; ++k) {
    a.lo[k] = minnum(a.lo[k], b.lo[k]);
    a.hi[k] = maxnum(a.hi[k], b.hi[k]);
  }
}
inline float box_area(const Box& b) {
  float e[3];
  for (int k = 0; k < 3; ++k) e[k] = maxnum(b.hi[k] - b.lo[k], 0.0f);
  return 2.0f * (e[0] * e[1] + e[0] * e[2] + e[1] * e[2]);
}

// Tree under construction: node kinds kept in flat vectors so worker threads
// only touch their own subtree's slots.
struct BuildTree {
  struct Node {
    Box box;
    uint32_t begin = 0, count = 0;  // primitive range (valid for leaves)
    std::vector<std::unique_ptr<Node>> kids;
    bool leaf() const { return kids.empty(); }
  };
};
using BNode = BuildTree::Node;

class Builder {
 public:
  Builder(const float* bounds6, uint32_t n) : n_(n) {
    prim_box_.resize(n);
    centroid_.resize(3 * (size_t)n);
    order_.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
      Box b;
      for (int k = 0; k < 3; ++k) {
        b.lo[k] = bounds6[6 * (size_t)i + k];
        b.hi[k] = bounds6[6 * (size_t)i + 3 + k];
        centroid_[3 * (size_t)i + k] = 0.5f * (b.lo[k] + b.hi[k]);
      }
      prim_box_[i] = b;
      order_[i] = i;
    }
  }

  std::unique_ptr<BNode> run(int threads) {
    threads_ = std::max(1, threads);
    auto root = std::make_unique<BNode>();
    pending_.store(1);
    submit([this, r = root.get()] { node_task(r, 0, n_); });
    worker_loop_until_done();
    return root;
  }

  const std::vector<uint32_t>& order() const { return order_; }

 private:
  // ---- task pool -------------------------------------------------------
  void submit(std::function<void()> f) {
    std::lock_guard<std::mutex> g(mu_);
    tasks_.push_back(std::move(f));
    cv_.notify_one();
  }
  void worker_loop_until_done() {
    std::vector<std::thread> pool;
    for (int i = 1; i < threads_; ++i) {
      try {
        pool.emplace_back([this] { work(); });
      } catch (const std::exception&) {
        break;  // fewer workers (thread limit): the tasks are the same, the tree too
      }
    }
    work();
    for (auto& t : pool) t.join();
  }
  void work() {
    for (;;) {
      std::function<void()> f;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [this] { return !tasks_.empty() || pending_.load() == 0; });
        if (tasks_.empty()) return;
        f = std::move(tasks_.back());
        tasks_.pop_back();
      }
      f();
      if (pending_.fetch_sub(1) == 1) {
        std::lock_guard<std::mutex> g(mu_);
        cv_.notify_all();
      }
    }
  }
  // Run `f` now or hand it to the pool.
  void spawn_or_run(uint32_t count, std::function<void()> f) {
    if (threads_ > 1 && count >= kParallelMin) {
      pending_.fetch_add(1);
      submit(std::move(f));
    } else {
      f();
    }
  }

  // ---- geometry helpers -------------------------------------------------
  Box range_box(uint32_t b, uint32_t n) const {
    Box r = box_empty();
    for (uint32_t i = b; i < b + n; ++i) box_grow(r, prim_box_[order_[i]]);
    return r;
  }
  Box range_centroid_box(uint32_t b, uint32_t n) const {
    Box r = box_empty();
    for (uint32_t i = b; i < b + n; ++i) {
      const float* c = &centroid_[3 * (size_t)order_[i]];
      Box cb{{c[0], c[1], c[2]}, {c[0], c[1], c[2]}};
      box_grow(r, cb);
    }
    return r;
  }
  static uint32_t bin_of(float c, float cmin, float scale) {
    float raw = (c - cmin) * scale;
    if (std::isnan(raw)) return 0;
    if (raw < 0.0f) raw = 0.0f;
    if (raw > (float)(kBins - 1)) raw = (float)(kBins - 1);
    return (uint32_t)raw;
  }

  struct Split {
    int axis = -1;
    float cmin = 0, cmax = 0;
    int bin = 0;
    float cost = INFINITY;
  };

  // SAH sweep over 16 bins per axis; an axis is kept only when strictly cheaper.
  bool best_split(uint32_t b, uint32_t n, const Box& parent, Split* out) const {
    if (n <= 1) return false;
    Box cb = range_centroid_box(b, n);
    float parent_area = maxnum(box_area(parent), 1.0e-30f);
    bool found = false;
    for (int axis = 0; axis < 3; ++axis) {
      float cmin = cb.lo[axis], cmax = cb.hi[axis];
      if (cmax - cmin <= 0.0f) continue;
      float scale = (float)kBins / maxnum(cmax - cmin, 1.0e-30f);
      Box bin_box[kBins];
      uint32_t bin_cnt[kBins] = {0};
      for (int i = 0; i < kBins; ++i) bin_box[i] = box_empty();
      for (uint32_t i = b; i < b + n; ++i) {
        uint32_t p = order_[i];
        uint32_t k = bin_of(centroid_[3 * (size_t)p + axis], cmin, scale);
        box_grow(bin_box[k], prim_box_[p]);
        bin_cnt[k] += 1;
      }
      Box suffix_box[kBins];
      Box acc = box_empty();
      for (int i = kBins - 1; i >= 0; --i) { box_grow(acc, bin_box[i]); suffix_box[i] = acc; }
      uint32_t total = 0;
      for (int i = 0; i < kBins; ++i) total += bin_cnt[i];
      if (total <= 1) continue;
      Box pre = box_empty();
      uint32_t left = 0;
      float best = INFINITY;
      int best_bin = -1;
      for (int s = 0; s < kBins - 1; ++s) {
        box_grow(pre, bin_box[s]);
        left += bin_cnt[s];
        uint32_t right = total - left;
        if (left == 0 || right == 0) continue;
        float cost = 1.0f + 1.0f * (box_area(pre) * (float)left + box_area(suffix_box[s + 1]) * (float)right) /
                                parent_area;
        if (cost < best) { best = cost; best_bin = s; }
      }
      if (best_bin < 0) continue;
      if (!found || best < out->cost) {
        out->axis = axis; out->cmin = cmin; out->cmax = cmax; out->bin = best_bin; out->cost = best;
        found = true;
      }
    }
    return found;
  }

  // Hoare-style sweep identical to the reference: left-side primitives stay,
  // others are swapped with the shrinking right end.
  uint32_t partition(uint32_t b, uint32_t n, const Split& s) {
    float scale = (float)kBins / maxnum(s.cmax - s.cmin, 1.0e-30f);
    uint32_t l = b, r = b + n;
    while (l < r) {
      uint32_t k = bin_of(centroid_[3 * (size_t)order_[l] + s.axis], s.cmin, scale);
      if ((int)k <= s.bin) ++l;
      else { --r; std::swap(order_[l], order_[r]); }
    }
    return l - b;
  }

  void make_leaf(BNode* node, uint32_t b, uint32_t n, const Box& box) {
    node->box = box; node->begin = b; node->count = n;
  }

  // build_qbvh_node (qbvh.rs:186-223): a node gets up to two children from each
  // side of its best binary split.
  void node_task(BNode* node, uint32_t b, uint32_t n) {
    Box box = range_box(b, n);
    if (n <= kLeafTarget) { make_leaf(node, b, n, box); return; }
    Split s;
    if (!best_split(b, n, box, &s)) { leaf_or_median(node, b, n, box); return; }
    if (s.cost >= 1.0f * (float)n && n <= kLeafMax) { make_leaf(node, b, n, box); return; }
    uint32_t mid = partition(b, n, s);
    if (mid == 0 || mid == n) { leaf_or_median(node, b, n, box); return; }
    node->box = box;
    expand_side(node, b, mid);
    expand_side(node, b + mid, n - mid);
  }

  // make_leaf_or_force_split (qbvh.rs:265-301)
  void leaf_or_median(BNode* node, uint32_t b, uint32_t n, const Box& box) {
    if (n <= kLeafMax) { make_leaf(node, b, n, box); return; }
    uint32_t mid = n / 2;
    float e[3] = {box.hi[0] - box.lo[0], box.hi[1] - box.lo[1], box.hi[2] - box.lo[2]};
    int axis = (e[0] >= e[1] && e[0] >= e[2]) ? 0 : (e[1] >= e[2] ? 1 : 2);
    const float* cen = centroid_.data();
    std::sort(order_.begin() + b, order_.begin() + b + n, [cen, axis](uint32_t x, uint32_t y) {
      float cx = cen[3 * (size_t)x + axis], cy = cen[3 * (size_t)y + axis];
      if (cx < cy) return true;
      if (cy < cx) return false;
      return x < y;
    });
    node->box = box;
    expand_side(node, b, mid);
    expand_side(node, b + mid, n - mid);
  }

  // split_into_children (qbvh.rs:229-263): one side becomes one or two children.
  void expand_side(BNode* parent, uint32_t b, uint32_t n) {
    if (n == 0) return;
    Box box = range_box(b, n);
    auto single = [&]() {
      parent->kids.push_back(std::make_unique<BNode>());
      BNode* c = parent->kids.back().get();
      node_task(c, b, n);
    };
    if (n <= kLeafTarget) { single(); return; }
    Split s;
    if (!best_split(b, n, box, &s)) { single(); return; }
    if (s.cost >= 1.0f * (float)n && n <= kLeafMax) { single(); return; }
    uint32_t mid = partition(b, n, s);
    if (mid == 0 || mid == n) { single(); return; }
    parent->kids.push_back(std::make_unique<BNode>());
    parent->kids.push_back(std::make_unique<BNode>());
    BNode* l = parent->kids[parent->kids.size() - 2].get();
    BNode* r = parent->kids.back().get();
    uint32_t nr = n - mid;
    spawn_or_run(mid, [this, l, b, mid] { node_task(l, b, mid); });
    spawn_or_run(nr, [this, r, b, mid, nr] { node_task(r, b + mid, nr); });
  }

  uint32_t n_;
  int threads_ = 1;
  std::vector<Box> prim_box_;
  std::vector<float> centroid_;
  std::vector<uint32_t> order_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::vector<std::function<void()>> tasks_;
  std::atomic<int> pending_{0};
};

// Pre-order flattening (qbvh.rs:491-516); returns the child word for `node`.
uint32_t emit(const BNode* node, std::vector<QbvhNodeHost>& out) {
  if (node->leaf()) return kLeafFlag | (node->count << 24) | node->begin;
  uint32_t idx = (uint32_t)out.size();
  out.emplace_back();
  QbvhNodeHost nn;
  for (int s = 0; s < 4; ++s) {
    for (int k = 0; k < 3; ++k) { nn.b[k][s] = INFINITY; nn.b[3 + k][s] = -INFINITY; }
    nn.children[s] = kLeafFlag;
  }
  nn.valid_mask = 0;
  nn.reserved[0] = nn.reserved[1] = nn.reserved[2] = 0;
  for (size_t i = 0; i < node->kids.size(); ++i) {
    const BNode* c = node->kids[i].get();
    uint32_t ref = emit(c, out);
    for (int k = 0; k < 3; ++k) { nn.b[k][i] = c->box.lo[k]; nn.b[3 + k][i] = c->box.hi[k]; }
    nn.children[i] = ref;
    nn.valid_mask |= 1u << i;
  }
  out[idx] = nn;
  return idx;
}

// Leaves store their absolute primitive offset, which equals the running
// offset of the reference's flattening because leaves are laid out in
// pre-order over contiguous ranges.
}  // namespace

bool build_qbvh_host(const float* bounds6, uint32_t n, int threads, QbvhHost* out) {
  out->nodes.clear();
  out->prim_indices.clear();
  if (n == 0) return false;
  Builder b(bounds6, n);
  std::unique_ptr<BNode> root = b.run(threads);
  out->prim_indices = b.order();
  emit(root.get(), out->nodes);
  return true;
}

}  // namespace tpt
