// Host-side types shared by the scene builder, the uploader and the C ABI.
#pragma once
#include <cstdint>
#include <vector>

namespace tpt {

// Leaf child words: bit 31 set, 7-bit primitive count at bit 24, 24-bit
// primitive offset (crates/renderer/src/qbvh.rs:15-51).
constexpr uint32_t kLeafFlag = 1u << 31;
constexpr uint32_t kEmptyWord = kLeafFlag;

// Same bytes as `tpt_qbvh_node` in include/tpt.h.
struct QbvhNodeHost {
  float b[6][4];  // min_x, min_y, min_z, max_x, max_y, max_z lanes
  uint32_t children[4];
  uint32_t valid_mask;
  uint32_t reserved[3];
};
static_assert(sizeof(QbvhNodeHost) == 128, "node is one 128-byte line");

struct QbvhHost {
  std::vector<QbvhNodeHost> nodes;
  std::vector<uint32_t> prim_indices;
};

bool build_qbvh_host(const float* bounds6, uint32_t n, int threads, QbvhHost* out);

}  // namespace tpt
