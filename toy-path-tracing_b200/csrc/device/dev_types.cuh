// Device-resident scene layout.
//
// HBM layout (all arrays 128-byte aligned):
//  - nodes:    every BLAS and the TLAS, 128 B per 4-wide node (one cache line):
//              six float4 lane vectors (min_x, min_y, min_z, max_x, max_y,
//              max_z) then one uint4 of child words.  Child words keep the
//              reference encoding (qbvh.rs:15-51) but are relative to the
//              owning structure: interior = node index from its node base,
//              leaf = offset from its primitive base.  Empty lanes hold
//              0x80000000 and are skipped without a box test.
//  - tris:     per mesh, triangles in BLAS leaf order, 48 B each: v0.xyz +
//              triangle index, v1.xyz + degenerate flag, v2.xyz + 0.
//  - instances: 64 B each: world_to_local as 4 columns of 3 floats (glam
//              transform_point3 order), BLAS node base, triangle base, root
//              word and material.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tpt {

constexpr uint32_t kLeafBit = 1u << 31;
constexpr uint32_t kEmptyChild = kLeafBit;
constexpr int kStackDepth = 128;  // qbvh.rs:609

struct __align__(128) DevNode {
  float4 lo_x, lo_y, lo_z, hi_x, hi_y, hi_z;
  uint4 child;
  uint4 pad;
};
static_assert(sizeof(DevNode) == 128, "node is one line");

struct __align__(16) DevTri {
  float4 v0;  // w = triangle index (bits)
  float4 v1;  // w = 1.0 when degenerate (cross(v2-v0, v1-v0) has zero length)
  float4 v2;
};

struct __align__(16) DevInstance {
  float4 m0;  // c0.x c0.y c0.z c1.x
  float4 m1;  // c1.y c1.z c2.x c2.y
  float4 m2;  // c2.z c3.x c3.y c3.z
  uint32_t node_base;
  uint32_t tri_base;
  uint32_t root_word;  // node index 0, or a leaf word when the BLAS has no nodes
  uint32_t material;
};
static_assert(sizeof(DevInstance) == 64, "instance record");

struct DevGeometry {
  const DevNode* nodes;
  const DevTri* tris;
  const DevInstance* instances;
  const uint32_t* tlas_prims;  // TLAS primitive_indices (instance ids)
  uint32_t tlas_node_base;
  uint32_t tlas_root_word;
  uint32_t num_instances;
  uint32_t pad;
  // per instance: the opacity its material's alpha test compares an AuxRng
  // draw with (1: no alpha test); NULL when no instance has one
  const float* inst_alpha;
};

// Device-side error word (bit flags), read back by the host after each call.
enum DevError : uint32_t {
  kDevErrStackOverflow = 1u << 0,
  kDevErrBadIndex = 1u << 1,
  kDevErrTimeout = 1u << 2,
  kDevErrCapacity = 1u << 3,
};

}  // namespace tpt
