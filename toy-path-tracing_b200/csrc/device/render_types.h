// Render-side device records shared by host (upload) and device code.  Plain
// structs only, so both g++ and nvcc compile this header.
#pragma once
#include <cstdint>

namespace tpt {

struct DevLightNodeRec {
  float flux;
  float mu[3];
  float sigma_s2;
  float nu[3];
  float lambda;
  float radius;
  uint32_t left, right, parent;
  uint32_t leaf_instance, leaf_triangle;
  float area;
};
static_assert(sizeof(DevLightNodeRec) == 64, "light node layout");

enum DevMatKind : uint32_t { kDevLambert = 0, kDevEmissive = 1, kDevOpenPbr = 2 };

struct alignas(16) DevMaterialRec {
  uint32_t kind;
  float rho[3];
  float color[3];
  float strength;
  uint32_t openpbr;  // index into the OpenPBR parameter table
  uint32_t pad[7];
};
static_assert(sizeof(DevMaterialRec) == 64, "material record");

struct alignas(16) DevShadeInstance {
  float l2w[12];  // local_to_world affine columns c0..c3 (xyz each)
  float n2w[9];   // normal_to_world, column-major
  uint32_t mesh;
  uint32_t material;
  uint32_t leaf_base;  // first emitter-map slot of this instance, or 0xFFFFFFFF
  uint32_t pad[8];
};
static_assert(sizeof(DevShadeInstance) == 128, "shade instance record");

struct DevMeshInfo {
  uint32_t vtx_base, idx_base, num_tris, flags;  // flags bit 0: normals, bit 1: uvs
};

struct DevRenderData {
  const DevShadeInstance* inst;
  const DevMeshInfo* meshes;
  const float* pos;
  const float* nrm;
  const float* uv;
  const uint32_t* idx;
  const DevMaterialRec* mats;
  const DevLightNodeRec* ltree;
  const uint32_t* emitter_leaf;
  const void* openpbr;  // OpenPBR parameter table
  uint32_t ltree_root;
  uint32_t has_tree;
  float tree_cat_pmf;  // LightSampler pmf of the Tree category
  uint32_t num_materials;
};

// Camera constants computed on the host (scene/camera.rs:21-39).
struct DevCamera {
  float eye[3], forward[3], right[3], up[3];
  float tan_half_fov_y;
  float exposure;
};

struct RenderLaunch {
  DevCamera cam;
  uint32_t width, height, spp, max_depth;
  uint32_t log2_spp, n_base4_digits;
  uint32_t integrator;  // 0 = MIS
  uint32_t pad;
};

// Wavefront state: per path slot of a chunk (capacity slots), two ray queues,
// the hit records of the current queue and the shadow queue.  Planes of a
// structured array are `capacity` elements apart.
struct WfBuffers {
  uint32_t capacity;
  float* beta;        // 3 planes
  float* L;           // 3 planes
  float* prev;        // 7 planes: previous vertex p (3), ns (3), BSDF pdf
  uint32_t* prev_mat; // previous vertex material index, bit 31 = delta sample
  uint32_t* depth;    // vertices processed
  uint32_t* q_slot[2];
  float* q_ray[2];    // 7 planes each: o, d, tmax
  int32_t* h_tri;
  int32_t* h_inst;
  float* h_t;
  float* h_bary;      // 3 planes
  uint32_t* s_slot;
  float* s_ray;       // 7 planes
  float* s_contrib;   // 3 planes
  uint32_t* s_target; // 2 planes: instance, triangle
  int32_t* s_tri;
  int32_t* s_inst;
  float* s_t;
  uint32_t* counts;   // [0], [1]: ray queue lengths, [2]: shadow queue length
};

}  // namespace tpt
