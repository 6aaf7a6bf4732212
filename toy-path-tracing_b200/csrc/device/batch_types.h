// Scene + job records the render kernels read: one DevRender per scene, and for
// batched wavefront renders (many jobs of uneven size in one launch sequence)
// one DevJob per job in a device array.  Plain structs: g++ and nvcc both
// compile this header.
#pragma once
#include <cstdint>

#include "dev_types.cuh"
#include "render_types.h"

namespace tpt {

struct DevRender {
  DevGeometry geo;
  DevRenderData d;
};

// One job of a batch.  The batch's paths form one index space: job j owns
// global paths [path_base, path_base + width * height * spp) (path = pixel *
// spp + sample within the job) and global pixels [pixel_base, pixel_base +
// width * height).  Jobs are sorted by path_base.
struct DevJob {
  DevRender render;
  RenderLaunch P;
  uint64_t path_base;
  uint64_t pixel_base;
  float* out;  // the job's image (device, width * height * 3)
  uint64_t pad;
};

}  // namespace tpt
