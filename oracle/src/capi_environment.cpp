// Oracle (test infrastructure): C entry points of the environment light, for
// the Python tests (the reference's environment.rs unit tests run against
// them) and for installing a map in an oracle render scene.
#include <cstring>

#include "environment.h"
#include "render.h"

using namespace orc;

extern "C" {

// EnvironmentLight::from_pixels; rgb: width * height * 3 floats.
void* orc_env_create(uint32_t width, uint32_t height, const float* rgb, float scale, float rotate_y) {
  return new Environment(Environment::from_pixels(width, height, rgb, scale, rotate_y));
}
void orc_env_free(void* h) { delete (Environment*)h; }

float orc_env_total_power(void* h) { return ((Environment*)h)->total_power(); }

void orc_env_radiance(void* h, const float* dir, float* out3) {
  const Vec3 r = ((Environment*)h)->radiance(Vec3(dir[0], dir[1], dir[2]));
  out3[0] = r.x;
  out3[1] = r.y;
  out3[2] = r.z;
}

// compensated: 0 the plain distribution, 1 the MIS-compensated one
float orc_env_pdf(void* h, const float* dir, int compensated) {
  const Environment* e = (Environment*)h;
  const Vec3 d(dir[0], dir[1], dir[2]);
  return compensated ? e->pdf_mis_compensated(d) : e->pdf(d);
}

// out9: direction (3), radiance (3), u, v, pdf; returns 0 when there is no sample
int orc_env_sample(void* h, float u, float v, int compensated, float* out9) {
  const Environment* e = (Environment*)h;
  EnvSample s;
  const bool ok = compensated ? e->sample_mis_compensated(u, v, &s) : e->sample(u, v, &s);
  if (!ok) return 0;
  const float vals[9] = {s.direction.x, s.direction.y, s.direction.z, s.radiance.x, s.radiance.y, s.radiance.z,
                         s.u, s.v, s.pdf};
  std::memcpy(out9, vals, sizeof vals);
  return 1;
}

void orc_env_direction_to_uv(const float* dir, float* uv) { env_direction_to_uv(Vec3(dir[0], dir[1], dir[2]), uv, uv + 1); }
void orc_env_uv_to_direction(float u, float v, float* dir) {
  const Vec3 d = env_uv_to_direction(u, v);
  dir[0] = d.x;
  dir[1] = d.y;
  dir[2] = d.z;
}

// Pyramid of one distribution: number of levels; dims (2 per level, coarsest
// first) and total weight when the pointers are given; leaf weights (padded
// width x height) into `leaf` when given.
uint32_t orc_env_pyramid(void* h, int compensated, uint32_t* dims, float* total, float* leaf) {
  const Environment* e = (Environment*)h;
  const EnvDistribution& d = compensated ? e->mis : e->dist;
  if (dims)
    for (size_t l = 0; l < d.levels.size(); ++l) {
      dims[2 * l] = d.levels[l].width;
      dims[2 * l + 1] = d.levels[l].height;
    }
  if (total) *total = d.total_weight;
  if (leaf) std::memcpy(leaf, d.levels.back().weights.data(), d.levels.back().weights.size() * sizeof(float));
  return (uint32_t)d.levels.size();
}

// Scene::set_environment_light on an oracle render scene (before its light
// tree is installed, which builds the light sampler).
void orc_render_scene_set_environment(void* scene, uint32_t width, uint32_t height, const float* rgb, float scale,
                                      float rotate_y) {
  auto* s = (RenderScene*)scene;
  s->env = Environment::from_pixels(width, height, rgb, scale, rotate_y);
  s->has_env = true;
}

}  // extern "C"
