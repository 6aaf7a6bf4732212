// Oracle C entry points for rendering (test infrastructure only).
#include <cmath>
#include <cstring>

#include "render.h"

using namespace orc;

extern "C" {

// Takes ownership of nothing: copies the geometry handle's contents.
void* orc_render_scene_create(void* geometry) {
  auto* s = new RenderScene();
  s->geo = *(Geometry*)geometry;
  return s;
}
void orc_render_scene_free(void* h) { delete (RenderScene*)h; }

// kind, rho[3], color[3], strength per material
void orc_render_scene_set_materials(void* h, const uint32_t* kinds, const float* rho, const float* color,
                                    const float* strength, uint32_t n) {
  auto* s = (RenderScene*)h;
  s->materials.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    s->materials[i].kind = kinds[i];
    s->materials[i].rho = Vec3(rho[3 * i], rho[3 * i + 1], rho[3 * i + 2]);
    s->materials[i].color = Vec3(color[3 * i], color[3 * i + 1], color[3 * i + 2]);
    s->materials[i].strength = strength[i];
  }
}

// NormalizedLambert / Emissive opacity per material (1 = opaque; OpenPBR
// materials take geometry_opacity from their parameters).  Call before the
// light tree (which finalises).
void orc_render_scene_set_opacity(void* h, const float* opacity, uint32_t n) {
  auto* s = (RenderScene*)h;
  for (uint32_t i = 0; i < n && i < s->materials.size(); ++i) s->materials[i].opacity = opacity[i];
}

// Scene::closest_hit with an AuxRng per ray (scene/mod.rs:340-395, 686-723):
// rays n x 6 (origin, direction); aux: the AuxRng states, advanced in place by
// the alpha tests' draws; out: instance, triangle (-1: miss), t per ray.
void orc_render_scene_closest_alpha(void* h, const float* rays, uint64_t n, uint32_t* aux, int32_t* inst,
                                    int32_t* tri, float* t) {
  const auto* s = (const RenderScene*)h;
  for (uint64_t i = 0; i < n; ++i) {
    Ray r;
    r.origin = Vec3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
    r.direction = Vec3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
    AuxRng a(0);
    a.state = aux[i];
    SceneHit hit;
    const bool found = s->geo.closest_hit(r, &hit, nullptr, &a);
    aux[i] = a.state;
    inst[i] = found ? hit.instance : -1;
    tri[i] = found ? hit.triangle : -1;
    t[i] = found ? hit.t : kInf;
  }
}

// Point lights: n x 7 floats (position, color, intensity); spot lights: n x 12
// (position, direction, color, intensity, total width, falloff start in
// radians: SpotLight::new); directional: n x 7 (direction, color, intensity:
// DirectionalLight::new).  Call before the light tree (which finalises).
void orc_render_scene_set_lights(void* h, const float* points, uint32_t np, const float* spots, uint32_t ns,
                                 const float* dirs, uint32_t nd) {
  auto* s = (RenderScene*)h;
  s->points.resize(np);
  for (uint32_t i = 0; i < np; ++i) {
    const float* a = points + 7 * i;
    s->points[i] = PointLight{Vec3(a[0], a[1], a[2]), Vec3(a[3], a[4], a[5]), a[6]};
  }
  const float pi = 3.14159274101257324f;
  s->spots.resize(ns);
  for (uint32_t i = 0; i < ns; ++i) {
    const float* a = spots + 12 * i;
    float total_width = clampf(a[10], 0.0f, pi);
    float falloff_start = clampf(a[11], 0.0f, total_width);
    Vec3 d(a[3], a[4], a[5]);
    s->spots[i] = SpotLight{Vec3(a[0], a[1], a[2]), d * (1.0f / length(d)), Vec3(a[6], a[7], a[8]), a[9],
                            std::cos(total_width), std::cos(falloff_start)};
  }
  s->dirs.resize(nd);
  for (uint32_t i = 0; i < nd; ++i) {
    const float* a = dirs + 7 * i;
    Vec3 d(a[0], a[1], a[2]);
    s->dirs[i] = DirLight{d * (1.0f / length(d)), Vec3(a[3], a[4], a[5]), a[6]};
  }
}

// Light tree nodes in the 64-byte tpt_light_node layout.
void orc_render_scene_set_light_tree(void* h, const void* nodes, uint64_t n, uint32_t root) {
  auto* s = (RenderScene*)h;
  s->tree.resize(n);
  if (n) std::memcpy(s->tree.data(), nodes, n * sizeof(LightNode));
  s->root = root;
  s->finalize();
}

static RenderJob make_job(const float* cam11, uint32_t w, uint32_t hgt, uint32_t spp, uint32_t depth,
                          uint32_t integrator, uint32_t seed) {
  RenderJob j;
  j.cam = Camera::make(Vec3(cam11[0], cam11[1], cam11[2]), Vec3(cam11[3], cam11[4], cam11[5]),
                       Vec3(cam11[6], cam11[7], cam11[8]), cam11[9], cam11[10]);
  j.width = w;
  j.height = hgt;
  j.spp = spp;
  j.max_depth = depth;
  j.integrator = integrator;
  j.seed = seed;
  return j;
}

// cam11: eye(3) look_at(3) up(3) fov_y exposure
void orc_render_pixels(void* h, const float* cam11, uint32_t w, uint32_t hgt, uint32_t spp, uint32_t depth,
                       uint32_t integrator, uint32_t p0, uint32_t p1, float* out, int nthreads, uint32_t seed) {
  render_pixels(*(RenderScene*)h, make_job(cam11, w, hgt, spp, depth, integrator, seed), p0, p1, out, nthreads);
}

void orc_render_samples(void* h, const float* cam11, uint32_t w, uint32_t hgt, uint32_t spp, uint32_t depth,
                        uint32_t integrator, uint64_t first, uint64_t count, float* out, int nthreads,
                        uint32_t seed) {
  render_samples(*(RenderScene*)h, make_job(cam11, w, hgt, spp, depth, integrator, seed), first, count, out,
                 nthreads);
}

}  // extern "C"
