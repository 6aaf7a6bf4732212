// Oracle C entry points for geometry, sampler and camera (called from Python
// tests through ctypes; test infrastructure only).
#include <thread>
#include <atomic>
#include "camera.h"
#include "sampler.h"

using namespace orc;

namespace {
template <class F>
void parallel_for(uint64_t n, int nthreads, F&& f) {
  if (nthreads <= 1 || n < 256) {
    for (uint64_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<uint64_t> next{0};
  const uint64_t chunk = 64;
  std::vector<std::thread> ts;
  for (int t = 0; t < nthreads; ++t)
    ts.emplace_back([&]() {
      for (;;) {
        uint64_t s = next.fetch_add(chunk);
        if (s >= n) break;
        uint64_t e = std::min(n, s + chunk);
        for (uint64_t i = s; i < e; ++i) f(i);
      }
    });
  for (auto& t : ts) t.join();
}

Ray ray_from_soa(const float* rays, uint64_t n, uint64_t i) {
  Ray r;
  r.origin = Vec3(rays[i], rays[n + i], rays[2 * n + i]);
  r.direction = Vec3(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]);
  return r;
}
}  // namespace

extern "C" {

// ---- primitives ----------------------------------------------------------
int orc_intersect_triangle(const float* ray6, float t_max, const float* v9, float* out4) {
  Ray r;
  r.origin = Vec3(ray6[0], ray6[1], ray6[2]);
  r.direction = Vec3(ray6[3], ray6[4], ray6[5]);
  TriHit h;
  if (!intersect_triangle(r, t_max, Vec3(v9[0], v9[1], v9[2]), Vec3(v9[3], v9[4], v9[5]),
                          Vec3(v9[6], v9[7], v9[8]), &h))
    return 0;
  out4[0] = h.t; out4[1] = h.bary.x; out4[2] = h.bary.y; out4[3] = h.bary.z;
  return 1;
}

// ---- standalone QBVH over boxes (qbvh.rs tests) --------------------------
void* orc_qbvh_build(const float* bounds6, uint64_t n) {
  std::vector<Bounds> b(n);
  for (uint64_t i = 0; i < n; ++i) {
    b[i].min = Vec3(bounds6[6 * i], bounds6[6 * i + 1], bounds6[6 * i + 2]);
    b[i].max = Vec3(bounds6[6 * i + 3], bounds6[6 * i + 4], bounds6[6 * i + 5]);
  }
  auto* q = new Qbvh();
  if (!build_qbvh(b, q)) { delete q; return nullptr; }
  return q;
}
void orc_qbvh_free(void* h) { delete (Qbvh*)h; }
uint64_t orc_qbvh_num_nodes(void* h) { return ((Qbvh*)h)->nodes.size(); }
uint64_t orc_qbvh_num_prims(void* h) { return ((Qbvh*)h)->primitive_indices.size(); }
void orc_qbvh_copy(void* h, void* nodes_out, uint32_t* prims_out) {
  Qbvh* q = (Qbvh*)h;
  if (nodes_out && !q->nodes.empty()) std::memcpy(nodes_out, q->nodes.data(), q->nodes.size() * sizeof(QbvhNode));
  if (prims_out) std::memcpy(prims_out, q->primitive_indices.data(), q->primitive_indices.size() * 4);
}
// Visit leaves with a closest-box callback (qbvh.rs tests' `qbvh_closest`):
// returns the box index with the smallest slab entry t, or -1.
int64_t orc_qbvh_closest_box(void* h, const float* bounds6, const float* ray6, float* t_out) {
  Qbvh* q = (Qbvh*)h;
  Ray r;
  r.origin = Vec3(ray6[0], ray6[1], ray6[2]);
  r.direction = Vec3(ray6[3], ray6[4], ray6[5]);
  Vec3 inv(safe_inv(r.direction.x), safe_inv(r.direction.y), safe_inv(r.direction.z));
  int64_t best = -1;
  float bt = kInf;
  traverse_qbvh(
      *q, r, kInf,
      [&](uint32_t off, uint32_t cnt, float tm) -> float {
        float nt = tm;
        for (uint32_t k = off; k < off + cnt; ++k) {
          uint32_t idx = q->primitive_indices[k];
          const float* b = bounds6 + 6 * idx;
          Vec3 t1 = (Vec3(b[0], b[1], b[2]) - r.origin) * inv;
          Vec3 t2 = (Vec3(b[3], b[4], b[5]) - r.origin) * inv;
          Vec3 tmn = vmin(t1, t2), tmx = vmax(t1, t2);
          float tmin = fmax_num(fmax_num(fmax_num(tmn.x, tmn.y), tmn.z), 0.0f);
          float tmax = fmin_num(fmin_num(fmin_num(tmx.x, tmx.y), tmx.z), nt);
          if (tmin <= tmax && (best < 0 || tmin < bt)) { best = idx; bt = tmin; nt = tmin; }
        }
        return nt;
      },
      nullptr, nullptr);
  if (t_out) *t_out = bt;
  return best;
}

// ---- two-level geometry --------------------------------------------------
void* orc_geometry_create() { return new Geometry(); }
void orc_geometry_free(void* g) { delete (Geometry*)g; }

// positions: n_vert*3; normals/uvs optional (may be null); indices: n_idx.
int64_t orc_geometry_add_mesh(void* gh, const float* pos, uint64_t n_vert, const float* nrm, const float* uv,
                              const uint32_t* idx, uint64_t n_idx) {
  Geometry* g = (Geometry*)gh;
  Mesh m;
  m.positions.resize(n_vert);
  m.normals.resize(n_vert);
  m.uvs.resize(n_vert);
  for (uint64_t i = 0; i < n_vert; ++i) {
    m.positions[i] = Vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    m.normals[i] = nrm ? Vec3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]) : Vec3(0, 0, 0);
    m.uvs[i] = uv ? Vec2(uv[2 * i], uv[2 * i + 1]) : Vec2(0, 0);
  }
  m.indices.assign(idx, idx + n_idx);
  // mesh.rs:59-69 + compute_bounds: union of vertex positions
  Bounds b;
  for (auto& p : m.positions) { Bounds pb; pb.min = p; pb.max = p; b = b.unite(pb); }
  m.bounds = b;
  g->meshes.push_back(std::move(m));
  return (int64_t)g->meshes.size() - 1;
}

// Matrices are column-major 4x4 (glam layout); normal_to_world is 3x3 column-major.
int64_t orc_geometry_add_instance(void* gh, uint32_t mesh, uint32_t material, const float* l2w, const float* w2l,
                                  const float* n2w) {
  Geometry* g = (Geometry*)gh;
  Instance in;
  in.mesh_index = mesh;
  in.material_index = material;
  std::memcpy(in.local_to_world.c, l2w, 64);
  std::memcpy(in.world_to_local.c, w2l, 64);
  std::memcpy(in.normal_to_world.c, n2w, 36);
  in.world_bounds = transform_bounds(g->meshes[mesh].bounds, in.local_to_world);
  g->instances.push_back(in);
  return (int64_t)g->instances.size() - 1;
}

// scene/mod.rs:305-317 and mesh.rs:114-119
void orc_geometry_build(void* gh) {
  Geometry* g = (Geometry*)gh;
  for (auto& m : g->meshes) {
    std::vector<Bounds> tb(m.triangle_count());
    for (size_t t = 0; t < tb.size(); ++t) {
      Vec3 v[3];
      m.triangle_positions(t, v);
      tb[t].min = vmin(vmin(v[0], v[1]), v[2]);
      tb[t].max = vmax(vmax(v[0], v[1]), v[2]);
    }
    build_qbvh(tb, &m.qbvh);
  }
  std::vector<Bounds> ib(g->instances.size());
  for (size_t i = 0; i < ib.size(); ++i) ib[i] = g->instances[i].world_bounds;
  build_qbvh(ib, &g->tlas);
}

uint64_t orc_geometry_mesh_qbvh_nodes(void* gh, uint32_t mesh) { return ((Geometry*)gh)->meshes[mesh].qbvh.nodes.size(); }
void orc_geometry_mesh_qbvh_copy(void* gh, uint32_t mesh, void* nodes, uint32_t* prims) {
  const Qbvh& q = ((Geometry*)gh)->meshes[mesh].qbvh;
  if (nodes && !q.nodes.empty()) std::memcpy(nodes, q.nodes.data(), q.nodes.size() * sizeof(QbvhNode));
  if (prims) std::memcpy(prims, q.primitive_indices.data(), q.primitive_indices.size() * 4);
}
uint64_t orc_geometry_tlas_nodes(void* gh) { return ((Geometry*)gh)->tlas.nodes.size(); }
void orc_geometry_tlas_copy(void* gh, void* nodes, uint32_t* prims) {
  const Qbvh& q = ((Geometry*)gh)->tlas;
  if (nodes && !q.nodes.empty()) std::memcpy(nodes, q.nodes.data(), q.nodes.size() * sizeof(QbvhNode));
  if (prims) std::memcpy(prims, q.primitive_indices.data(), q.primitive_indices.size() * 4);
}

// rays: 7 planes of n floats (ox, oy, oz, dx, dy, dz, tmax).  mode 0 = closest hit
// (tmax plane ignored: Scene::closest_hit always starts at +inf), 1 = any hit below tmax.
// Outputs: prim (triangle index, -1 = miss), inst, t, bary (3 planes), stats (2 per ray: nodes, tris).
void orc_geometry_query(void* gh, const float* rays, uint64_t n, int mode, int32_t* prim, int32_t* inst, float* t,
                        float* bary, uint32_t* stats, int nthreads) {
  const Geometry* g = (const Geometry*)gh;
  parallel_for(n, nthreads, [&](uint64_t i) {
    Ray r = ray_from_soa(rays, n, i);
    SceneHit h;
    TraversalStats st;
    bool found = mode == 0 ? g->closest_hit(r, &h, stats ? &st : nullptr)
                           : g->any_hit(r, rays[6 * n + i], &h, stats ? &st : nullptr);
    prim[i] = found ? h.triangle : -1;
    if (inst) inst[i] = found ? h.instance : -1;
    if (t) t[i] = found ? h.t : kInf;
    if (bary) {
      bary[i] = found ? h.bary.x : 0.0f;
      bary[n + i] = found ? h.bary.y : 0.0f;
      bary[2 * n + i] = found ? h.bary.z : 0.0f;
    }
    if (stats) {
      stats[2 * i] = (uint32_t)st.nodes;
      stats[2 * i + 1] = (uint32_t)st.triangles;
    }
  });
}

// ---- sampler ---------------------------------------------------------------
void orc_sampler_vertex_randoms(uint32_t px, uint32_t py, uint32_t sample, uint32_t spp, uint32_t rx, uint32_t ry,
                                uint32_t depth, float* out12, uint32_t* seed_out) {
  PathSampler s(px, py, sample, spp, rx, ry);
  VertexRandoms r = s.path_vertex_randoms(depth);
  float v[12] = {r.light.u_category, r.light.u_tree, r.light.u_light_aux, r.light.u_surface.x, r.light.u_surface.y,
                 r.material.u_lobe, r.material.u_layer, r.material.u_dir.x, r.material.u_dir.y, r.material.u_extra0,
                 r.material.u_extra1, r.u_rr};
  std::memcpy(out12, v, sizeof v);
  *seed_out = r.aux_rng_seed;
}
void orc_sampler_camera(uint32_t px, uint32_t py, uint32_t sample, uint32_t spp, uint32_t rx, uint32_t ry,
                        float* out2, uint32_t* aux_seed) {
  PathSampler s(px, py, sample, spp, rx, ry);
  Vec2 c = s.camera_sample();
  out2[0] = c.x; out2[1] = c.y;
  *aux_seed = s.initial_aux_rng_seed();
}
// Per query (px, py, sample, depth) of a width x height image at spp: the
// camera sample and path_vertex_randoms(depth) (path_sampler.rs:97-118, the 11
// values in dimension order, u_extra2/3 included) as 16 floats, and the
// initial and vertex aux seeds; the layout tpt_sampler_values_device writes.
void orc_sampler_values(uint32_t width, uint32_t height, uint32_t spp, uint64_t n, const uint32_t* q, float* out,
                        uint32_t* seeds, int nthreads) {
  parallel_for(n, nthreads, [&](uint64_t i) {
    const uint32_t* qi = q + 4 * i;
    PathSampler s(qi[0], qi[1], qi[2], spp, width, height);
    const Vec2 c = s.camera_sample();
    const VertexRandoms r = s.path_vertex_randoms(qi[3]);
    const float v[16] = {c.x, c.y, r.light.u_category, r.light.u_tree, r.light.u_light_aux, r.light.u_surface.x,
                         r.light.u_surface.y, r.material.u_lobe, r.material.u_layer, r.material.u_dir.x,
                         r.material.u_dir.y, r.material.u_extra0, r.material.u_extra1, r.material.u_extra2,
                         r.material.u_extra3, r.u_rr};
    std::memcpy(out + 16 * i, v, sizeof v);
    seeds[2 * i] = s.initial_aux_rng_seed();
    seeds[2 * i + 1] = r.aux_rng_seed;
  });
}
uint64_t orc_zsobol_sample_index(uint32_t spp, uint32_t rx, uint32_t ry, uint32_t px, uint32_t py, uint32_t sample,
                                 uint32_t dim) {
  IndexSampler s(spp, rx, ry);
  return s.sample_index(px, py, sample, dim);
}
void orc_shuffled_scrambled_sobol(uint32_t index, uint32_t seed, int depth, uint32_t* out) {
  shuffled_scrambled_sobol(index, seed, depth, out);
}
float orc_uint_to_float(uint32_t v) { return uint_to_float(v); }
uint64_t orc_encode_morton_2(uint32_t x, uint32_t y) { return encode_morton_2(x, y); }
uint32_t orc_laine_karras(uint32_t v, uint32_t seed) { return laine_karras_permutation(v, seed); }
uint32_t orc_reverse_and_shuffle(uint32_t v, uint32_t seed) { return reverse_and_shuffle(v, seed); }
uint32_t orc_pcg_hash(uint32_t v) { return pcg_hash(v); }
uint32_t orc_pcg_state_transition(uint32_t v) { return pcg_state_transition(v); }
uint32_t orc_pcg_output(uint32_t v) { return pcg_output(v); }
uint64_t orc_mix_bits(uint64_t v) { return mix_bits(v); }

// ---- camera ----------------------------------------------------------------
// params: eye(3), look_at(3), up(3), fov_y, exposure.  out: o(3) d(3) rxo(3) ryo(3) rxd(3) ryd(3) width spread.
void orc_camera_ray(const float* params, uint32_t rx, uint32_t ry, uint32_t px, uint32_t py, float ux, float uy,
                    uint32_t spp, float* out20) {
  Camera c = Camera::make(Vec3(params[0], params[1], params[2]), Vec3(params[3], params[4], params[5]),
                          Vec3(params[6], params[7], params[8]), params[9], params[10]);
  Ray r = c.generate_ray_differential(rx, ry, px, py, Vec2(ux, uy), spp);
  float v[20] = {r.origin.x, r.origin.y, r.origin.z, r.direction.x, r.direction.y, r.direction.z,
                 r.diff.rx_origin.x, r.diff.rx_origin.y, r.diff.rx_origin.z, r.diff.ry_origin.x, r.diff.ry_origin.y,
                 r.diff.ry_origin.z, r.diff.rx_direction.x, r.diff.rx_direction.y, r.diff.rx_direction.z,
                 r.diff.ry_direction.x, r.diff.ry_direction.y, r.diff.ry_direction.z, r.cone_width, r.cone_spread};
  std::memcpy(out20, v, sizeof v);
}

}  // extern "C"

extern "C" {
// Step sequence of each closest-hit query in visit order: 'N' per 4-wide node
// test, 'L' per BLAS leaf (one byte per step, zero-terminated, max_len bytes per
// ray).  Used to model SIMT schedules of the device traversal on the CPU.
void orc_geometry_step_sequence(void* gh, const float* rays, uint64_t n, char* out, uint32_t max_len, int nthreads) {
  const Geometry* g = (const Geometry*)gh;
  parallel_for(n, nthreads, [&](uint64_t i) {
    Ray r = ray_from_soa(rays, n, i);
    char* o = out + i * max_len;
    uint32_t k = 0;
    // replay Geometry::closest_hit with a recording leaf callback
    if (g->instances.empty()) { o[0] = 0; return; }
    float best_t = kInf;
    traverse_qbvh(
        g->tlas, r, kInf,
        [&](uint32_t offset, uint32_t count, float cur) -> float {
          float t_max = cur;
          for (uint32_t oi = offset; oi < offset + count; ++oi) {
            const Instance& inst = g->instances[g->tlas.primitive_indices[oi]];
            Ray lr;
            lr.origin = inst.world_to_local.transform_point3(r.origin);
            lr.direction = inst.world_to_local.transform_vector3(r.direction);
            const Mesh& mesh = g->meshes[inst.mesh_index];
            TraversalStats st;
            uint64_t last_nodes = 0;
            traverse_qbvh(
                mesh.qbvh, lr, t_max,
                [&](uint32_t off2, uint32_t cnt2, float cur2) -> float {
                  // node tests since the previous callback happened before this leaf
                  for (; last_nodes < st.nodes && k + 1 < max_len; ++last_nodes) o[k++] = 'N';
                  if (k + 1 < max_len) o[k++] = 'L';
                  float tm = cur2;
                  for (uint32_t q = off2; q < off2 + cnt2; ++q) {
                    Vec3 v[3];
                    mesh.triangle_positions(mesh.qbvh.primitive_indices[q], v);
                    TriHit h;
                    if (intersect_triangle(lr, tm, v[0], v[1], v[2], &h)) { tm = h.t; best_t = h.t; }
                  }
                  return tm;
                },
                nullptr, &st);
            for (; last_nodes < st.nodes && k + 1 < max_len; ++last_nodes) o[k++] = 'N';
            if (best_t < t_max) t_max = best_t;
          }
          return t_max;
        },
        nullptr, nullptr);
    o[k] = 0;
  });
}
}
