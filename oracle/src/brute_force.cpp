// Test infrastructure: an FP64 brute-force ray/triangle oracle, independent of
// the QBVH (no acceleration structure: every ray against every triangle) and of
// the f32 watertight test of math/ray.rs:107-209 (Moller-Trumbore solved in
// double precision, no epsilon).  It checks which triangle is nearest along a
// ray, which is what `Scene::closest_hit` (scene/mod.rs:340-395) returns, as
// the reference's own brute-force comparison does
// (qbvh.rs:902-969, traverse_closest_matches_brute_force_on_grid).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

namespace {

// Rays in chunks of 16 handed out to nthreads threads.
template <class F>
void rays_in_parallel(uint64_t n, int nthreads, F&& f) {
  std::atomic<uint64_t> next{0};
  auto run = [&]() {
    for (;;) {
      const uint64_t s = next.fetch_add(16);
      if (s >= n) break;
      for (uint64_t i = s; i < std::min(n, s + 16); ++i) f(i);
    }
  };
  std::vector<std::thread> ts;
  for (int t = 1; t < nthreads; ++t) ts.emplace_back(run);
  run();
  for (auto& t : ts) t.join();
}

struct D3 {
  double x, y, z;
};
inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Moller-Trumbore in double: t > 0 and barycentrics (u, v, 1-u-v) all >= 0.
// Returns t (infinity on a miss) and the smallest barycentric (negative when
// the ray passes outside the triangle, by how much).
inline double mt_f64(D3 o, D3 d, D3 v0, D3 v1, D3 v2, double* min_bary) {
  const D3 e1 = sub(v1, v0), e2 = sub(v2, v0);
  const D3 p = cross(d, e2);
  const double det = dot(e1, p);
  *min_bary = -1.0;
  if (det == 0.0) return INFINITY;
  const double inv = 1.0 / det;
  const D3 s = sub(o, v0);
  const double u = dot(s, p) * inv;
  const D3 q = cross(s, e1);
  const double v = dot(d, q) * inv;
  const double w = 1.0 - u - v;
  *min_bary = std::fmin(std::fmin(u, v), w);
  const double t = dot(e2, q) * inv;
  if (u < 0.0 || v < 0.0 || w < 0.0 || !(t > 0.0)) return INFINITY;
  return t;
}

inline D3 vtx(const float* pos, uint32_t i) { return {(double)pos[3 * i], (double)pos[3 * i + 1], (double)pos[3 * i + 2]}; }

}  // namespace

extern "C" {

// For each ray (7 planes of n floats: o, d, tmax; tmax not read, as
// closest_hit starts at +inf): the nearest triangle over all ntri triangles
// (prim, -1 on a miss), its FP64 t, and the FP64 t of the nearest *other*
// triangle (+inf if none) so that near-ties can be recognised.
void orc_brute_force_f64(const float* pos, const uint32_t* idx, uint64_t ntri, const float* rays, uint64_t n,
                         int32_t* prim, double* t_best, double* t_second, int nthreads) {
  rays_in_parallel(n, nthreads, [&](uint64_t r) {
    const D3 o{rays[r], rays[n + r], rays[2 * n + r]};
    const D3 d{rays[3 * n + r], rays[4 * n + r], rays[5 * n + r]};
    double b1 = INFINITY, b2 = INFINITY;
    int32_t best = -1;
    for (uint64_t k = 0; k < ntri; ++k) {
      double mb;
      const double t = mt_f64(o, d, vtx(pos, idx[3 * k]), vtx(pos, idx[3 * k + 1]), vtx(pos, idx[3 * k + 2]), &mb);
      if (t < b1) {
        b2 = b1;
        b1 = t;
        best = (int32_t)k;
      } else if (t < b2) {
        b2 = t;
      }
    }
    prim[r] = best;
    t_best[r] = b1;
    t_second[r] = b2;
  });
}

// The FP64 t (+inf on a miss) and smallest barycentric of triangle tri[r] for
// ray r (tri[r] < 0: t = +inf, min_bary = -1).
void orc_triangle_f64(const float* pos, const uint32_t* idx, const int32_t* tri, const float* rays, uint64_t n,
                      double* t_out, double* min_bary, int nthreads) {
  rays_in_parallel(n, nthreads, [&](uint64_t r) {
    if (tri[r] < 0) {
      t_out[r] = INFINITY;
      min_bary[r] = -1.0;
      return;
    }
    const D3 o{rays[r], rays[n + r], rays[2 * n + r]};
    const D3 d{rays[3 * n + r], rays[4 * n + r], rays[5 * n + r]};
    const uint64_t k = (uint64_t)tri[r];
    t_out[r] = mt_f64(o, d, vtx(pos, idx[3 * k]), vtx(pos, idx[3 * k + 1]), vtx(pos, idx[3 * k + 2]), &min_bary[r]);
  });
}

}  // extern "C"
