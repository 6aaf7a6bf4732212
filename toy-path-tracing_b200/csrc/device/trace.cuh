// Two-level 4-wide BVH traversal on the device, one ray per thread.
//
// Semantics follow the reference exactly (bit-for-bit on the same tree):
//  - slab test of qbvh.rs:578-607 with SSE minps/maxps NaN rules; rays whose
//    reciprocal direction has an infinite lane take the exact select path,
//    all others the cheaper fminf/fmaxf path (identical when no NaN can arise);
//  - per node, hit lanes are ordered by entry distance (stable), leaves are
//    visited far-to-near and interior nodes pushed so the nearest pops first
//    (qbvh.rs:640-671).  Leaves are pushed onto the stack above the interior
//    children, which gives the same leaf order and the same t_max for every
//    later box test as calling them in place;
//  - TLAS leaves expand to instance markers; an instance marker transforms the
//    ray (glam Mat4::transform_point3/_vector3 order) and traverses its BLAS
//    with the shared running t_max (scene/mod.rs:340-395, 686-723);
//  - pbrt-v4 watertight triangle test with the f64 fallback (math/ray.rs:107-209);
//    ties on t keep the later-tested triangle.
// The library is compiled with -fmad=false so that no multiply-add is fused
// unless written as fmaf (the reference's `mul_add`).
#pragma once
#include "dev_types.cuh"

namespace tpt {

__device__ __forceinline__ float safe_inv(float d) { return d == 0.0f ? __int_as_float(0x7f800000) : 1.0f / d; }

// Per-(local-)ray data reused by every box and triangle test.
struct RayPre {
  float ox, oy, oz;     // origin
  float ix, iy, iz;     // safe reciprocal direction
  float dx, dy, dz;     // direction
  float sx, sy, sz;     // shear constants of the watertight test
  int kx, ky, kz;       // axis permutation (kz = largest |d| component)
  bool exact;           // an infinite reciprocal lane: use select min/max
  bool no_tri;          // permuted d.z == 0: no triangle can be hit
};

__device__ __forceinline__ float pick3(float a, float b, float c, int k) { return k == 0 ? a : (k == 1 ? b : c); }

__device__ __forceinline__ void ray_setup(RayPre& r, float ox, float oy, float oz, float dx, float dy, float dz) {
  r.ox = ox; r.oy = oy; r.oz = oz;
  r.dx = dx; r.dy = dy; r.dz = dz;
  r.ix = safe_inv(dx); r.iy = safe_inv(dy); r.iz = safe_inv(dz);
  // NaN can only come from 0 * inf in (b - o) * inv, i.e. from a reciprocal
  // lane that is infinite (or zero, for an infinite direction component).
  r.exact = !(isfinite(r.ix) && isfinite(r.iy) && isfinite(r.iz) && r.ix != 0.0f && r.iy != 0.0f && r.iz != 0.0f);
  float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
  int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);  // math/mod.rs:148-156
  int kx = kz + 1; if (kx == 3) kx = 0;
  int ky = kx + 1; if (ky == 3) ky = 0;
  r.kx = kx; r.ky = ky; r.kz = kz;
  float pdx = pick3(dx, dy, dz, kx), pdy = pick3(dx, dy, dz, ky), pdz = pick3(dx, dy, dz, kz);
  r.no_tri = (pdz == 0.0f);
  r.sx = -pdx / pdz;
  r.sy = -pdy / pdz;
  r.sz = 1.0f / pdz;
}

__device__ __forceinline__ float dop(float a, float b, float c, float d) {
  float cd = c * d;
  float e = fmaf(a, b, -cd);
  float err = fmaf(-c, d, cd);
  return e + err;
}

// math/ray.rs:107-209 with the ray-only work hoisted into RayPre.
__device__ __forceinline__ bool tri_test(const RayPre& r, float t_max, const DevTri& tri, float& t_out, float& b0,
                                         float& b1, float& b2) {
  // degenerate flag precomputed on the host with the reference's formula
  if (tri.v1.w != 0.0f || r.no_tri) return false;
  float p0x = pick3(tri.v0.x, tri.v0.y, tri.v0.z, r.kx) - pick3(r.ox, r.oy, r.oz, r.kx);
  float p0y = pick3(tri.v0.x, tri.v0.y, tri.v0.z, r.ky) - pick3(r.ox, r.oy, r.oz, r.ky);
  float p0z = pick3(tri.v0.x, tri.v0.y, tri.v0.z, r.kz) - pick3(r.ox, r.oy, r.oz, r.kz);
  float p1x = pick3(tri.v1.x, tri.v1.y, tri.v1.z, r.kx) - pick3(r.ox, r.oy, r.oz, r.kx);
  float p1y = pick3(tri.v1.x, tri.v1.y, tri.v1.z, r.ky) - pick3(r.ox, r.oy, r.oz, r.ky);
  float p1z = pick3(tri.v1.x, tri.v1.y, tri.v1.z, r.kz) - pick3(r.ox, r.oy, r.oz, r.kz);
  float p2x = pick3(tri.v2.x, tri.v2.y, tri.v2.z, r.kx) - pick3(r.ox, r.oy, r.oz, r.kx);
  float p2y = pick3(tri.v2.x, tri.v2.y, tri.v2.z, r.ky) - pick3(r.ox, r.oy, r.oz, r.ky);
  float p2z = pick3(tri.v2.x, tri.v2.y, tri.v2.z, r.kz) - pick3(r.ox, r.oy, r.oz, r.kz);
  p0x = p0x + r.sx * p0z; p0y = p0y + r.sy * p0z;
  p1x = p1x + r.sx * p1z; p1y = p1y + r.sy * p1z;
  p2x = p2x + r.sx * p2z; p2y = p2y + r.sy * p2z;
  float e0 = dop(p1x, p2y, p1y, p2x);
  float e1 = dop(p2x, p0y, p2y, p0x);
  float e2 = dop(p0x, p1y, p0y, p1x);
  if (e0 == 0.0f || e1 == 0.0f || e2 == 0.0f) {
    e0 = (float)((double)p2y * (double)p1x - (double)p2x * (double)p1y);
    e1 = (float)((double)p0y * (double)p2x - (double)p0x * (double)p2y);
    e2 = (float)((double)p1y * (double)p0x - (double)p1x * (double)p0y);
  }
  if ((e0 < 0.0f || e1 < 0.0f || e2 < 0.0f) && (e0 > 0.0f || e1 > 0.0f || e2 > 0.0f)) return false;
  float det = e0 + e1 + e2;
  if (det == 0.0f) return false;
  p0z = p0z * r.sz; p1z = p1z * r.sz; p2z = p2z * r.sz;
  float ts = e0 * p0z + e1 * p1z + e2 * p2z;
  if ((det < 0.0f && (ts >= 0.0f || ts < t_max * det)) || (det > 0.0f && (ts <= 0.0f || ts > t_max * det)))
    return false;
  float inv_det = 1.0f / det;
  float t = ts * inv_det;
  const float eps = 5.9604644775390625e-08f;  // f32::EPSILON / 2
  const float g2 = (2.0f * eps) / (1.0f - 2.0f * eps);
  const float g3 = (3.0f * eps) / (1.0f - 3.0f * eps);
  const float g5 = (5.0f * eps) / (1.0f - 5.0f * eps);
  float max_zt = fmaxf(fmaxf(fabsf(p0z), fabsf(p1z)), fabsf(p2z));
  float delta_z = g3 * max_zt;
  float max_xt = fmaxf(fmaxf(fabsf(p0x), fabsf(p1x)), fabsf(p2x));
  float max_yt = fmaxf(fmaxf(fabsf(p0y), fabsf(p1y)), fabsf(p2y));
  float delta_x = g5 * (max_xt + max_zt);
  float delta_y = g5 * (max_yt + max_zt);
  float delta_e = 2.0f * (g2 * max_xt * max_yt + delta_y * max_xt + delta_x * max_yt);
  float max_e = fmaxf(fmaxf(fabsf(e0), fabsf(e1)), fabsf(e2));
  float delta_t = 3.0f * (g3 * max_e * max_zt + delta_e * max_zt + delta_z * max_e) * fabsf(inv_det);
  if (t <= delta_t) return false;
  t_out = t;
  b0 = e0 * inv_det; b1 = e1 * inv_det; b2 = e2 * inv_det;
  return true;
}

// Slab test of one 4-wide node: returns the lane hit mask, lane entry
// distances in tmin[], child words in ch[].
__device__ __forceinline__ uint32_t box4(const DevNode* __restrict__ n, const RayPre& r, float t_max, float tmin[4],
                                         uint32_t ch[4]) {
  const float4 lx = __ldg(&n->lo_x), ly = __ldg(&n->lo_y), lz = __ldg(&n->lo_z);
  const float4 hx = __ldg(&n->hi_x), hy = __ldg(&n->hi_y), hz = __ldg(&n->hi_z);
  const uint4 c = __ldg(&n->child);
  const float lox[4] = {lx.x, lx.y, lx.z, lx.w}, loy[4] = {ly.x, ly.y, ly.z, ly.w}, loz[4] = {lz.x, lz.y, lz.z, lz.w};
  const float hix[4] = {hx.x, hx.y, hx.z, hx.w}, hiy[4] = {hy.x, hy.y, hy.z, hy.w}, hiz[4] = {hz.x, hz.y, hz.z, hz.w};
  ch[0] = c.x; ch[1] = c.y; ch[2] = c.z; ch[3] = c.w;
  uint32_t mask = 0;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    float t1x = (lox[s] - r.ox) * r.ix, t2x = (hix[s] - r.ox) * r.ix;
    float t1y = (loy[s] - r.oy) * r.iy, t2y = (hiy[s] - r.oy) * r.iy;
    float t1z = (loz[s] - r.oz) * r.iz, t2z = (hiz[s] - r.oz) * r.iz;
    float a, b;
    if (r.exact) {
      float mnx = t1x < t2x ? t1x : t2x, mxx = t1x > t2x ? t1x : t2x;
      float mny = t1y < t2y ? t1y : t2y, mxy = t1y > t2y ? t1y : t2y;
      float mnz = t1z < t2z ? t1z : t2z, mxz = t1z > t2z ? t1z : t2z;
      a = mnx > mny ? mnx : mny; a = a > mnz ? a : mnz; a = a > 0.0f ? a : 0.0f;
      b = mxx < mxy ? mxx : mxy; b = b < mxz ? b : mxz; b = b < t_max ? b : t_max;
    } else {
      a = fmaxf(fmaxf(fmaxf(fminf(t1x, t2x), fminf(t1y, t2y)), fminf(t1z, t2z)), 0.0f);
      b = fminf(fminf(fminf(fmaxf(t1x, t2x), fmaxf(t1y, t2y)), fmaxf(t1z, t2z)), t_max);
    }
    tmin[s] = a;
    // lanes whose child word decodes to Empty (leaf bit, zero count) never count
    if (a <= b && (ch[s] >> 24) != 0x80u) mask |= 1u << s;
  }
  return mask;
}

// Stable ascending order of the hit lanes by entry distance; returns the
// child words sorted far-to-near in w[0..n).  Missing lanes sort last.
__device__ __forceinline__ int order_far_to_near(uint32_t mask, const float tmin[4], const uint32_t ch[4],
                                                 uint32_t w[4]) {
  float k[4];
  int s[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    bool v = (mask >> i) & 1u;
    k[i] = v ? tmin[i] : __int_as_float(0x7f800000);
    s[i] = v ? i : 4 + i;
    w[i] = ch[i];
  }
  // 5-comparator network on (key, lane) pairs: a total order, so any correct
  // network reproduces the reference's stable insertion sort.
#define TPT_CS(a, b)                                                           \
  {                                                                            \
    bool sw = (k[a] > k[b]) || (k[a] == k[b] && s[a] > s[b]);                  \
    float tk = sw ? k[b] : k[a]; k[b] = sw ? k[a] : k[b]; k[a] = tk;           \
    int ts = sw ? s[b] : s[a]; s[b] = sw ? s[a] : s[b]; s[a] = ts;             \
    uint32_t tw = sw ? w[b] : w[a]; w[b] = sw ? w[a] : w[b]; w[a] = tw;        \
  }
  TPT_CS(0, 1) TPT_CS(2, 3) TPT_CS(0, 2) TPT_CS(1, 3) TPT_CS(1, 2)
#undef TPT_CS
  return __popc(mask);
}

struct TraceResult {
  float t;
  int32_t tri;
  int32_t inst;
  float b0, b1, b2;
};

struct TraceCounters {
  uint32_t nodes;
  uint32_t tris;
};

// MODE 0: closest hit.  MODE 1: stop at the first accepted triangle.
// Returns false only on a device check failure (stack overflow), in which case
// *err receives the flag.
template <int MODE, bool STATS>
__device__ __forceinline__ bool trace_ray(const DevGeometry& G, float ox, float oy, float oz, float dx, float dy,
                                          float dz, float t_max, TraceResult& res, TraceCounters& cnt,
                                          uint32_t* err) {
  uint32_t stack[kStackDepth];
  int sp = 0;
  float closest = t_max;
  res.t = __int_as_float(0x7f800000);
  res.tri = -1;
  res.inst = -1;
  res.b0 = res.b1 = res.b2 = 0.0f;
  if (STATS) { cnt.nodes = 0; cnt.tris = 0; }
  if (G.num_instances == 0) return true;

  RayPre world, local;
  ray_setup(world, ox, oy, oz, dx, dy, dz);
  bool in_blas = false;
  int floor_sp = 0;
  uint32_t node_base = 0, tri_base = 0, inst_id = 0;

  stack[sp++] = G.tlas_root_word;
  while (sp > 0) {
    if (in_blas && sp == floor_sp) in_blas = false;
    const uint32_t w = stack[--sp];
    if (w & kLeafBit) {
      const uint32_t count = (w >> 24) & 0x7Fu, off = w & 0xFFFFFFu;
      if (!in_blas) {
        if (count == 0) {
          // instance marker: enter its BLAS with the ray in instance space
          inst_id = off;
          const DevInstance* I = G.instances + inst_id;
          const float4 m0 = __ldg(&I->m0), m1 = __ldg(&I->m1), m2 = __ldg(&I->m2);
          const uint4 meta = __ldg(reinterpret_cast<const uint4*>(&I->node_base));
          // res = c0*x; res = c1*y + res; res = c2*z + res; (+ c3 for points)
          float lox = m0.x * ox, loy = m0.y * ox, loz = m0.z * ox;
          lox = m0.w * oy + lox; loy = m1.x * oy + loy; loz = m1.y * oy + loz;
          lox = m1.z * oz + lox; loy = m1.w * oz + loy; loz = m2.x * oz + loz;
          lox = m2.y + lox; loy = m2.z + loy; loz = m2.w + loz;
          float ldx = m0.x * dx, ldy = m0.y * dx, ldz = m0.z * dx;
          ldx = m0.w * dy + ldx; ldy = m1.x * dy + ldy; ldz = m1.y * dy + ldz;
          ldx = m1.z * dz + ldx; ldy = m1.w * dz + ldy; ldz = m2.x * dz + ldz;
          ray_setup(local, lox, loy, loz, ldx, ldy, ldz);
          node_base = meta.x;
          tri_base = meta.y;
          in_blas = true;
          floor_sp = sp;
          stack[sp++] = meta.z;
        } else {
          // TLAS leaf: its instances in order
          if (sp + (int)count > kStackDepth) { atomicOr(err, kDevErrStackOverflow); return false; }
          for (int j = (int)count - 1; j >= 0; --j) stack[sp++] = kLeafBit | __ldg(G.tlas_prims + off + j);
        }
      } else {
        // BLAS leaf: triangles in leaf order, t_max shrinking on each hit
        for (uint32_t j = 0; j < count; ++j) {
          const DevTri* T = G.tris + tri_base + off + j;
          DevTri tri;
          tri.v0 = __ldg(&T->v0); tri.v1 = __ldg(&T->v1); tri.v2 = __ldg(&T->v2);
          if (STATS) cnt.tris++;
          float t, b0, b1, b2;
          if (tri_test(local, closest, tri, t, b0, b1, b2)) {
            closest = t;
            res.t = t; res.tri = __float_as_int(tri.v0.w); res.inst = (int32_t)inst_id;
            res.b0 = b0; res.b1 = b1; res.b2 = b2;
            if (MODE == 1) return true;
          }
        }
      }
    } else {
      const RayPre& r = in_blas ? local : world;
      const DevNode* n = G.nodes + (in_blas ? node_base : G.tlas_node_base) + w;
      if (STATS) cnt.nodes++;
      float tmin[4];
      uint32_t ch[4];
      uint32_t mask = box4(n, r, closest, tmin, ch);
      if (mask == 0) continue;
      uint32_t sorted[4];
      int nh = order_far_to_near(mask, tmin, ch, sorted);
      if (sp + nh > kStackDepth) { atomicOr(err, kDevErrStackOverflow); return false; }
      // interior children far-to-near (nearest on top), then leaves near-to-far
      // (farthest on top): pops give leaves far-to-near, then nearest interior.
      for (int k = nh - 1; k >= 0; --k)
        if (!(sorted[k] & kLeafBit)) stack[sp++] = sorted[k];
      for (int k = 0; k < nh; ++k)
        if (sorted[k] & kLeafBit) stack[sp++] = sorted[k];
    }
  }
  return true;
}

}  // namespace tpt
