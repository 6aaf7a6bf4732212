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
//    ties on t keep the later-tested triangle;
//  - closest_mesh_hit_with_filter's alpha test (scene/mod.rs:360-377, 686-723):
//    when the caller passes an AuxRng state, a candidate hit on an instance
//    whose material has an alpha test draws u from it (aux_rng.rs:21-28) and
//    is kept iff u < the material's opacity, in the candidates' test order.
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

// Per-thread traversal stack: the first SH entries live in shared memory
// (entry k of thread i at base[k * blockDim.x], bank-conflict free), deeper
// entries in a local-memory spill area.  Total depth kStackDepth (qbvh.rs:609).
template <int SH>
struct SplitStack {
  uint32_t* sh;
  uint32_t spill[kStackDepth - SH];
  __device__ __forceinline__ void set(int k, uint32_t v) {
    if (k < SH) sh[k * blockDim.x] = v;
    else spill[k - SH] = v;
  }
  __device__ __forceinline__ uint32_t get(int k) const { return k < SH ? sh[k * blockDim.x] : spill[k - SH]; }
};

// Stack entries: interior node (bit 31 clear), BLAS/TLAS leaf (bit 31, count
// >= 1), instance marker (bit 31, count 0, instance id), or kNone.  kNone can
// never be a real leaf word: the upload rejects leaf ranges past 2^24.
constexpr uint32_t kNone = 0xFFFFFFFFu;

// Traversal of one ray, advanced one entry at a time.  `next` holds the entry
// to process next (the would-be top of the stack kept in a register).
struct TravState {
  float wox, woy, woz, wdx, wdy, wdz;  // world-space ray
  RayPre r;                            // ray of the current level (world at the TLAS, instance space in a BLAS)
  float closest;                       // running t_max
  TraceResult res;
  uint32_t next;
  int sp, floor_sp;
  bool in_blas;
  bool alpha_on;                       // an AuxRng state was given and the scene has alpha tests
  uint32_t node_base, tri_base, inst_id;
  float alpha;                         // the current instance's opacity (1: no test)
  uint32_t aux;                        // AuxRng state
};

// AuxRng::next_f32 (aux_rng.rs:21-28)
__device__ __forceinline__ float aux_next_f32(uint32_t& state) {
  state = state * 747796405u + 2891336453u;
  uint32_t s = state;
  s ^= s >> (4u + (s >> 28));
  s *= 277803737u;
  s ^= s >> 22;
  return (float)(s >> 8) * (1.0f / 16777216.0f);
}

// Enter instance `id`'s BLAS with the ray transformed by world_to_local
// (glam Mat4::transform_point3 / transform_vector3 order), scene/mod.rs:357.
__device__ __forceinline__ void enter_instance(const DevGeometry& G, TravState& s, uint32_t id) {
  s.inst_id = id;
  s.alpha = s.alpha_on ? __ldg(G.inst_alpha + id) : 1.0f;
  const DevInstance* I = G.instances + id;
  const float4 m0 = __ldg(&I->m0), m1 = __ldg(&I->m1), m2 = __ldg(&I->m2);
  const uint4 meta = __ldg(reinterpret_cast<const uint4*>(&I->node_base));
  const float ox = s.wox, oy = s.woy, oz = s.woz, dx = s.wdx, dy = s.wdy, dz = s.wdz;
  float lox = m0.x * ox, loy = m0.y * ox, loz = m0.z * ox;
  lox = m0.w * oy + lox; loy = m1.x * oy + loy; loz = m1.y * oy + loz;
  lox = m1.z * oz + lox; loy = m1.w * oz + loy; loz = m2.x * oz + loz;
  lox = m2.y + lox; loy = m2.z + loy; loz = m2.w + loz;
  float ldx = m0.x * dx, ldy = m0.y * dx, ldz = m0.z * dx;
  ldx = m0.w * dy + ldx; ldy = m1.x * dy + ldy; ldz = m1.y * dy + ldz;
  ldx = m1.z * dz + ldx; ldy = m1.w * dz + ldy; ldz = m2.x * dz + ldz;
  ray_setup(s.r, lox, loy, loz, ldx, ldy, ldz);
  s.node_base = meta.x;
  s.tri_base = meta.y;
  s.in_blas = true;
  s.floor_sp = s.sp;
  s.next = meta.z;
}

template <class Stack>
__device__ __forceinline__ void trav_pop(TravState& s, Stack& st) {
  if (s.sp == 0) {
    s.next = kNone;
    return;
  }
  if (s.in_blas && s.sp == s.floor_sp) {
    // the instance's BLAS is done: back to the TLAS with the world ray
    s.in_blas = false;
    ray_setup(s.r, s.wox, s.woy, s.woz, s.wdx, s.wdy, s.wdz);
  }
  s.next = st.get(--s.sp);
}

// aux: the ray's AuxRng state (NULL: no alpha tests), advanced by the draws
__device__ __forceinline__ void trav_init(const DevGeometry& G, TravState& s, float ox, float oy, float oz, float dx,
                                          float dy, float dz, float t_max, const uint32_t* aux = nullptr) {
  s.alpha_on = aux != nullptr && G.inst_alpha != nullptr;
  s.aux = aux ? *aux : 0u;
  s.alpha = 1.0f;
  s.wox = ox; s.woy = oy; s.woz = oz; s.wdx = dx; s.wdy = dy; s.wdz = dz;
  s.closest = t_max;
  s.res.t = __int_as_float(0x7f800000);
  s.res.tri = -1;
  s.res.inst = -1;
  s.res.b0 = s.res.b1 = s.res.b2 = 0.0f;
  s.in_blas = false;
  s.floor_sp = 0;
  s.sp = 0;
  s.node_base = s.tri_base = s.inst_id = 0;
  s.next = kNone;
  if (G.num_instances == 0) return;
  const uint32_t root = G.tlas_root_word;
  if ((root & kLeafBit) && ((root >> 24) & 0x7Fu) == 1u) {
    // TLAS is a single-instance root leaf (qbvh.rs:615-620): go straight to it
    enter_instance(G, s, __ldg(G.tlas_prims + (root & 0xFFFFFFu)));
  } else {
    ray_setup(s.r, ox, oy, oz, dx, dy, dz);
    s.next = root;
  }
}

// Processes the interior node in `next`.  The hit children end up, bottom to
// top, as interiors far-to-near then leaves near-to-far (qbvh.rs:640-671: leaves
// are handled far-to-near at once, the nearest interior is popped first); the
// would-be top becomes `next`, the rest go to the stack.
template <bool STATS, class Stack>
__device__ __forceinline__ void node_step(const DevGeometry& G, TravState& s, Stack& st, TraceCounters& cnt,
                                          uint32_t* err) {
  const DevNode* n = G.nodes + (s.in_blas ? s.node_base : G.tlas_node_base) + s.next;
  if (STATS) cnt.nodes++;
  float tmin[4];
  uint32_t ch[4];
  const uint32_t mask = box4(n, s.r, s.closest, tmin, ch);
  const int nh = __popc(mask);
  if (nh == 0) {
    trav_pop(s, st);
    return;
  }
  if (nh == 1) {
    s.next = (mask & 1u) ? ch[0] : (mask & 2u) ? ch[1] : (mask & 4u) ? ch[2] : ch[3];
    return;
  }
  if (s.sp + nh - 1 > kStackDepth) {
    atomicOr(err, kDevErrStackOverflow);
    s.sp = 0;
    s.next = kNone;
    return;
  }
  // before[i][j]: lane i precedes lane j in the stable ascending order by tmin
  bool v[4], leaf[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    v[i] = (mask >> i) & 1u;
    leaf[i] = (ch[i] & kLeafBit) != 0;
  }
  bool pre[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = i + 1; j < 4; ++j) {
      pre[i][j] = tmin[i] <= tmin[j];
      pre[j][i] = !pre[i][j];
    }
  int n_int = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) n_int += (v[i] && !leaf[i]) ? 1 : 0;
  const int top = nh - 1;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (!v[i]) continue;
    int pos = 0;
    if (!leaf[i]) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (j != i && v[j] && !leaf[j] && pre[i][j]) ++pos;  // interiors farther than i
    } else {
      pos = n_int;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (j != i && v[j] && leaf[j] && pre[j][i]) ++pos;  // leaves nearer than i
    }
    if (pos == top) s.next = ch[i];
    else st.set(s.sp + pos, ch[i]);
  }
  s.sp += nh - 1;
}

// Processes the leaf, TLAS leaf or instance marker in `next`.
template <int MODE, bool STATS, class Stack>
__device__ __forceinline__ void leaf_step(const DevGeometry& G, TravState& s, Stack& st, TraceCounters& cnt,
                                          uint32_t* err) {
  const uint32_t w = s.next;
  const uint32_t count = (w >> 24) & 0x7Fu, off = w & 0xFFFFFFu;
  if (s.in_blas) {
    // BLAS leaf: triangles in leaf order, t_max shrinking on each hit
    const DevTri* T = G.tris + s.tri_base + off;
    for (uint32_t j = 0; j < count; ++j) {
      DevTri tri;
      tri.v0 = __ldg(&T[j].v0);
      tri.v1 = __ldg(&T[j].v1);
      tri.v2 = __ldg(&T[j].v2);
      if (STATS) cnt.tris++;
      float t, b0, b1, b2;
      if (tri_test(s.r, s.closest, tri, t, b0, b1, b2)) {
        // any_hit of an alpha-tested material: keep the hit iff u < opacity
        if (s.alpha < 1.0f && !(aux_next_f32(s.aux) < s.alpha)) continue;
        s.closest = t;
        s.res.t = t;
        s.res.tri = __float_as_int(tri.v0.w);
        s.res.inst = (int32_t)s.inst_id;
        s.res.b0 = b0; s.res.b1 = b1; s.res.b2 = b2;
        if (MODE == 1) {
          s.sp = 0;
          s.next = kNone;
          return;
        }
      }
    }
    trav_pop(s, st);
  } else if (count == 0) {
    enter_instance(G, s, off);
  } else {
    // TLAS leaf: its instances in order; the first is entered now
    if (s.sp + (int)count > kStackDepth) {
      atomicOr(err, kDevErrStackOverflow);
      s.sp = 0;
      s.next = kNone;
      return;
    }
    for (int j = (int)count - 1; j >= 1; --j) st.set(s.sp++, kLeafBit | __ldg(G.tlas_prims + off + j));
    enter_instance(G, s, __ldg(G.tlas_prims + off));
  }
}

// One thread traces one ray to the end (used where a thread owns its ray).
template <int MODE, bool STATS, class Stack>
__device__ __forceinline__ void trace_ray(const DevGeometry& G, Stack& st, float ox, float oy, float oz, float dx,
                                          float dy, float dz, float t_max, TraceResult& res, TraceCounters& cnt,
                                          uint32_t* err, uint32_t* aux = nullptr) {
  TravState s;
  trav_init(G, s, ox, oy, oz, dx, dy, dz, t_max, aux);
  if (STATS) { cnt.nodes = 0; cnt.tris = 0; }
  while (s.next != kNone) {
    if (!(s.next & kLeafBit)) node_step<STATS>(G, s, st, cnt, err);
    else leaf_step<MODE, STATS>(G, s, st, cnt, err);
  }
  res = s.res;
  if (aux) *aux = s.aux;
}

// trace_ray for lanes that trace together: the lanes in `act` (all of which
// call this) step through interior nodes together until each faces a leaf,
// then test their leaves together ("while-while"), so the warp runs one code
// path at a time.  Each ray's own visit order is unchanged.
template <int MODE, class Stack>
__device__ __forceinline__ void trace_ray_ww(const DevGeometry& G, Stack& st, unsigned act, float ox, float oy,
                                             float oz, float dx, float dy, float dz, float t_max, TraceResult& res,
                                             uint32_t* err, uint32_t* aux = nullptr) {
  TravState s;
  TraceCounters c;
  trav_init(G, s, ox, oy, oz, dx, dy, dz, t_max, aux);
  for (;;) {
    for (;;) {
      const bool want = !(s.next & kLeafBit);
      if (!__any_sync(act, want)) break;
      if (want) node_step<false>(G, s, st, c, err);
    }
    if (s.next != kNone) leaf_step<MODE, false>(G, s, st, c, err);
    if (!__any_sync(act, s.next != kNone)) break;
  }
  res = s.res;
  if (aux) *aux = s.aux;
}

}  // namespace tpt
