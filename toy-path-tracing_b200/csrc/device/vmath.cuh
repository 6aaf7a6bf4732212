// Device vector math with the reference's evaluation order (glam 0.32 scalar
// Vec3/Mat3/Mat4, crates/renderer/src/math/*).  Compiled with -fmad=false so
// every product and sum rounds separately, as in the Rust code.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tpt {

constexpr float kPiF = 3.14159274101257324f;   // std::f32::consts::PI
constexpr float kTauF = 6.28318548202514648f;  // std::f32::consts::TAU

struct V3 {
  float x, y, z;
};
__host__ __device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__host__ __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__host__ __device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__host__ __device__ __forceinline__ V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
__host__ __device__ __forceinline__ float length_sq(V3 a) { return dot(a, a); }
__device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ V3 normalize(V3 a) { return a * (1.0f / length(a)); }
__device__ __forceinline__ V3 normalize_or_zero(V3 a) {
  const float r = 1.0f / length(a);
  return (isfinite(r) && r > 0.0f) ? a * r : V3{0.0f, 0.0f, 0.0f};
}
__device__ __forceinline__ float max_element(V3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
__device__ __forceinline__ float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
// glam face_forward (math/mod.rs:42-48)
__device__ __forceinline__ V3 face_forward(V3 n, V3 ref) { return dot(n, ref) < 0.0f ? -n : n; }
// math/mod.rs:108-110
__device__ __forceinline__ V3 interp3(V3 b, V3 v0, V3 v1, V3 v2) { return b.x * v0 + b.y * v1 + b.z * v2; }

// Column-major 4x3 affine part of a glam Mat4 (c0, c1, c2, c3 columns).
struct Affine {
  float c[12];
};
__device__ __forceinline__ V3 xform_point(const float* c, V3 p) {
  float x = c[0] * p.x, y = c[1] * p.x, z = c[2] * p.x;
  x = c[3] * p.y + x; y = c[4] * p.y + y; z = c[5] * p.y + z;
  x = c[6] * p.z + x; y = c[7] * p.z + y; z = c[8] * p.z + z;
  x = c[9] + x; y = c[10] + y; z = c[11] + z;
  return {x, y, z};
}
// glam Mat3::mul_vec3 (column-major m[9])
__device__ __forceinline__ V3 mat3_mul(const float* m, V3 v) {
  float x = m[0] * v.x, y = m[1] * v.x, z = m[2] * v.x;
  x = x + m[3] * v.y; y = y + m[4] * v.y; z = z + m[5] * v.y;
  x = x + m[6] * v.z; y = y + m[7] * v.z; z = z + m[8] * v.z;
  return {x, y, z};
}

// OrthonormalBasis (math/orthonormal_basis.rs:11-71)
struct Frame {
  V3 t, b, n;
};
__device__ __forceinline__ Frame frame_from_normal(V3 normal) {
  V3 n = length_sq(normal) > 0.0f ? normalize(normal) : V3{0.0f, 0.0f, 1.0f};
  const float sign = copysignf(1.0f, n.z);
  const float a = -1.0f / (sign + n.z);
  const float b = n.x * n.y * a;
  Frame f;
  f.t = V3{1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x};
  f.b = V3{b, sign + n.y * n.y * a, -n.y};
  f.n = n;
  return f;
}
__device__ __forceinline__ Frame frame_from_normal_tangent(V3 normal, V3 hint) {
  V3 n = length_sq(normal) > 0.0f ? normalize(normal) : V3{0.0f, 0.0f, 1.0f};
  V3 t = normalize_or_zero(hint - dot(hint, n) * n);
  if (length_sq(t) == 0.0f) return frame_from_normal(n);
  Frame f;
  f.b = normalize_or_zero(cross(n, t));
  f.t = normalize_or_zero(cross(f.b, n));
  f.n = n;
  return f;
}
__device__ __forceinline__ V3 to_world(const Frame& f, V3 d) { return normalize(d.x * f.t + d.y * f.b + d.z * f.n); }
__device__ __forceinline__ V3 to_local(const Frame& f, V3 w) { return V3{dot(w, f.t), dot(w, f.b), dot(w, f.n)}; }

// math/mod.rs:163-175
__device__ __forceinline__ float balance_heuristic(float a, float b) {
  const float s = a + b;
  if (a <= 0.0f || s <= 0.0f) return 0.0f;
  return a / s;
}

}  // namespace tpt
