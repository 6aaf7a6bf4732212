// Oracle (test infrastructure only): a CPU restatement of the reference path
// tracer's per-sample hot path, used by tests/, the smoke check and the CPU
// baseline leg of bench.py as the checker.  Nothing in the shipped library
// links or calls this code.
//
// Arithmetic follows the reference crate `crates/renderer` (Rust, glam 0.32
// scalar Vec3, no FMA contraction; `mul_add` is an explicit fused multiply-add).
// Build with -ffp-contract=off and without -ffast-math so that every f32
// operation rounds exactly like the Rust code.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <limits>
#include <algorithm>

namespace orc {

static constexpr float kInf = std::numeric_limits<float>::infinity();

struct Vec2 {
  float x = 0, y = 0;
  Vec2() = default;
  Vec2(float a, float b) : x(a), y(b) {}
};

// glam::Vec3 (scalar build): every method below follows glam's formula so
// that the rounding sequence is the same.
struct Vec3 {
  float x = 0, y = 0, z = 0;
  Vec3() = default;
  Vec3(float a, float b, float c) : x(a), y(b), z(c) {}
  static Vec3 splat(float v) { return Vec3(v, v, v); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  Vec3 operator+(const Vec3& o) const { return Vec3(x + o.x, y + o.y, z + o.z); }
  Vec3 operator-(const Vec3& o) const { return Vec3(x - o.x, y - o.y, z - o.z); }
  Vec3 operator*(const Vec3& o) const { return Vec3(x * o.x, y * o.y, z * o.z); }
  Vec3 operator/(const Vec3& o) const { return Vec3(x / o.x, y / o.y, z / o.z); }
  Vec3 operator*(float s) const { return Vec3(x * s, y * s, z * s); }
  Vec3 operator/(float s) const { return Vec3(x / s, y / s, z / s); }
  Vec3 operator-() const { return Vec3(-x, -y, -z); }
  Vec3& operator+=(const Vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  Vec3& operator*=(const Vec3& o) { x *= o.x; y *= o.y; z *= o.z; return *this; }
  Vec3& operator/=(float s) { x /= s; y /= s; z /= s; return *this; }
  bool operator==(const Vec3& o) const { return x == o.x && y == o.y && z == o.z; }
};
inline Vec3 operator*(float s, const Vec3& v) { return Vec3(s * v.x, s * v.y, s * v.z); }

// Rust f32::min / f32::max (IEEE minNum/maxNum: a NaN operand yields the other).
inline float fmin_num(float a, float b) { return std::fmin(a, b); }
inline float fmax_num(float a, float b) { return std::fmax(a, b); }

inline float dot(const Vec3& a, const Vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec3 cross(const Vec3& a, const Vec3& b) {
  return Vec3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
inline float length_squared(const Vec3& v) { return dot(v, v); }
inline float length(const Vec3& v) { return std::sqrt(dot(v, v)); }
inline Vec3 normalize(const Vec3& v) { return v * (1.0f / length(v)); }
inline Vec3 normalize_or_zero(const Vec3& v) {
  float rcp = 1.0f / length(v);
  if (std::isfinite(rcp) && rcp > 0.0f) return v * rcp;
  return Vec3(0, 0, 0);
}
inline Vec3 vabs(const Vec3& v) { return Vec3(std::fabs(v.x), std::fabs(v.y), std::fabs(v.z)); }
inline Vec3 vmin(const Vec3& a, const Vec3& b) { return Vec3(fmin_num(a.x, b.x), fmin_num(a.y, b.y), fmin_num(a.z, b.z)); }
inline Vec3 vmax(const Vec3& a, const Vec3& b) { return Vec3(fmax_num(a.x, b.x), fmax_num(a.y, b.y), fmax_num(a.z, b.z)); }
inline float max_element(const Vec3& v) { return fmax_num(fmax_num(v.x, v.y), v.z); }
inline bool is_finite(const Vec3& v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }
inline float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

// glam::Mat4, column major: cols[c][r].
struct Mat4 {
  float c[4][4];
  static Mat4 identity() {
    Mat4 m; std::memset(&m, 0, sizeof m);
    for (int i = 0; i < 4; ++i) m.c[i][i] = 1.0f;
    return m;
  }
  // glam Mat4::transform_point3: x_axis*x, then y_axis*y + res, z_axis*z + res, w_axis + res.
  Vec3 transform_point3(const Vec3& p) const {
    float r[3];
    for (int i = 0; i < 3; ++i) r[i] = c[0][i] * p.x;
    for (int i = 0; i < 3; ++i) r[i] = c[1][i] * p.y + r[i];
    for (int i = 0; i < 3; ++i) r[i] = c[2][i] * p.z + r[i];
    for (int i = 0; i < 3; ++i) r[i] = c[3][i] + r[i];
    return Vec3(r[0], r[1], r[2]);
  }
  // glam Mat4::transform_vector3: same without the translation column.
  Vec3 transform_vector3(const Vec3& v) const {
    float r[3];
    for (int i = 0; i < 3; ++i) r[i] = c[0][i] * v.x;
    for (int i = 0; i < 3; ++i) r[i] = c[1][i] * v.y + r[i];
    for (int i = 0; i < 3; ++i) r[i] = c[2][i] * v.z + r[i];
    return Vec3(r[0], r[1], r[2]);
  }
};

// glam::Mat3 (column major) times vector, same accumulation order as above.
struct Mat3 {
  float c[3][3];
  Vec3 mul_vec3(const Vec3& v) const {
    float r[3];
    for (int i = 0; i < 3; ++i) r[i] = c[0][i] * v.x;
    for (int i = 0; i < 3; ++i) r[i] = c[1][i] * v.y + r[i];
    for (int i = 0; i < 3; ++i) r[i] = c[2][i] * v.z + r[i];
    return Vec3(r[0], r[1], r[2]);
  }
};

}  // namespace orc
