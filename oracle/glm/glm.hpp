// Minimal GLM-compatible subset, written from the mathematics, used only to
// compile the reference's own physics sources (src/physics/*.cpp) as the CPU
// baseline and FP32 cross-check of the oracle.  GLM itself is not installed
// here.  Float vectors, column-major matrices (m[col][row]) and (w,x,y,z)
// quaternion construction follow GLM's documented conventions.
#pragma once
#include <cmath>
#include <algorithm>
#include <type_traits>
#include <cstdint>
#include <cstddef>
#include <limits>

namespace glm {

struct vec3 {
  float x, y, z;
  vec3() : x(0), y(0), z(0) {}
  template <class T, class = typename std::enable_if<std::is_arithmetic<T>::value>::type>
  explicit vec3(T s) : x(float(s)), y(float(s)), z(float(s)) {}
  template <class A, class B, class C>
  vec3(A a, B b, C c) : x(float(a)), y(float(b)), z(float(c)) {}
  float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  const float& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  vec3& operator+=(const vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  vec3& operator-=(const vec3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  vec3& operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
  vec3& operator/=(float s) { x /= s; y /= s; z /= s; return *this; }
};
inline vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
inline vec3 operator*(const vec3& a, const vec3& b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline vec3 operator*(const vec3& a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator*(float s, const vec3& a) { return vec3(s * a.x, s * a.y, s * a.z); }
inline vec3 operator/(const vec3& a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }
inline vec3 operator/(const vec3& a, const vec3& b) { return vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline bool operator==(const vec3& a, const vec3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline bool operator!=(const vec3& a, const vec3& b) { return !(a == b); }

inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline vec3 cross(const vec3& a, const vec3& b) {
  return vec3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
inline float length(const vec3& a) { return std::sqrt(dot(a, a)); }
inline vec3 normalize(const vec3& a) { return a * (1.0f / std::sqrt(dot(a, a))); }
inline vec3 min(const vec3& a, const vec3& b) {
  return vec3(std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z));
}
inline vec3 max(const vec3& a, const vec3& b) {
  return vec3(std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z));
}
inline vec3 abs(const vec3& a) { return vec3(std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)); }
inline vec3 floor(const vec3& a) { return vec3(std::floor(a.x), std::floor(a.y), std::floor(a.z)); }
template <class T>
inline T clamp(T v, T lo, T hi) { return std::min(std::max(v, lo), hi); }

struct ivec3 {
  int x, y, z;
  ivec3() : x(0), y(0), z(0) {}
  ivec3(int a, int b, int c) : x(a), y(b), z(c) {}
  ivec3(const vec3& v) : x(int(v.x)), y(int(v.y)), z(int(v.z)) {}
};

struct vec4 {
  float x, y, z, w;
  vec4() : x(0), y(0), z(0), w(0) {}
  template <class T, class = typename std::enable_if<std::is_arithmetic<T>::value>::type>
  explicit vec4(T s) : x(float(s)), y(float(s)), z(float(s)), w(float(s)) {}
  template <class A, class B, class C, class D>
  vec4(A a, B b, C c, D d) : x(float(a)), y(float(b)), z(float(c)), w(float(d)) {}
  vec4(const vec3& v, float s) : x(v.x), y(v.y), z(v.z), w(s) {}
  float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  const float& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};
inline vec4 operator+(const vec4& a, const vec4& b) { return vec4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline vec4 operator*(const vec4& a, float s) { return vec4(a.x * s, a.y * s, a.z * s, a.w * s); }

// Column-major 3x3: c[i] is column i.
struct mat3 {
  vec3 c[3];
  mat3() { c[0] = vec3(1, 0, 0); c[1] = vec3(0, 1, 0); c[2] = vec3(0, 0, 1); }
  explicit mat3(float d) { c[0] = vec3(d, 0, 0); c[1] = vec3(0, d, 0); c[2] = vec3(0, 0, d); }
  mat3(const vec3& a, const vec3& b, const vec3& d) { c[0] = a; c[1] = b; c[2] = d; }
  vec3& operator[](int i) { return c[i]; }
  const vec3& operator[](int i) const { return c[i]; }
};
inline vec3 operator*(const mat3& m, const vec3& v) {
  return vec3(m[0].x * v.x + m[1].x * v.y + m[2].x * v.z,
              m[0].y * v.x + m[1].y * v.y + m[2].y * v.z,
              m[0].z * v.x + m[1].z * v.y + m[2].z * v.z);
}
inline mat3 operator*(const mat3& a, const mat3& b) {
  return mat3(a * b[0], a * b[1], a * b[2]);
}
inline mat3 transpose(const mat3& m) {
  return mat3(vec3(m[0].x, m[1].x, m[2].x), vec3(m[0].y, m[1].y, m[2].y),
              vec3(m[0].z, m[1].z, m[2].z));
}

struct mat4 {
  vec4 c[4];
  mat4() { c[0] = vec4(1, 0, 0, 0); c[1] = vec4(0, 1, 0, 0); c[2] = vec4(0, 0, 1, 0); c[3] = vec4(0, 0, 0, 1); }
  explicit mat4(float d) { c[0] = vec4(d, 0, 0, 0); c[1] = vec4(0, d, 0, 0); c[2] = vec4(0, 0, d, 0); c[3] = vec4(0, 0, 0, d); }
  vec4& operator[](int i) { return c[i]; }
  const vec4& operator[](int i) const { return c[i]; }
};
inline vec4 operator*(const mat4& m, const vec4& v) {
  return m[0] * v.x + m[1] * v.y + m[2] * v.z + m[3] * v.w;
}
inline mat4 operator*(const mat4& a, const mat4& b) {
  mat4 r;
  for (int i = 0; i < 4; ++i) r[i] = a * b[i];
  return r;
}
inline mat4 translate(const mat4& m, const vec3& v) {
  mat4 r = m;
  r[3] = m[0] * v.x + m[1] * v.y + m[2] * v.z + m[3];
  return r;
}
inline mat4 scale(const mat4& m, const vec3& v) {
  mat4 r = m;
  r[0] = m[0] * v.x;
  r[1] = m[1] * v.y;
  r[2] = m[2] * v.z;
  return r;
}

// Quaternion: constructed as (w, x, y, z).
struct quat {
  float x, y, z, w;
  quat() : x(0), y(0), z(0), w(1) {}
  template <class A, class B, class C, class D>
  quat(A w_, B x_, C y_, D z_) : x(float(x_)), y(float(y_)), z(float(z_)), w(float(w_)) {}
  quat(float s, const vec3& v) : x(v.x), y(v.y), z(v.z), w(s) {}
  quat& operator+=(const quat& o) { x += o.x; y += o.y; z += o.z; w += o.w; return *this; }
};
inline quat operator*(const quat& p, const quat& q) {
  return quat(p.w * q.w - p.x * q.x - p.y * q.y - p.z * q.z,
              p.w * q.x + p.x * q.w + p.y * q.z - p.z * q.y,
              p.w * q.y + p.y * q.w + p.z * q.x - p.x * q.z,
              p.w * q.z + p.z * q.w + p.x * q.y - p.y * q.x);
}
inline quat operator*(const quat& q, float s) { return quat(q.w * s, q.x * s, q.y * s, q.z * s); }
inline quat operator*(float s, const quat& q) { return quat(q.w * s, q.x * s, q.y * s, q.z * s); }
inline quat operator+(const quat& a, const quat& b) { return quat(a.w + b.w, a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator*(const quat& q, const vec3& v) {
  vec3 u(q.x, q.y, q.z);
  vec3 t = cross(u, v) * 2.0f;
  return v + t * q.w + cross(u, t);
}
inline float length(const quat& q) { return std::sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z); }
inline quat normalize(const quat& q) {
  float len = length(q);
  if (len <= 0.0f) return quat(1, 0, 0, 0);
  float inv = 1.0f / len;
  return quat(q.w * inv, q.x * inv, q.y * inv, q.z * inv);
}
inline quat angleAxis(float angle, const vec3& axis) {
  float s = std::sin(angle * 0.5f);
  return quat(std::cos(angle * 0.5f), axis.x * s, axis.y * s, axis.z * s);
}
inline mat3 mat3_cast(const quat& q) {
  float qxx = q.x * q.x, qyy = q.y * q.y, qzz = q.z * q.z;
  float qxz = q.x * q.z, qxy = q.x * q.y, qyz = q.y * q.z;
  float qwx = q.w * q.x, qwy = q.w * q.y, qwz = q.w * q.z;
  mat3 r;
  r[0] = vec3(1.0f - 2.0f * (qyy + qzz), 2.0f * (qxy + qwz), 2.0f * (qxz - qwy));
  r[1] = vec3(2.0f * (qxy - qwz), 1.0f - 2.0f * (qxx + qzz), 2.0f * (qyz + qwx));
  r[2] = vec3(2.0f * (qxz + qwy), 2.0f * (qyz - qwx), 1.0f - 2.0f * (qxx + qyy));
  return r;
}
inline mat4 mat4_cast(const quat& q) {
  mat3 m = mat3_cast(q);
  mat4 r(1.0f);
  for (int i = 0; i < 3; ++i) r[i] = vec4(m[i], 0.0f);
  return r;
}

}  // namespace glm
