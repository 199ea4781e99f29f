// TEST INFRASTRUCTURE ONLY.  A minimal, project-written stand-in for <glm/glm.hpp>, sufficient to
// compile the reference's cuda_rasterizer/ sources (glm is not installed in this image).  It
// provides only what those sources use: vec3, vec4, column-major mat3 with m[col][row] indexing,
// their arithmetic, transpose, dot, length and max(vec3, scalar).  Products are evaluated term by
// term in column-major order, r[c][i] = a[0][i] b[c][0] + a[1][i] b[c][1] + a[2][i] b[c][2], and
// vector operators act component-wise with the left operand first, which is how glm 0.9.x
// evaluates them.
#pragma once
#include <cmath>

#if defined(__CUDACC__)
#define OMNIGS_GLM_FN __host__ __device__ __forceinline__
#else
#define OMNIGS_GLM_FN inline
#endif

namespace glm {

struct vec3 {
  float x, y, z;
  OMNIGS_GLM_FN vec3() = default;
  OMNIGS_GLM_FN explicit vec3(float s) : x(s), y(s), z(s) {}
  template <class A, class B, class C>
  OMNIGS_GLM_FN vec3(A a, B b, C c) : x((float)a), y((float)b), z((float)c) {}
  OMNIGS_GLM_FN float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  OMNIGS_GLM_FN const float& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  OMNIGS_GLM_FN vec3& operator+=(const vec3& v) { x += v.x; y += v.y; z += v.z; return *this; }
  OMNIGS_GLM_FN vec3& operator-=(const vec3& v) { x -= v.x; y -= v.y; z -= v.z; return *this; }
  OMNIGS_GLM_FN vec3& operator+=(float s) { x += s; y += s; z += s; return *this; }
  OMNIGS_GLM_FN vec3& operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
  OMNIGS_GLM_FN vec3& operator/=(float s) { x /= s; y /= s; z /= s; return *this; }
};

struct vec4 {
  float x, y, z, w;
  OMNIGS_GLM_FN vec4() = default;
  template <class A, class B, class C, class D>
  OMNIGS_GLM_FN vec4(A a, B b, C c, D d) : x((float)a), y((float)b), z((float)c), w((float)d) {}
};

OMNIGS_GLM_FN vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
OMNIGS_GLM_FN vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
OMNIGS_GLM_FN vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
OMNIGS_GLM_FN vec3 operator*(const vec3& a, const vec3& b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
OMNIGS_GLM_FN vec3 operator*(float s, const vec3& v) { return vec3(s * v.x, s * v.y, s * v.z); }
OMNIGS_GLM_FN vec3 operator*(const vec3& v, float s) { return vec3(v.x * s, v.y * s, v.z * s); }
OMNIGS_GLM_FN vec3 operator/(const vec3& v, float s) { return vec3(v.x / s, v.y / s, v.z / s); }
OMNIGS_GLM_FN vec3 operator+(const vec3& v, float s) { return vec3(v.x + s, v.y + s, v.z + s); }

struct mat3 {
  vec3 c[3];
  OMNIGS_GLM_FN mat3() = default;
  OMNIGS_GLM_FN explicit mat3(float s) {
    c[0] = vec3(s, 0.0f, 0.0f);
    c[1] = vec3(0.0f, s, 0.0f);
    c[2] = vec3(0.0f, 0.0f, s);
  }
  template <class A0, class A1, class A2, class A3, class A4, class A5, class A6, class A7, class A8>
  OMNIGS_GLM_FN mat3(A0 a0, A1 a1, A2 a2, A3 a3, A4 a4, A5 a5, A6 a6, A7 a7, A8 a8) {
    c[0] = vec3(a0, a1, a2);
    c[1] = vec3(a3, a4, a5);
    c[2] = vec3(a6, a7, a8);
  }
  OMNIGS_GLM_FN vec3& operator[](int i) { return c[i]; }
  OMNIGS_GLM_FN const vec3& operator[](int i) const { return c[i]; }
};

OMNIGS_GLM_FN mat3 operator*(const mat3& a, const mat3& b) {
  mat3 r;
  for (int col = 0; col < 3; ++col)
    for (int i = 0; i < 3; ++i) r[col][i] = a[0][i] * b[col][0] + a[1][i] * b[col][1] + a[2][i] * b[col][2];
  return r;
}
OMNIGS_GLM_FN mat3 operator*(float s, const mat3& m) {
  mat3 r;
  for (int col = 0; col < 3; ++col) r[col] = m[col] * s;
  return r;
}
OMNIGS_GLM_FN mat3 operator*(const mat3& m, float s) { return s * m; }
OMNIGS_GLM_FN mat3 transpose(const mat3& m) {
  mat3 r;
  for (int col = 0; col < 3; ++col)
    for (int i = 0; i < 3; ++i) r[col][i] = m[i][col];
  return r;
}
OMNIGS_GLM_FN float dot(const vec3& a, const vec3& b) {
  const vec3 t = a * b;
  return t.x + t.y + t.z;
}
OMNIGS_GLM_FN float length(const vec3& v) { return sqrtf(dot(v, v)); }
OMNIGS_GLM_FN float max_scalar(float a, float b) { return (a < b) ? b : a; }
OMNIGS_GLM_FN vec3 max(const vec3& v, float s) { return vec3(max_scalar(v.x, s), max_scalar(v.y, s), max_scalar(v.z, s)); }

}  // namespace glm
