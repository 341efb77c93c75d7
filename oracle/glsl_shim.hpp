// The GLSL vocabulary the reference's fragment shaders use, in single
// precision, so that their translated source (glsl_to_cpp.py) compiles as C++
// — test infrastructure only (oracle/shade_harness.cpp).
//
// Built-ins follow the GLSL definitions: min(x, y) = y < x ? y : x,
// max(x, y) = x < y ? y : x, mix(x, y, a) = x (1 - a) + y a,
// reflect(I, N) = I - 2 dot(N, I) N, normalize(v) = v * (1 / sqrt(dot(v, v))),
// dot summed x, y, z in order.  Texture lookups call the oracle's samplers.
#pragma once

#include <cmath>
#include <cstdint>

extern "C" {
void orc_sample_cube(const uint8_t* sky, int32_t face, const float dir[3], float out[4]);
void orc_sample_2d(const uint8_t* img, int32_t w, int32_t h, float s, float t, float out[4]);
}

namespace glsl_shim {

struct vec2 {
  float x, y;
  vec2() : x(0), y(0) {}
  template <class A> explicit vec2(A a) : x(float(a)), y(float(a)) {}
  template <class A, class B> vec2(A a, B b) : x(float(a)), y(float(b)) {}
};

struct vec3 {
  union { float x; float r; };
  union { float y; float g; };
  union { float z; float b; };
  vec3() : x(0), y(0), z(0) {}
  template <class A> explicit vec3(A a) : x(float(a)), y(float(a)), z(float(a)) {}
  template <class A, class B, class C> vec3(A a, B b, C c) : x(float(a)), y(float(b)), z(float(c)) {}
};

struct vec4 {
  union { float x; float r; };
  union { float y; float g; };
  union { float z; float b; };
  union { float w; float a; };
  vec4() : x(0), y(0), z(0), w(0) {}
  template <class A> explicit vec4(A s) : x(float(s)), y(float(s)), z(float(s)), w(float(s)) {}
  template <class A> vec4(const vec3& v, A s) : x(v.x), y(v.y), z(v.z), w(float(s)) {}
  template <class A, class B, class C, class D>
  vec4(A p, B q, C s, D t) : x(float(p)), y(float(q)), z(float(s)), w(float(t)) {}
};

struct mat4 { float m[16]; };
struct sampler2D { const uint8_t* img = nullptr; int w = 0, h = 0; const float* value = nullptr; };
struct samplerCube { const uint8_t* faces = nullptr; int face = 0; };

// component-wise arithmetic; scalars are converted to float first
#define AQ_SHIM_OPS(V, N)                                                                          \
  inline V operator+(V a, const V& b) { for (int i = 0; i < N; ++i) (&a.x)[i] = (&a.x)[i] + (&b.x)[i]; return a; } \
  inline V operator-(V a, const V& b) { for (int i = 0; i < N; ++i) (&a.x)[i] = (&a.x)[i] - (&b.x)[i]; return a; } \
  inline V operator*(V a, const V& b) { for (int i = 0; i < N; ++i) (&a.x)[i] = (&a.x)[i] * (&b.x)[i]; return a; } \
  inline V operator/(V a, const V& b) { for (int i = 0; i < N; ++i) (&a.x)[i] = (&a.x)[i] / (&b.x)[i]; return a; } \
  template <class S> inline V operator*(V a, S s) { const float f = float(s); for (int i = 0; i < N; ++i) (&a.x)[i] = (&a.x)[i] * f; return a; } \
  template <class S> inline V operator*(S s, V a) { const float f = float(s); for (int i = 0; i < N; ++i) (&a.x)[i] = f * (&a.x)[i]; return a; } \
  template <class S> inline V operator/(V a, S s) { const float f = float(s); for (int i = 0; i < N; ++i) (&a.x)[i] = (&a.x)[i] / f; return a; } \
  template <class S> inline V operator+(V a, S s) { const float f = float(s); for (int i = 0; i < N; ++i) (&a.x)[i] = (&a.x)[i] + f; return a; } \
  template <class S> inline V operator-(V a, S s) { const float f = float(s); for (int i = 0; i < N; ++i) (&a.x)[i] = (&a.x)[i] - f; return a; } \
  template <class S> inline V operator-(S s, V a) { const float f = float(s); for (int i = 0; i < N; ++i) (&a.x)[i] = f - (&a.x)[i]; return a; } \
  inline V operator-(V a) { for (int i = 0; i < N; ++i) (&a.x)[i] = -(&a.x)[i]; return a; } \
  inline V& operator+=(V& a, const V& b) { a = a + b; return a; } \
  inline V& operator-=(V& a, const V& b) { a = a - b; return a; } \
  template <class S> inline V& operator/=(V& a, S s) { a = a / s; return a; } \
  template <class S> inline V& operator*=(V& a, S s) { a = a * s; return a; } \
  inline float dot(const V& a, const V& b) { float s = a.x * b.x; for (int i = 1; i < N; ++i) s = s + (&a.x)[i] * (&b.x)[i]; return s; } \
  inline V min(V a, const V& b) { for (int i = 0; i < N; ++i) (&a.x)[i] = (&b.x)[i] < (&a.x)[i] ? (&b.x)[i] : (&a.x)[i]; return a; } \
  inline V max(V a, const V& b) { for (int i = 0; i < N; ++i) (&a.x)[i] = (&a.x)[i] < (&b.x)[i] ? (&b.x)[i] : (&a.x)[i]; return a; } \
  inline V normalize(const V& v) { return v * (1.0f / std::sqrt(dot(v, v))); } \
  inline float length(const V& v) { return std::sqrt(dot(v, v)); } \
  inline V reflect(const V& i, const V& n) { return i - n * dot(n, i) * 2.0f; } \
  inline V mix(const V& x, const V& y, float a) { return x * (1.0f - a) + y * a; }

AQ_SHIM_OPS(vec2, 2)
AQ_SHIM_OPS(vec3, 3)
AQ_SHIM_OPS(vec4, 4)
#undef AQ_SHIM_OPS

inline float min(float x, float y) { return y < x ? y : x; }
inline float max(float x, float y) { return x < y ? y : x; }
inline float max(int x, float y) { return max(float(x), y); }
inline float max(float x, int y) { return max(x, float(y)); }
inline float exp(float x) { return std::exp(x); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float abs(float x) { return std::fabs(x); }
inline float pow(float x, float y) { return std::pow(x, y); }
inline float pow(float x, int y) { return std::pow(x, float(y)); }
inline float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }

inline vec2 xy(const vec3& v) { return vec2(v.x, v.y); }
inline vec2 xy(const vec4& v) { return vec2(v.x, v.y); }
inline vec2 xz(const vec3& v) { return vec2(v.x, v.z); }
inline vec3 xyz(const vec4& v) { return vec3(v.x, v.y, v.z); }
inline vec3 rgb(const vec4& v) { return vec3(v.x, v.y, v.z); }
inline vec4 set_rgb(vec4 v, const vec3& c) { v.x = c.x; v.y = c.y; v.z = c.z; return v; }

inline vec4 texture(const sampler2D& s, const vec2& c) {
  if (s.value) return vec4(s.value[0], s.value[1], s.value[2], s.value[3]);
  float o[4];
  orc_sample_2d(s.img, s.w, s.h, c.x, c.y, o);
  return vec4(o[0], o[1], o[2], o[3]);
}

inline vec4 texture(const samplerCube& s, const vec3& d) {
  const float dd[3] = {d.x, d.y, d.z};
  float o[4];
  orc_sample_cube(s.faces, s.face, dd, o);
  return vec4(o[0], o[1], o[2], o[3]);
}

}  // namespace glsl_shim
