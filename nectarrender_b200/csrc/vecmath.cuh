// vecmath.cuh — float3 arithmetic with the reference's operation order.
//
// The reference's Vector/Color templates (nectar_render/csrc/core/include/
// core/vector.h:16-519) define every operator as an element loop on a copy
// (`result = u; result op= v`). The functions below write the same scalar
// expression trees so that, compiled with the same fast-math flags, the same
// multiply/add pairs contract into the same FMAs. Division and reciprocal
// forms are kept exactly: `u / float` is `(1/t) * u` (vector.h:251-254),
// `u / v` adds FMIN to the divisor (vector.h:82-88, 245-250), `normalize` is
// `v / length` (vector.h:268-269).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#ifndef NR_HD
#define NR_HD __host__ __device__ __forceinline__
#endif

namespace nr {

// nectar_render/csrc/core/include/core/constants.h:7-13
constexpr float EPS = 1e-4f;
constexpr float FMIN = 1e-8f;
constexpr float FMAX = 1e32f;
constexpr float PI = 3.1415926535897932385f;
constexpr float PI2 = PI * 2.0f;
constexpr float PI4 = PI2 * PI2;  // 4*pi^2, as in the reference

struct V3 {
  float x, y, z;
};
struct V2 {
  float x, y;
};

NR_HD V3 v3(float a, float b, float c) { return V3{a, b, c}; }
NR_HD V3 v3(float a) { return V3{a, a, a}; }
NR_HD float comp(const V3& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

NR_HD V3 operator+(const V3& a, const V3& b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
NR_HD V3 operator-(const V3& a, const V3& b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
NR_HD V3 operator*(const V3& a, const V3& b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
NR_HD V3 operator*(const V3& a, float t) { return V3{a.x * t, a.y * t, a.z * t}; }
NR_HD V3 operator*(float t, const V3& a) { return V3{a.x * t, a.y * t, a.z * t}; }
NR_HD V3 operator+(const V3& a, float t) { return V3{a.x + t, a.y + t, a.z + t}; }
NR_HD V3 operator-(const V3& a, float t) { return V3{a.x - t, a.y - t, a.z - t}; }
NR_HD V3 operator-(const V3& a) { return V3{-a.x, -a.y, -a.z}; }
// u / t == (1/t) * u  (vector.h:251-254)
NR_HD V3 operator/(const V3& a, float t) {
  float r = 1.0f / t;
  return V3{a.x * r, a.y * r, a.z * r};
}
// u / v : elementwise u / (v + FMIN)  (vector.h:82-88)
NR_HD V3 operator/(const V3& a, const V3& b) {
  return V3{a.x / (b.x + FMIN), a.y / (b.y + FMIN), a.z / (b.z + FMIN)};
}
NR_HD V3& operator+=(V3& a, const V3& b) {
  a.x += b.x;
  a.y += b.y;
  a.z += b.z;
  return a;
}
NR_HD V3& operator*=(V3& a, const V3& b) {
  a.x *= b.x;
  a.y *= b.y;
  a.z *= b.z;
  return a;
}

// length_squared: (e0*e0 + e1*e1) then += e2*e2  (vector.h:100-108)
NR_HD float length_squared(const V3& v) {
  float o = v.x * v.x + v.y * v.y;
  o += v.z * v.z;
  return o;
}
NR_HD float length(const V3& v) { return sqrtf(length_squared(v)); }
NR_HD V3 normalize(const V3& v) { return v / length(v); }
NR_HD bool near_zero(const V3& v) { return length(v) < 1e-8f; }

NR_HD float dot(const V3& u, const V3& v) { return u.x * v.x + u.y * v.y + u.z * v.z; }
NR_HD V3 cross(const V3& u, const V3& v) {
  return V3{u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}
// vector.h:469-474
NR_HD V3 reflect(const V3& v, const V3& n) { return v - 2.0f * dot(v, n) * n; }
// vector.h:476-485; the reference evaluates 1.0 - |perp|^2 in double.
NR_HD V3 refract(const V3& uv, const V3& n, float ior) {
  float cos_theta = fminf(dot(-uv, n), 1.0f);
  V3 perp = ior * (uv + cos_theta * n);
  V3 parallel = -sqrtf(fabsf((float)(1.0 - (double)length_squared(perp)))) * n;
  return perp + parallel;
}

// Matrix3 (nectar_render/csrc/core/include/core/matrix.h:6-62), row major.
struct M3 {
  float m[3][3];
};
NR_HD V3 mul(const M3& a, const V3& v) {
  return V3{a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z,
            a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
            a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z};
}

// Orthonormal basis around w (nectar_render/csrc/core/include/core/onb.h:5-24).
struct ONB {
  V3 u, v, w;
};
NR_HD ONB make_onb(const V3& n) {
  ONB b;
  b.w = normalize(n);
  V3 a = (fabsf(b.w.x) > 0.9f) ? V3{0.0f, 1.0f, 0.0f} : V3{1.0f, 0.0f, 0.0f};
  b.v = normalize(cross(b.w, a));
  b.u = cross(b.w, b.v);
  return b;
}
// (v[0]*u) + (v[1]*v) + (v[2]*w)  (onb.h:20-22)
NR_HD V3 onb_transform(const ONB& b, const V3& v) {
  return (v.x * b.u) + (v.y * b.v) + (v.z * b.w);
}

}  // namespace nr
