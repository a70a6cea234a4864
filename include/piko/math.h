// Math helpers of the reference's stage interface (pikoc/api/include/piko/math.h),
// namespace piko, with the semantics of the reference's CPU backend
// (math.h:17-216 CPU branches, 258-330): std::min / std::max comparisons,
// IEEE division for rcp_approx, wrapping imad, toABGR truncating without
// saturation, fromABGR dividing by 255, unfused a * b + c.  Device code only
// (stage code under NVRTC); every function is an inline device function
// there (-default-device).
#ifndef PIKO_COMPAT_MATH_H
#define PIKO_COMPAT_MATH_H

#include "builtinTypes.h"

#ifdef __PIKOC_DEVICE__
namespace piko {

// std::min / std::max on floats: the second argument only when it compares
// strictly less / greater (NaN handling differs from fminf / fmaxf)
inline float fminf(float x, float y) { return (y < x) ? y : x; }
inline float fmaxf(float x, float y) { return (x < y) ? y : x; }
inline double fmin(double x, double y) { return (y < x) ? y : x; }
inline double fmax(double x, double y) { return (x < y) ? y : x; }
inline float floorf(float x) { return ::floorf(x); }
inline double floor(double x) { return ::floor(x); }
inline float ceilf(float x) { return ::ceilf(x); }
inline double ceil(double x) { return ::ceil(x); }
inline float sqrtf(float x) { return __fsqrt_rn(x); }
inline double sqrt(double x) { return __dsqrt_rn(x); }
inline float powf(float x, float y) { return ::powf(x, y); }
inline float sinf(float x) { return ::sinf(x); }
inline float cosf(float x) { return ::cosf(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline int ffsll(unsigned long long x) { return __ffsll((long long)x); }
inline int popcll(unsigned long long x) { return __popcll(x); }
inline int imax(int a, int b) { return a > b ? a : b; }
inline int imin(int a, int b) { return a < b ? a : b; }

inline void membar_bin() {}
inline void BinSynchronize() {}
inline int max_max(int a, int b, int c) { return imax(imax(a, b), c); }
inline int min_min(int a, int b, int c) { return imin(imin(a, b), c); }
inline int max_add(int a, int b, int c) { return (int)((unsigned)imax(a, b) + (unsigned)c); }
inline int min_add(int a, int b, int c) { return (int)((unsigned)imin(a, b) + (unsigned)c); }
inline int shl_add(int a, unsigned b, int c) { return (int)(((unsigned)a << b) + (unsigned)c); }
inline int shr_add(int a, unsigned b, int c) { return (int)((unsigned)(a >> b) + (unsigned)c); }
inline unsigned shl_max(unsigned a, unsigned b, unsigned c) { return (unsigned)imax((int)(a << b), (int)c); }
inline unsigned shr_max(unsigned a, unsigned b, unsigned c) { return (unsigned)imax((int)(a >> b), (int)c); }
inline unsigned shl_min(unsigned a, unsigned b, unsigned c) { return (unsigned)imin((int)(a << b), (int)c); }
inline unsigned shr_min(unsigned a, unsigned b, unsigned c) { return (unsigned)imin((int)(a >> b), (int)c); }
inline unsigned add_add(unsigned a, unsigned b, unsigned c) { return a + b + c; }
inline unsigned sub_add(unsigned a, unsigned b, unsigned c) { return a - b + c; }
inline unsigned add_sub(unsigned a, unsigned b, unsigned c) { return a + b - c; }
inline int imad(int a, int b, int c) { return (int)((unsigned)a * (unsigned)b + (unsigned)c); }
inline float rcp_approx(float a) { return __fdiv_rn(1.0f, a); }
// (unsigned)a on the CPU: the low 32 bits of a 64-bit truncation
inline unsigned f32_to_u32_sat_rmi(float a)
{
  if (::fabsf(a) < 2147483648.0f) return (unsigned)__float2int_rz(a);
  return (a > -9223372036854775808.0f && a < 9223372036854775808.0f) ? (unsigned)__float2ll_rz(a) : 0u;
}
inline float fma_rm(float a, float b, float c) { return __fadd_rn(__fmul_rn(a, b), c); }
inline unsigned idiv_fast(unsigned a, unsigned b) { return a / b; }

inline unsigned toABGR(cvec3f c)
{
  return 0xff000000u | (f32_to_u32_sat_rmi(c.z * 255.0f) << 16) | (f32_to_u32_sat_rmi(c.y * 255.0f) << 8) |
         f32_to_u32_sat_rmi(c.x * 255.0f);
}
inline cvec3f fromABGR(unsigned c)
{
  return gencvec3f((float)(c & 255u) / 255.0f, (float)((c >> 8) & 255u) / 255.0f, (float)((c >> 16) & 255u) / 255.0f);
}

inline float magnitude(cvec3f v) { return piko::sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
inline float magnitude(cvec4f v) { return piko::sqrtf(v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w); }
inline cvec3f normalize(cvec3f v)
{
  const float m = magnitude(v);
  v.x /= m;
  v.y /= m;
  v.z /= m;
  return v;
}
inline float distance(cvec2f a, cvec2f b)
{
  const cvec2f c = a - b;
  return piko::sqrtf(c.x * c.x + c.y * c.y);
}
inline float distance(cvec4f a, cvec4f b) { return magnitude(a - b); }
inline float dotvec(const cvec3f& a, const cvec3f& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline cvec4f cross(cvec4f a, cvec4f b)
{
  cvec4f r;
  r.x = a.y * b.z - a.z * b.y;
  r.y = a.z * b.x - a.x * b.z;
  r.z = a.x * b.y - a.y * b.x;
  r.w = 0.0f;
  return r;
}
inline cvec3f cross(cvec3f a, cvec3f b) { return ::cross(a, b); }
// column-major matrix times (v, 1) / times v, sums left to right
inline cvec4f matmultfloat4(const float* m, cvec3f v)
{
  return gencvec4f(m[0] * v.x + m[4] * v.y + m[8] * v.z + m[12], m[1] * v.x + m[5] * v.y + m[9] * v.z + m[13],
                   m[2] * v.x + m[6] * v.y + m[10] * v.z + m[14], m[3] * v.x + m[7] * v.y + m[11] * v.z + m[15]);
}
inline cvec4f matmultfloat4(const float* m, cvec4f v)
{
  return gencvec4f(m[0] * v.x + m[4] * v.y + m[8] * v.z + m[12] * v.w,
                   m[1] * v.x + m[5] * v.y + m[9] * v.z + m[13] * v.w,
                   m[2] * v.x + m[6] * v.y + m[10] * v.z + m[14] * v.w,
                   m[3] * v.x + m[7] * v.y + m[11] * v.z + m[15] * v.w);
}

}  // namespace piko
#endif  // __PIKOC_DEVICE__

#endif
