// Small vector types of the reference's stage interface (pikoc/api/include/piko/cvec.h):
// flat structs with x, y, z, w members, gencvec* constructors and the usual
// arithmetic, usable on the host and, in stage code compiled by NVRTC with
// -default-device, on the device.
#ifndef PIKO_COMPAT_CVEC_H
#define PIKO_COMPAT_CVEC_H

#include "maths.h"

#ifndef M_PI
#define M_PI 3.1415926f
#endif

struct cvec2f { float x, y; };
struct cvec3f { float x, y, z; };
struct cvec4f { float x, y, z, w; };
struct cvec2i { int x, y; };
struct cvec3i { int x, y, z; };
struct cvec4i { int x, y, z, w; };

inline cvec2f gencvec2f(const float& x, const float& y) { cvec2f v; v.x = x; v.y = y; return v; }
inline cvec3f gencvec3f(const float& x, const float& y, const float& z) { cvec3f v; v.x = x; v.y = y; v.z = z; return v; }
inline cvec4f gencvec4f(const float& x, const float& y, const float& z, const float& w)
{
  cvec4f v; v.x = x; v.y = y; v.z = z; v.w = w; return v;
}
inline cvec2i gencvec2i(const int& x, const int& y) { cvec2i v; v.x = x; v.y = y; return v; }
inline cvec3i gencvec3i(const int& x, const int& y, const int& z) { cvec3i v; v.x = x; v.y = y; v.z = z; return v; }
inline cvec4i gencvec4i(const int& x, const int& y, const int& z, const int& w)
{
  cvec4i v; v.x = x; v.y = y; v.z = z; v.w = w; return v;
}

inline void zerovec(cvec2f& v) { v.x = v.y = 0.0f; }
inline void zerovec(cvec3f& v) { v.x = v.y = v.z = 0.0f; }
inline void zerovec(cvec4f& v) { v.x = v.y = v.z = v.w = 0.0f; }
inline void zerovec(cvec2i& v) { v.x = v.y = 0; }

inline cvec2f addvec(const cvec2f& a, const cvec2f& b) { return gencvec2f(a.x + b.x, a.y + b.y); }
inline cvec3f addvec(const cvec3f& a, const cvec3f& b) { return gencvec3f(a.x + b.x, a.y + b.y, a.z + b.z); }
inline cvec4f addvec(const cvec4f& a, const cvec4f& b) { return gencvec4f(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline cvec2f subvec(const cvec2f& a, const cvec2f& b) { return gencvec2f(a.x - b.x, a.y - b.y); }
inline cvec3f subvec(const cvec3f& a, const cvec3f& b) { return gencvec3f(a.x - b.x, a.y - b.y, a.z - b.z); }
inline cvec4f subvec(const cvec4f& a, const cvec4f& b) { return gencvec4f(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
inline cvec2f mulvec(const cvec2f& a, const float& k) { return gencvec2f(a.x * k, a.y * k); }
inline cvec3f mulvec(const cvec3f& a, const float& k) { return gencvec3f(a.x * k, a.y * k, a.z * k); }
inline cvec4f mulvec(const cvec4f& a, const float& k) { return gencvec4f(a.x * k, a.y * k, a.z * k, a.w * k); }
inline void mulvecInplace(cvec3f& a, const float& k) { a.x = a.x * k; a.y = a.y * k; a.z = a.z * k; }
inline void mulvecInplace(cvec4f& a, const float& k) { a.x = a.x * k; a.y = a.y * k; a.z = a.z * k; a.w = a.w * k; }

inline cvec2f operator+(const cvec2f& a, const cvec2f& b) { return addvec(a, b); }
inline cvec3f operator+(const cvec3f& a, const cvec3f& b) { return addvec(a, b); }
inline cvec4f operator+(const cvec4f& a, const cvec4f& b) { return addvec(a, b); }
inline cvec2f operator-(const cvec2f& a, const cvec2f& b) { return subvec(a, b); }
inline cvec3f operator-(const cvec3f& a, const cvec3f& b) { return subvec(a, b); }
inline cvec4f operator-(const cvec4f& a, const cvec4f& b) { return subvec(a, b); }
inline cvec2f operator*(const cvec2f& a, const float& k) { return mulvec(a, k); }
inline cvec3f operator*(const cvec3f& a, const float& k) { return mulvec(a, k); }
inline cvec4f operator*(const cvec4f& a, const float& k) { return mulvec(a, k); }
inline cvec2f operator*(const float& k, const cvec2f& a) { return mulvec(a, k); }
inline cvec3f operator*(const float& k, const cvec3f& a) { return mulvec(a, k); }
inline cvec4f operator*(const float& k, const cvec4f& a) { return mulvec(a, k); }
inline cvec3f& operator+=(cvec3f& a, const cvec3f& b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
inline cvec3f& operator-=(cvec3f& a, const cvec3f& b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
inline cvec3f& operator*=(cvec3f& a, const float& k) { a.x *= k; a.y *= k; a.z *= k; return a; }

inline float magsqr(const cvec3f& v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
inline float dotvec(const cvec2f& a, const cvec2f& b) { return a.x * b.x + a.y * b.y; }
inline float dotvec(const cvec3f& a, const cvec3f& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dotvec(const cvec4f& a, const cvec4f& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline cvec3f cross(const cvec3f& a, const cvec3f& b)
{
  return gencvec3f(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline cvec3f cvec4fxyz(cvec4f& v) { return gencvec3f(v.x, v.y, v.z); }

#endif
