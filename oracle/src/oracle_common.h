/* TEST INFRASTRUCTURE — the oracle's CPU restatement, never the product path.
 *
 * Scalar helpers shared by oracle_raster.c and oracle_reyes.c.  They pin the
 * arithmetic of the reference's CPU backend (g++ on x86-64, SSE single
 * precision, no FMA contraction, wrapping int32) so the restatement and the
 * device kernels can be compared bit for bit.
 */
#ifndef PIKO_ORACLE_COMMON_H
#define PIKO_ORACLE_COMMON_H

#include <stdint.h>
#include <string.h>
#include <math.h>
#include <limits.h>

/* wrapping int32 arithmetic (the oracle is built with -fwrapv as well) */
static inline int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
static inline int32_t wsub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
static inline int32_t wmul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }
static inline int32_t wshl(int32_t a, int s) { return (int32_t)((uint32_t)a << s); }

/* (int)f as x86-64 cvttss2si computes it: truncation, and INT_MIN for NaN or
 * values outside the int32 range. */
static inline int32_t cvt_i32(float f)
{
  if (!(f >= -2147483648.0f && f < 2147483648.0f)) return INT32_MIN;
  return (int32_t)f;
}

/* (unsigned)f as g++ emits it on x86-64: a 64-bit cvttss2si whose low 32 bits
 * are kept (0 for NaN and for |f| >= 2^63). */
static inline uint32_t cvt_u32(float f)
{
  if (!(f > -9223372036854775808.0f && f < 9223372036854775808.0f)) return 0u;
  return (uint32_t)(uint64_t)(int64_t)f;
}

static inline int32_t f2bits(float f) { int32_t i; memcpy(&i, &f, 4); return i; }
static inline float bits2f(int32_t i) { float f; memcpy(&f, &i, 4); return f; }

/* std::min / std::max as the reference's piko::fminf/fmaxf resolve on the CPU
 * (piko/math.h:24-52): b if b < a else a, which differs from C fminf on NaN. */
static inline float std_minf(float a, float b) { return (b < a) ? b : a; }
static inline float std_maxf(float a, float b) { return (a < b) ? b : a; }
static inline int imin_(int a, int b) { return a < b ? a : b; }
static inline int imax_(int a, int b) { return a > b ? a : b; }

/* Sample positions of the multi-sample Reyes variant (no reference
 * counterpart: the reference samples each pixel once, at its centre).  Sample
 * s of pixel (x, y), s < 4, lies in quadrant (s & 1, s >> 1) of the pixel at a
 * jitter drawn from this integer hash of (seed, x, y, 2s + axis); the device
 * kernels use the same function. */
static inline uint32_t sample_hash(uint32_t seed, uint32_t x, uint32_t y, uint32_t k)
{
  uint32_t h = seed * 0x9E3779B1u;
  h ^= x * 0x85EBCA77u;
  h ^= y * 0xC2B2AE3Du;
  h ^= k * 0x27D4EB2Fu;
  h ^= h >> 16; h *= 0x7FEB352Du;
  h ^= h >> 15; h *= 0x846CA68Bu;
  h ^= h >> 16;
  return h;
}
static inline void sample_pos(int spp, uint32_t seed, int x, int y, int s, float* px, float* py)
{
  if (spp == 1) { *px = (float)x + 0.5f; *py = (float)y + 0.5f; return; }
  const float jx = (float)(sample_hash(seed, (uint32_t)x, (uint32_t)y, 2u * (uint32_t)s) >> 8) * 5.9604644775390625e-8f;
  const float jy = (float)(sample_hash(seed, (uint32_t)x, (uint32_t)y, 2u * (uint32_t)s + 1u) >> 8) * 5.9604644775390625e-8f;
  *px = (float)x + ((float)(s & 1) + jx) * 0.5f;
  *py = (float)y + ((float)(s >> 1) + jy) * 0.5f;
}
/* depth order of the sample resolve: total over non-NaN floats, -0 == +0 */
static inline uint32_t zorder_u(float z)
{
  uint32_t b; memcpy(&b, &z, 4);
  if (b == 0x80000000u) b = 0u;
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

#endif
