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

#endif
