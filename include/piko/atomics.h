// Atomics of the reference's stage interface (pikoc/api/include/piko/atomics.h),
// namespace piko; device code only.  On the GPU these are real atomics (the
// reference's CPU backend uses plain read-modify-writes, which race when its
// runner uses several threads).
#ifndef PIKO_COMPAT_ATOMICS_H
#define PIKO_COMPAT_ATOMICS_H

#ifdef __PIKOC_DEVICE__
namespace piko {
inline int atomicIncrement(int* v) { return ::atomicAdd(v, 1); }
inline int atomicDecrement(int* v) { return ::atomicSub(v, 1); }
inline int atomicMin(int* v, int x) { return ::atomicMin(v, x); }
inline int atomicMinLocal(int* v, int x) { return ::atomicMin(v, x); }
inline int atomicAdd(int* v, int x) { return ::atomicAdd(v, x); }
inline float atomicAdd(float* v, float x) { return ::atomicAdd(v, x); }
}  // namespace piko
#endif

#endif
