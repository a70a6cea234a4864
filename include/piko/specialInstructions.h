// Bit casts of the reference's stage interface (pikoc/api/include/piko/specialInstructions.h).
#ifndef PIKO_COMPAT_SPECIAL_INSTRUCTIONS_H
#define PIKO_COMPAT_SPECIAL_INSTRUCTIONS_H
#ifdef __PIKOC_DEVICE__
inline int float_as_int(float f) { return __float_as_int(f); }
inline float int_as_float(int d) { return __int_as_float(d); }
#else
#include <cstring>
inline int float_as_int(float f) { int i; std::memcpy(&i, &f, 4); return i; }
inline float int_as_float(int d) { float f; std::memcpy(&f, &d, 4); return f; }
#endif
#endif
