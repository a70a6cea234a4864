// Debug print helpers of the reference's stage interface
// (pikoc/api/include/piko/helperRoutines.h).
#ifndef PIKO_COMPAT_HELPER_ROUTINES_H
#define PIKO_COMPAT_HELPER_ROUTINES_H

#ifdef __PIKOC_DEVICE__
inline void printInt(int v) { printf("%d\n", v); }
inline void printFloat(float v) { printf("%f\n", (double)v); }
#endif

#endif
