// Device-side helpers of the reference's stage interface
// (pikoc/api/include/piko/deviceFunctions.h).  Stage code compiled here runs on
// the GPU through NVRTC; `__constant__` in stage code (a qualifier the
// reference's compiler accepts on pointer parameters, rasterMacros.h:14) is
// dropped, as the reference's CPU backend drops it.
#ifndef PIKO_COMPAT_DEVICE_FUNCTIONS_H
#define PIKO_COMPAT_DEVICE_FUNCTIONS_H

#ifdef __PIKOC_DEVICE__
#ifdef __constant__
#undef __constant__
#endif
#define __constant__

// thread and block of the current process launch
inline int getTID() { return (int)threadIdx.x; }
inline int getBlockID() { return (int)blockIdx.x; }
inline int getNumThreads() { return (int)blockDim.x; }
inline int getGID() { return (int)(blockIdx.x * blockDim.x + threadIdx.x); }
#endif

#endif
