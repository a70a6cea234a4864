// Stand-in for <math.h> in stage code compiled by NVRTC, which has no C
// library headers: the math functions stage code calls are NVRTC built-ins.
#ifndef PIKO_NVRTC_MATH_H
#define PIKO_NVRTC_MATH_H
#endif
