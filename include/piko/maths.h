// Scalar constants of the reference's stage interface (pikoc/api/include/piko/maths.h).
#ifndef PIKO_COMPAT_MATHS_H
#define PIKO_COMPAT_MATHS_H
#ifndef PIKO_PI
#define PIKO_PI 3.14159265358979f
#endif
#endif
