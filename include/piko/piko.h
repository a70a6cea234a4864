// Umbrella header of the reference's stage interface (pikoc/api/include/piko/piko.h).
#ifndef PIKO_COMPAT_PIKO_H
#define PIKO_COMPAT_PIKO_H
#include "builtinTypes.h"
#endif
