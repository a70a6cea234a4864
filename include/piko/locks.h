// Lock helpers of the reference's stage interface (pikoc/api/include/piko/locks.h);
// device code only.
#ifndef PIKO_COMPAT_LOCKS_H
#define PIKO_COMPAT_LOCKS_H

#ifdef __PIKOC_DEVICE__
inline int myAtomicExch(int* v1, int v2) { return atomicExch(v1, v2); }
inline int myAny(int pred) { return __any_sync(__activemask(), pred); }
inline int myBallot(int pred) { return (int)__ballot_sync(__activemask(), pred); }
#endif

#endif
