// Pipe interface of the reference (pikoc/api/include/piko/pipe.h): PikoPipe and
// pikoConnect, which records in each stage object where its output port goes
// and where its input port comes from; the runtime reads the graph from them.
#ifndef PIKO_COMPAT_PIPE_H
#define PIKO_COMPAT_PIPE_H

#ifdef __PIKOC_HOST__
#include "stage.h"

template <class S1, class S2>
static void pikoConnect(S1& outStg, S2& inStg, const int outPortNum, const int inPortNum)
{
  outStg.outPort[outPortNum] = &inStg;
  inStg.inPort[inPortNum] = &outStg;
}

class PikoPipe {};
#endif

#endif
