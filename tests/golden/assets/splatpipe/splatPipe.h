#ifndef SPLAT_PIPE_H_
#define SPLAT_PIPE_H_

#include "piko/pipe.h"
#include "splatTypes.h"
#include "splat.pikostage"

#ifdef __PIKOC_HOST__

class SplatPipe : public PikoPipe
{
  SplatStage splat;
public:
  ConstantState*      constState_;
  MutableState*       mutableState_;
  int         count_;
  PikoScreen  pikoScreen;
  PikoArray<splat_point> h_input;

#ifdef __PIKO_DEVICE_MEMBERS__
  __PIKO_DEVICE_MEMBERS__
#endif

  SplatPipe() {}

  void run        (ConstantState& constState, MutableState& mutableState, splat_point* input, int count);
  void allocate   (ConstantState& constState, MutableState& mutableState, splat_point* input, int count);
  void prepare    ();
  void run_single ();
  void destroy    ();
};

#endif // __PIKOC_HOST__

#endif // SPLAT_PIPE_H_
