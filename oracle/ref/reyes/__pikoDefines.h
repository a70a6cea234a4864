// Test infrastructure (oracle only): the defines block that `pikoc --target=CPU`
// writes for ReyesPipe (pikoc/src/Backend/CPUBackend.cpp:11-36), written by hand
// because pikoc itself cannot be built here.
#define __PIKOC_CPU__

#ifndef __PIKOC_DEVICE__
  #define __PIKOC_DEVICE__
#endif

#define __PIKO_DEVICE_MEMBERS__ \
  StageFloor* d_pikoScreen; \
  MutableState *d_mutableState; \
  PikoArray<piko_patch> *d_input; \
  SplitStage *d_split; \
  DiceStage *d_dice; \
  ShadeStage *d_shade; \
  ;
