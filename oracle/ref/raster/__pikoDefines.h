// Test infrastructure (oracle only): the defines block that `pikoc --target=CPU`
// writes for RasterPipe (pikoc/src/Backend/CPUBackend.cpp:11-36), written by hand
// because pikoc itself cannot be built here.
#define __PIKOC_CPU__

#ifndef __PIKOC_DEVICE__
  #define __PIKOC_DEVICE__
#endif

#define __PIKO_DEVICE_MEMBERS__ \
  StageFloor* d_pikoScreen; \
  MutableState *d_mutableState; \
  PikoArray<raster_wtri> *d_input; \
  VertexShaderStage *d_vertexShader; \
  RasterStage *d_raster; \
  ;
