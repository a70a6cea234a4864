// Built-in types of the reference's stage interface (pikoc/api/include/piko/builtinTypes.h):
// ConstantState, MutableState, Primitive (every queued type derives from it)
// and Pixel, the screen's input.
#ifndef PIKO_COMPAT_BUILTIN_TYPES_H
#define PIKO_COMPAT_BUILTIN_TYPES_H

typedef int binID;

#include "cvec.h"

struct cvec2u {
  unsigned int x, y;
};

struct ConstantState {
  int screenSizeX;
  int screenSizeY;
  float halfW, halfH;
  float projMatrix[16];
  float viewMatrix[16];
  float viewProjMatrix[16];
  int debX, debY;
};

// The reference's MutableState is a fixed 1024x768 depth array; here zBuffer
// points at screenSizeX * screenSizeY floats: host memory in the caller's
// state (copied to the device by prepare()), device memory in stage code.
struct MutableState {
  float* zBuffer;
};

struct Primitive {
  unsigned binID;
  unsigned launchIdx;
};

struct Pixel : public Primitive {
  cvec2u pos;        // (0, 0) is the bottom-left pixel
  unsigned int color;  // RGBA8, R in the low byte
  void setColor(float r, float g, float b, float a)
  {
    color = ((unsigned)(a * 255.0f) << 24) | ((unsigned)(b * 255.0f) << 16) | ((unsigned)(g * 255.0f) << 8) |
            (unsigned)(r * 255.0f);
  }
};

struct boundingBox {
  cvec2f hi, lo;
};

#endif
