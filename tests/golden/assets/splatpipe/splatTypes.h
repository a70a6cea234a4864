// A test pipeline written the way the reference's sample pipelines are (a
// PikoPipe class header plus .pikostage files), for pikoc.py: points are binned
// by position and each stamps a 2x2 block of pixels with its colour.  Later
// points in input order overwrite earlier ones where blocks overlap, as in the
// reference's one-thread run.
#ifndef SPLAT_TYPES_H
#define SPLAT_TYPES_H

#include "piko/piko.h"
#include "piko/builtinTypes.h"

struct splat_point : public Primitive {
  int id;
  float x, y;          // pixel coordinates
  unsigned color;      // RGBA8
};

#endif
