// Stage interface of the reference (pikoc/api/include/piko/stage.h): the
// Stage<binSizeX, binSizeY, threadsPerTile, In, Out> base class, the
// schedule and assignment policies, and the host-side PikoScreen / PikoArray a
// pipe class holds.  The Stage base is piko::Stage of piko_stage_device.cuh
// (sequential keys, bin lists, emit routing); this header names it and the
// reference's types the way stage files spell them.
#ifndef PIKO_COMPAT_STAGE_H
#define PIKO_COMPAT_STAGE_H

#include "builtinTypes.h"
#include "deviceFunctions.h"

#ifndef PIKO_COMPAT_API
#define PIKO_COMPAT_API
#endif
namespace piko {
typedef ::ConstantState ConstantState;
typedef ::MutableState MutableState;
typedef ::Pixel Pixel;
}  // namespace piko
#include "../piko_stage_device.cuh"

#define NUM_PORTS 5

using piko::SchedulePolicy;
using piko::LOAD_BALANCE;
using piko::ROUND_ROBIN;
using piko::SERIAL;
using piko::ALL;
using piko::AssignPolicy;
using piko::PREVIOUS_BINS;
using piko::BOUNDING_BOX;
using piko::POSITION;

template <int binSizeX, int binSizeY, int threadsPerTile, class InPrimType, class OutPrimType>
using Stage = piko::Stage<binSizeX, binSizeY, threadsPerTile, InPrimType, OutPrimType>;

#ifdef __PIKOC_HOST__
#include <cstdlib>
#include <cstring>
#include <vector>

namespace piko {
class PipeCore;
}

// The screen of a pipe: getData() returns W * H RGBA8 words owned by the
// pipe (stage.h:108-117), copied from the device when called.
class PikoScreen {
 public:
  piko::PipeCore* core_ = nullptr;
  std::vector<unsigned> h_data_;
  unsigned* getData();
};

// The pipe's copy of its input (CPUBackend.cpp:331-332).
template <class T>
class PikoArray {
 public:
  std::vector<T> data_;
  void allocate(int n) { data_.resize(n > 0 ? (size_t)n : 1u); }
  void copyFrom(const T* src, int n)
  {
    allocate(n);
    if (n > 0) std::memcpy((void*)data_.data(), (const void*)src, sizeof(T) * (size_t)n);
  }
  T* getData() { return data_.data(); }
};
#endif  // __PIKOC_HOST__

#endif
