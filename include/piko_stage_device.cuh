/*
 * piko_stage_device.cuh - the device half of Piko's stage API (see
 * piko_stage.cuh for the pipeline runtime): the Stage base class, the
 * sequential keys, and the AssignBin / Process kernel bodies.  It compiles
 * with nvcc and with NVRTC (no host headers), so that stage code written
 * against the reference's interface can be compiled at run time
 * (piko-public_b200/pikoc.py with include/piko/).  In that mode
 * (PIKO_COMPAT_API defined) ConstantState, MutableState and Pixel are the
 * reference-named global types of include/piko/builtinTypes.h, aliased into
 * namespace piko before this header is included.
 */
#pragma once

namespace piko {

enum SchedulePolicy { LOAD_BALANCE, ROUND_ROBIN, SERIAL, ALL };
enum AssignPolicy { PREVIOUS_BINS, BOUNDING_BOX, POSITION };

constexpr int kNumPorts = 5;          // ports per stage (stage.h:19)
constexpr int kScreen = -1;           // connect(..., kScreen): the PikoScreen drain
constexpr int kMaxLoopRounds = 64;    // rounds of a self-looping stage per frame

#ifndef PIKO_COMPAT_API
// ConstantState (piko/builtinTypes.h:20-33): the same fields, read by stages as
// the member `constState` (the reference's generated code keeps it in a
// global of that name; here each stage object carries a copy per launch).
struct ConstantState {
  int screenSizeX, screenSizeY;
  float halfW, halfH;
  float projMatrix[16];
  float viewMatrix[16];
  float viewProjMatrix[16];
};

// The reference's MutableState holds a fixed 1024x768 depth array; here it
// points at a device depth buffer of screenSizeX * screenSizeY floats.
struct MutableState {
  float* zBuffer;
};

struct int2p { int x, y; };
struct Pixel {
  int2p pos;       // pos (0, 0) is the bottom-left pixel
  unsigned color;  // RGBA8, R in the low byte
};

// ------------------------------------------------------------------ helpers
// The small vector types of the reference's piko/cvec.h and the helpers of its
// piko/math.h that stage code calls, with the semantics of the reference's CPU
// backend (pikoc/api/include/piko/math.h:258-330), so that stage code ported
// from .pikostage files computes what the reference's CPU run computes:
// rcp_approx is an IEEE division (not the GPU's approximate reciprocal), imad
// wraps (not the GPU's saturating vmad), toABGR truncates without saturation,
// fromABGR divides by 255.

struct cvec2i { int x, y; };
struct cvec2f { float x, y; };
struct cvec3f { float x, y, z; };
struct cvec4f { float x, y, z, w; };

__host__ __device__ inline cvec2i gencvec2i(int x, int y) { return cvec2i{x, y}; }
__host__ __device__ inline cvec2f gencvec2f(float x, float y) { return cvec2f{x, y}; }
__host__ __device__ inline cvec3f gencvec3f(float x, float y, float z) { return cvec3f{x, y, z}; }
__host__ __device__ inline cvec4f gencvec4f(float x, float y, float z, float w) { return cvec4f{x, y, z, w}; }
__host__ __device__ inline cvec3f operator+(cvec3f a, cvec3f b) { return cvec3f{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline cvec3f operator-(cvec3f a, cvec3f b) { return cvec3f{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline cvec3f operator*(cvec3f a, float s) { return cvec3f{a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline cvec2i operator+(cvec2i a, cvec2i b) { return cvec2i{a.x + b.x, a.y + b.y}; }
__host__ __device__ inline cvec2i operator-(cvec2i a, cvec2i b) { return cvec2i{a.x - b.x, a.y - b.y}; }

__host__ __device__ inline int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ inline int imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ inline int max_max(int a, int b, int c) { return imax(imax(a, b), c); }
__host__ __device__ inline int min_min(int a, int b, int c) { return imin(imin(a, b), c); }
__host__ __device__ inline int max_add(int a, int b, int c) { return (int)((unsigned)imax(a, b) + (unsigned)c); }
__host__ __device__ inline int min_add(int a, int b, int c) { return (int)((unsigned)imin(a, b) + (unsigned)c); }
__host__ __device__ inline int shl_add(int a, unsigned b, int c) { return (int)(((unsigned)a << b) + (unsigned)c); }
__host__ __device__ inline int shr_add(int a, unsigned b, int c) { return (int)((unsigned)(a >> b) + (unsigned)c); }
__host__ __device__ inline unsigned add_add(unsigned a, unsigned b, unsigned c) { return a + b + c; }
__host__ __device__ inline unsigned sub_add(unsigned a, unsigned b, unsigned c) { return a - b + c; }
__host__ __device__ inline unsigned add_sub(unsigned a, unsigned b, unsigned c) { return a + b - c; }
// a * b + c in wrapping 32-bit arithmetic (the CPU backend's int expression)
__host__ __device__ inline int imad(int a, int b, int c) { return (int)((unsigned)a * (unsigned)b + (unsigned)c); }
__host__ __device__ inline float rcp_approx(float a) { return 1.0f / a; }
__host__ __device__ inline unsigned idiv_fast(unsigned a, unsigned b) { return a / b; }
// a * b + c with two roundings (the CPU backend does not fuse)
__host__ __device__ inline float fma_rm(float a, float b, float c)
{
#ifdef __CUDA_ARCH__
  return __fadd_rn(__fmul_rn(a, b), c);
#else
  return a * b + c;
#endif
}
__host__ __device__ inline int popcll(unsigned long long x)
{
#ifdef __CUDA_ARCH__
  return __popcll(x);
#else
  return __builtin_popcountll(x);
#endif
}
__host__ __device__ inline int ffsll(unsigned long long x)
{
#ifdef __CUDA_ARCH__
  return __ffsll((long long)x);
#else
  return __builtin_ffsll((long long)x);
#endif
}
// (unsigned)(c * 255.0f) per channel, alpha 255, no saturation (the CPU
// backend's conversion keeps the low 32 bits of a 64-bit truncation)
__host__ __device__ inline unsigned abgr_channel(float v)
{
#ifdef __CUDA_ARCH__
  if (fabsf(v) < 2147483648.0f) return (unsigned)__float2int_rz(v);
  return (v > -9223372036854775808.0f && v < 9223372036854775808.0f) ? (unsigned)__float2ll_rz(v) : 0u;
#else
  return (unsigned)(long long)v;
#endif
}
__host__ __device__ inline unsigned toABGR(cvec3f c)
{
  return 0xff000000u | (abgr_channel(c.z * 255.0f) << 16) | (abgr_channel(c.y * 255.0f) << 8) | abgr_channel(c.x * 255.0f);
}
__host__ __device__ inline cvec3f fromABGR(unsigned c)
{
  return cvec3f{(float)(c & 255u) / 255.0f, (float)((c >> 8) & 255u) / 255.0f, (float)((c >> 16) & 255u) / 255.0f};
}
// column-major 4x4 matrix times (v, 1), left-to-right sums (piko/math.h:365-383)
__host__ __device__ inline cvec4f matmultfloat4(const float* m, cvec3f v)
{
  return cvec4f{m[0] * v.x + m[4] * v.y + m[8] * v.z + m[12], m[1] * v.x + m[5] * v.y + m[9] * v.z + m[13],
                m[2] * v.x + m[6] * v.y + m[10] * v.z + m[14], m[3] * v.x + m[7] * v.y + m[11] * v.z + m[15]};
}

#endif  // PIKO_COMPAT_API

namespace detail {

enum : unsigned { kStatusQueueOverflow = 1u, kStatusListOverflow = 2u, kStatusEmitOverflow = 4u };

// Sequential keys: (position of the emitting primitive in its stage's
// one-thread processing order) << kSeqBits | (emits before this one in the
// same process call).  Screen keys add the stage index above kPosBits.
constexpr int kSeqBits = 20;
constexpr int kPosBits = 40;
constexpr unsigned long long kSeqMask = (1ull << kSeqBits) - 1;

// screen modes of a process launch
enum : int { kScreenDirect = 0, kScreenDepthOnly = 1, kScreenKeys = 2, kScreenColour = 3 };

// Device view of one stage for one launch.
struct StageRun {
  int numBinsX, numBinsY, binSizeX, binSizeY;
  unsigned* binCount;       // [bins] assignments per bin (count pass)
  unsigned* binStart;       // [bins] first entry of each bin in the sorted list
  unsigned long long* pairs;      // [listCap] (bin << 32 | input rank), write pass
  unsigned long long* binList;    // [listCap] pairs sorted: the bin lists in one-thread order
  unsigned listCap;
  unsigned* pairCount;      // write-pass cursor
  const unsigned* perm;     // input rank -> input queue index
  int policy, split;        // from specifySchedule
  int stage;                // index of the stage in the pipe
  unsigned long long keyBase;     // primitives the stage processed in earlier rounds of a self loop
  int pass;                 // 0: the stage's run; 1, 2: the screen resolve runs
  int screenMode;
  // emit routing, per port
  void* outData[kNumPorts];
  unsigned long long* outKeys[kNumPorts];
  unsigned* outCount[kNumPorts];
  unsigned outCap[kNumPorts];
  unsigned outSize[kNumPorts];  // bytes per primitive sent on the port
  int outKind[kNumPorts];   // 0 unconnected, 1 stage input queue, 2 screen
  unsigned* fb;
  unsigned long long* pixKey;   // [W * H] greatest sequential key + 1 per pixel
  int W, H;
  unsigned* status;
};

template <class A, class B> struct same_type { static constexpr bool value = false; };
template <class A> struct same_type<A, A> { static constexpr bool value = true; };
template <class T> T& lvalue_of();
template <class T, class = void> struct has_bin_id { static constexpr bool value = false; };
template <class T> struct has_bin_id<T, decltype((void)lvalue_of<T>().binID, void())> {
  static constexpr bool value = true;
};

}  // namespace detail

// The data every stage object carries, first in its layout so that the
// runtime can set it in a stage object it only knows as bytes.
struct StageCommon {
  ConstantState constState;            // the frame's constants (set per launch)
  MutableState* mutableState = nullptr;
  detail::StageRun* run_ = nullptr;
  int binID_ = 0;
  unsigned rank_ = 0;                  // input rank being assigned
  unsigned long long procKey_ = 0;     // sequential position of the primitive being processed
  unsigned emitSeq_ = 0;               // emits of this process call so far
  // pikoConnect's links (host side, the reference's outPort / inPort)
  void* outPort[kNumPorts] = {};
  void* inPort[kNumPorts] = {};
};

template <int BinSizeX, int BinSizeY, int ThreadsPerTile, class InPrim, class OutPrim>
class Stage : public StageCommon {
 public:
  using In = InPrim;
  using Out = OutPrim;
  static constexpr int kBinSizeX = BinSizeX, kBinSizeY = BinSizeY, kThreadsPerTile = ThreadsPerTile;

  __device__ int getNumBins() const { return run_->numBinsX * run_->numBinsY; }
  __device__ int getNumBinsX() const { return run_->numBinsX; }
  __device__ int getNumBinsY() const { return run_->numBinsY; }
  __device__ int getBinSizeX() const { return run_->binSizeX; }
  __device__ int getBinSizeY() const { return run_->binSizeY; }
  __device__ int getBinID() const { return binID_; }
  // 0 in the stage's run; 1 and 2 in the screen resolve runs of a stage that
  // feeds the screen (side effects other than emits and depth updates belong
  // in pass 0)
  __device__ int passIndex() const { return run_->pass; }

 protected:
  __device__ void assignToBin(const In&, int binID)
  {
    detail::StageRun& r = *run_;
    if (binID < 0 || binID >= r.numBinsX * r.numBinsY) return;
    if (r.pairs == nullptr) {
      atomicAdd(&r.binCount[binID], 1u);
    } else {
      const unsigned slot = atomicAdd(r.pairCount, 1u);
      if (slot < r.listCap) r.pairs[slot] = ((unsigned long long)(unsigned)binID << 32) | rank_;
      else atomicOr(r.status, (unsigned)detail::kStatusListOverflow);
    }
  }
  // PREVIOUS_BINS: the bin of the stage run that emitted p (its CTA's bin)
  __device__ void assignToBin(const In& p, AssignPolicy pol)
  {
    if (pol == PREVIOUS_BINS) assignToBin(p, (int)p.binID);
  }

  __device__ void specifySchedule(SchedulePolicy pol, int tileSplitSize = 0)
  {
    run_->policy = (int)pol;
    run_->split = tileSplitSize;
  }

  __device__ void emit(const Out& p, int port) { emit_impl(p, port); }

 public:
  // emit's body; a stage class that declares its own emit (as the reference's
  // stage files do, for pikoc to define) gets a definition calling this
  __device__ void emit_impl(const Out& p, int port)
  {
    detail::StageRun& r = *run_;
    if (port < 0 || port >= kNumPorts) return;
    const unsigned seq = emitSeq_++;
    if (seq > detail::kSeqMask) atomicOr(r.status, (unsigned)detail::kStatusEmitOverflow);
    const unsigned long long key = procKey_ | seq;
    if (r.outKind[port] == 2) {
      if constexpr (detail::same_type<Out, Pixel>::value) {
        const long long x = (long long)p.pos.x, y = (long long)p.pos.y;
        if (x < 0 || x >= r.W || y < 0 || y >= r.H) return;
        const unsigned long long i = (unsigned long long)y * (unsigned long long)r.W + (unsigned long long)x;
        const unsigned long long skey = ((unsigned long long)r.stage << (detail::kPosBits + detail::kSeqBits)) | key;
        if (r.screenMode == detail::kScreenDirect) r.fb[i] = p.color;
        else if (r.screenMode == detail::kScreenKeys) atomicMax(&r.pixKey[i], skey + 1);
        else if (r.screenMode == detail::kScreenColour && r.pixKey[i] == skey + 1) r.fb[i] = p.color;
      }
    } else if (r.outKind[port] == 1 && r.pass == 0) {
      const unsigned slot = atomicAdd(r.outCount[port], 1u);
      if (slot < r.outCap[port]) {
        Out q = p;
        if constexpr (detail::has_bin_id<Out>::value) q.binID = binID_;
        static_cast<Out*>(r.outData[port])[slot] = q;
        r.outKeys[port][slot] = key;
      } else {
        atomicOr(r.status, (unsigned)detail::kStatusQueueOverflow);
      }
    }
  }
};

namespace detail {

// AssignBin over the input in rank order: pass 0 counts per bin, pass 1
// records (bin, rank) pairs.
template <class S>
__device__ void assign_body(S& stage, StageRun* run, const typename S::In* in, unsigned n, int pass)
{
  __shared__ StageRun s_run;
  if (threadIdx.x == 0) {
    s_run = *run;
    if (pass == 0) s_run.pairs = nullptr;
  }
  __syncthreads();
  stage.run_ = &s_run;
  for (unsigned r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    stage.rank_ = r;
    stage.assignBin(in[s_run.perm[r]]);
  }
}

// Process: a bin's entries are its range of the sorted list; entry j (the
// j-th primitive of the round in one-thread order) is processed with
// sequential key (keyBase + j) << kSeqBits, keyBase counting the primitives
// of the stage's earlier rounds (a self loop's rounds run in order).
template <class S>
__device__ void process_body(S& stage, StageRun* run, const typename S::In* in, unsigned* workNext, MutableState* ms,
                             int pass, int screenMode)
{
  __shared__ StageRun s_run;
  __shared__ int s_bin;
  __shared__ unsigned s_lo, s_hi;
  if (threadIdx.x == 0) {
    s_run = *run;
    s_run.pass = pass;
    s_run.screenMode = screenMode;
  }
  __syncthreads();
  stage.run_ = &s_run;
  stage.mutableState = ms;
  // the schedule of this stage, named by its schedule() (the same for every bin)
  if (threadIdx.x == 0) stage.schedule(0);
  __syncthreads();
  const int policy = s_run.policy;
  const int bins = s_run.numBinsX * s_run.numBinsY;
  const int split = s_run.policy == ALL ? (s_run.split > 0 ? s_run.split : 1) : 1;
  const unsigned items = (unsigned)bins * (unsigned)split;
  if (policy == SERIAL && blockIdx.x != 0) return;
  unsigned rr = blockIdx.x;
  for (;;) {
    if (threadIdx.x == 0) {
      unsigned it;
      if (policy == LOAD_BALANCE || policy == ALL) it = atomicAdd(workNext, 1u);
      else if (policy == SERIAL) it = rr, rr += 1;
      else it = rr, rr += gridDim.x;   // ROUND_ROBIN
      if (it >= items) {
        s_bin = -1;
      } else {
        const int b = (int)(it / (unsigned)split), part = (int)(it % (unsigned)split);
        const unsigned lo = s_run.binStart[b], hi = lo + s_run.binCount[b];
        const unsigned cnt = hi - lo, per = (cnt + (unsigned)split - 1) / (unsigned)split;
        s_bin = b;
        s_lo = min(hi, lo + per * (unsigned)part);
        s_hi = min(hi, s_lo + per);
      }
    }
    __syncthreads();
    const int b = s_bin;
    if (b < 0) break;
    stage.binID_ = b;
    for (unsigned j = s_lo + threadIdx.x; j < s_hi && j < s_run.listCap; j += blockDim.x) {
      const unsigned rank = (unsigned)s_run.binList[j];
      stage.procKey_ = (s_run.keyBase + j) << kSeqBits;
      stage.emitSeq_ = 0;
      stage.process(in[s_run.perm[rank]]);
    }
    __syncthreads();
  }
}

// The kernels of a stage type (the nvcc path instantiates these; the NVRTC
// path wraps the bodies in extern "C" kernels of fixed names).
template <class S>
__global__ void assign_kernel(S stage, StageRun* run, const typename S::In* in, unsigned n, int pass)
{
  assign_body(stage, run, in, n, pass);
}
template <class S>
__global__ void process_kernel(S stage, StageRun* run, const typename S::In* in, unsigned* workNext, MutableState* ms,
                               int pass, int screenMode)
{
  process_body(stage, run, in, workNext, ms, pass, screenMode);
}

}  // namespace detail
}  // namespace piko
