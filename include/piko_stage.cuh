/*
 * piko_stage.cuh - Piko's stage API for user pipelines on B200 (sm_100a),
 * header-only CUDA C++.
 *
 * The reference's boundary is source level: a pipeline is a set of classes
 * derived from Stage<binSizeX, binSizeY, threadsPerTile, In, Out> that
 * implement assignBin / schedule / process and call assignToBin,
 * specifySchedule and emit (pikoc/api/include/piko/stage.h:138-391,
 * pikoc/api/include/piko/deviceFunctions.h:22-50), wired by pikoConnect
 * (pikoc/api/include/piko/pipe.h:8-12), and pikoc compiles them into per-stage
 * kernels (pikoc/src/pikoc.cpp:196-318).  Here the same classes compile with
 * nvcc against this header, and piko::Pipe runs them:
 *
 *   for each stage, in the order given (stages only feed later stages, or
 *   themselves through a self loop):
 *     order       every queued primitive carries the position it would have
 *                 in the reference's one-thread run (below); the stage's input
 *                 is ranked by it (a radix sort);
 *     AssignBin   one thread per input primitive calls assignBin(p); its
 *                 assignToBin calls fill per-bin counts, an exclusive scan gives
 *                 each bin its range, and a second pass records (bin, rank)
 *                 pairs that a radix sort turns into the bin lists, each in
 *                 rank order -- the order the one-thread run appends them;
 *     Schedule    schedule(binID) names the policy (LOAD_BALANCE: CTAs take bins
 *                 from a queue; ROUND_ROBIN: CTA c takes bins c, c + CTAs, ...;
 *                 SERIAL: one CTA takes every bin in order; ALL: the
 *                 primitives of each bin are split over tileSplitSize CTAs);
 *     Process     a persistent launch of threadsPerTile-thread CTAs; for each
 *                 bin, thread t processes primitives t, t + threadsPerTile, ...
 *                 (the reference's process loop, pikoc/src/pikoc.cpp:236-262);
 *                 emit(p, port) appends p to the input of the stage connected
 *                 to that port, or, for a port connected to the screen, draws
 *                 p.color at p.pos as PikoScreen::assignBin does (stage.h:57-61);
 *     a stage connected to itself runs again on what it emitted to itself until
 *     nothing is left (at most kMaxLoopRounds rounds), like the reference's
 *     Split loop (pikoc/src/pikoc.cpp:294-308).
 *
 * One-thread order.  The reference's CPU backend run with one thread
 * processes a stage's bins in index order and each bin's list in the order
 * assignToBin appended to it, and an emit appends at once (the next stage's
 * assignBin runs inside emit).  So the n-th primitive a stage processes has
 * sequential position n, and what it emits is ordered by (n, emit count of
 * that process call).  Each queued primitive carries that key; ranking a
 * stage's input by it and sorting each bin list by rank reproduces the
 * one-thread order exactly, whatever order the GPU threads ran in.
 *
 * The screen.  PikoScreen keeps the last Pixel written (stage.h:57-61), and a
 * stage typically emits a Pixel only after its depth test on
 * mutableState->zBuffer (an atomicMin loop, raster.pikostage:274-285) passes.
 * Run in one thread, that leaves the colour of the last fragment, in
 * sequential order, among those at the final depth of the pixel.  Threads
 * racing on the depth buffer emit a different set, so a stage that feeds the
 * screen (and does not loop) runs three times: a first run draws nothing to
 * the screen and leaves the final depths; in the second every emitted Pixel
 * (now exactly the fragments at the final depth, whose depth test still
 * passes) keeps the greatest sequential key per pixel; the third writes the
 * colour of the Pixel with that key.  The colour then equals the one-thread
 * reference's.  The second and third runs emit nothing to other stages; a
 * process with other side effects (counters, other buffers) must do them only
 * when passIndex() == 0.  A self-looping stage's screen emits are written as
 * they come (the last writer wins).
 *
 * Bin size 0 means one full-screen bin (pikoc/include/PikoSummary.hpp:279); the
 * bin grid is screenSize / binSize rounded down, as in the reference.
 * Queues and bin lists that outgrow their capacity are grown and the frame is
 * run again; device-side work never waits on another CTA.  The two reference
 * pipelines also run as hand-fused kernels behind the C ABI (piko_b200.h); this
 * header is the general path for other pipelines.  Sorting uses the CUDA
 * toolkit's CUB radix sort.
 */
#pragma once

#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

namespace piko {

enum SchedulePolicy { LOAD_BALANCE, ROUND_ROBIN, SERIAL, ALL };
enum AssignPolicy { PREVIOUS_BINS, BOUNDING_BOX, POSITION };

constexpr int kNumPorts = 5;          // ports per stage (stage.h:19)
constexpr int kScreen = -1;           // connect(..., kScreen): the PikoScreen drain
constexpr int kMaxLoopRounds = 64;    // rounds of a self-looping stage per frame

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
  int pass;                 // 0: the stage's run; 1, 2: the screen resolve runs
  int screenMode;
  // emit routing, per port
  void* outData[kNumPorts];
  unsigned long long* outKeys[kNumPorts];
  unsigned* outCount[kNumPorts];
  unsigned outCap[kNumPorts];
  int outKind[kNumPorts];   // 0 unconnected, 1 stage input queue, 2 screen
  unsigned* fb;
  unsigned long long* pixKey;   // [W * H] greatest sequential key + 1 per pixel
  int W, H;
  unsigned* status;
};

}  // namespace detail

template <int BinSizeX, int BinSizeY, int ThreadsPerTile, class InPrim, class OutPrim>
class Stage {
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

  // set by piko::Pipe before each launch
  ConstantState constState;
  MutableState* mutableState = nullptr;
  detail::StageRun* run_ = nullptr;
  int binID_ = 0;
  unsigned rank_ = 0;                  // input rank being assigned
  unsigned long long procKey_ = 0;     // sequential position of the primitive being processed
  unsigned emitSeq_ = 0;               // emits of this process call so far

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
    if (pol == PREVIOUS_BINS) assignToBin(p, p.binID);
  }

  __device__ void specifySchedule(SchedulePolicy pol, int tileSplitSize = 0)
  {
    run_->policy = (int)pol;
    run_->split = tileSplitSize;
  }

  __device__ void emit(const Out& p, int port)
  {
    detail::StageRun& r = *run_;
    if (port < 0 || port >= kNumPorts) return;
    const unsigned seq = emitSeq_++;
    if (seq > detail::kSeqMask) atomicOr(r.status, (unsigned)detail::kStatusEmitOverflow);
    const unsigned long long key = procKey_ | seq;
    if (r.outKind[port] == 2) {
      if constexpr (std::is_same<Out, Pixel>::value) {
        if (p.pos.x < 0 || p.pos.x >= r.W || p.pos.y < 0 || p.pos.y >= r.H) return;
        const size_t i = (size_t)p.pos.y * (size_t)r.W + (size_t)p.pos.x;
        const unsigned long long skey = ((unsigned long long)r.stage << (detail::kPosBits + detail::kSeqBits)) | key;
        if (r.screenMode == detail::kScreenDirect) r.fb[i] = p.color;
        else if (r.screenMode == detail::kScreenKeys) atomicMax(&r.pixKey[i], skey + 1);
        else if (r.screenMode == detail::kScreenColour && r.pixKey[i] == skey + 1) r.fb[i] = p.color;
      }
    } else if (r.outKind[port] == 1 && r.pass == 0) {
      const unsigned slot = atomicAdd(r.outCount[port], 1u);
      if (slot < r.outCap[port]) {
        Out q = p;
        if constexpr (has_bin_id<Out>::value) q.binID = binID_;
        static_cast<Out*>(r.outData[port])[slot] = q;
        r.outKeys[port][slot] = key;
      } else {
        atomicOr(r.status, (unsigned)detail::kStatusQueueOverflow);
      }
    }
  }

 private:
  template <class T, class = void> struct has_bin_id : std::false_type {};
  template <class T> struct has_bin_id<T, decltype((void)std::declval<T&>().binID, void())> : std::true_type {};
};

namespace detail {

#define PIKO_STAGE_CHECK(call)                                                         \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string("piko::Pipe: ") + cudaGetErrorString(e_)); \
  } while (0)

// AssignBin over the input in rank order: pass 0 counts per bin, pass 1
// records (bin, rank) pairs (run->pairs set).
template <class S>
__global__ void assign_kernel(S stage, StageRun* run, const typename S::In* in, unsigned n, int pass)
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

// exclusive scan of bin counts by one CTA (bins of one stage are few enough)
__global__ void scan_bins(StageRun* run)
{
  __shared__ unsigned s_sum[1024];
  __shared__ unsigned s_carry;
  const int bins = run->numBinsX * run->numBinsY;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int base = 0; base < bins; base += 1024) {
    const int i = base + (int)threadIdx.x;
    const unsigned v = i < bins ? run->binCount[i] : 0u;
    s_sum[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      const unsigned t = threadIdx.x >= (unsigned)o ? s_sum[threadIdx.x - o] : 0u;
      __syncthreads();
      s_sum[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < bins) run->binStart[i] = s_carry + s_sum[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) s_carry += s_sum[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0 && s_carry > run->listCap) atomicOr(run->status, (unsigned)kStatusListOverflow);
}

__global__ void iota_kernel(unsigned* out, unsigned n)
{
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = i;
}

// Process: a bin's entries are its range of the sorted list; entry j (the
// j-th primitive of the stage in one-thread order) is processed with
// sequential key j << kSeqBits.
template <class S>
__global__ void process_kernel(S stage, StageRun* run, const typename S::In* in, unsigned* workNext, MutableState* ms,
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
        const unsigned n = hi - lo, per = (n + (unsigned)split - 1) / (unsigned)split;
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
      stage.procKey_ = (unsigned long long)j << kSeqBits;
      stage.emitSeq_ = 0;
      stage.process(in[s_run.perm[rank]]);
    }
    __syncthreads();
  }
}

}  // namespace detail

// A pipeline of stages S0..Sn-1 (given in an order where every connection goes
// to a later stage or to the stage itself), drawn into a W x H screen.
template <class... S>
class Pipe {
 public:
  static constexpr int kStages = (int)sizeof...(S);
  using In0 = typename std::tuple_element<0, std::tuple<S...>>::type::In;

  Pipe() { for (auto& l : links_) for (int& t : l) t = -2; }
  ~Pipe() { destroy(); }
  Pipe(const Pipe&) = delete;
  Pipe& operator=(const Pipe&) = delete;

  std::tuple<S...> stages;   // user stage objects (copied into each launch)

  // pikoConnect(out, in, outPort, inPort): output port `port` of stage `from`
  // feeds stage `to` (kScreen: the screen).
  void connect(int from, int port, int to)
  {
    if (from < 0 || from >= kStages || port < 0 || port >= kNumPorts || to < kScreen || to >= kStages ||
        (to >= 0 && to < from))
      throw std::invalid_argument("piko::Pipe::connect: a port feeds a later stage, the stage itself or kScreen");
    links_[from][port] = to;
  }

  // allocate(): the caller's states (kept by pointer, re-read by prepare(),
  // as the generated allocate does) and a copy of the input primitives.
  void allocate(ConstantState& cs, MutableState& ms, const In0* input, int count)
  {
    cs_ = &cs;
    ms_ = &ms;
    W_ = cs.screenSizeX;
    H_ = cs.screenSizeY;
    if (W_ <= 0 || H_ <= 0 || count < 0) throw std::invalid_argument("piko::Pipe::allocate");
    if (!stream_) PIKO_STAGE_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    alloc_common();
    count_ = (unsigned)count;
    grow(q_[0], std::max<size_t>(count_, 1), sizeof(In0));
    // every later stage's input queue and every self loop's queue, sized up
    // front: a queue that earlier stages already wrote must not move during a
    // frame, so queues grow only between frames (after an overflow)
    const size_t initial = std::max<size_t>(4 * (size_t)std::max(count_, 1u), 1u << 16);
    for (int j = 1; j < kStages; ++j) grow_target(j, initial);
    for (int j = 0; j < kStages; ++j)
      if (links_has_self_loop(j)) grow_loop(j, initial);
    if (count) PIKO_STAGE_CHECK(cudaMemcpyAsync(q_[0].data, input, sizeof(In0) * count_, cudaMemcpyHostToDevice, stream_));
    PIKO_STAGE_CHECK(cudaStreamSynchronize(stream_));
  }

  void prepare()
  {
    cs_copy_ = *cs_;
    MutableState m = *ms_;
    PIKO_STAGE_CHECK(cudaMemcpyAsync(d_ms_, &m, sizeof(MutableState), cudaMemcpyHostToDevice, stream_));
    PIKO_STAGE_CHECK(cudaStreamSynchronize(stream_));
  }

  // One frame, synchronous; queues that overflow are grown and the frame runs
  // again (at most 8 times).
  void run_single()
  {
    for (int attempt = 0; attempt < 8; ++attempt)
      if (frame()) return;
    throw std::runtime_error("piko::Pipe::run_single: queues kept overflowing");
  }

  // PikoScreen::getData(): the screen, W*H RGBA8 words (device pointer), and a host copy.
  unsigned* screen() { return d_fb_; }
  void getData(unsigned* host) const
  {
    PIKO_STAGE_CHECK(cudaMemcpy(host, d_fb_, sizeof(unsigned) * (size_t)W_ * H_, cudaMemcpyDeviceToHost));
  }
  void clearScreen(unsigned color)
  {
    std::vector<unsigned> c((size_t)W_ * H_, color);
    PIKO_STAGE_CHECK(cudaMemcpy(d_fb_, c.data(), sizeof(unsigned) * c.size(), cudaMemcpyHostToDevice));
  }
  // primitives each stage processed in the last frame (all rounds)
  const std::vector<unsigned long long>& processed() const { return processed_; }
  int rounds(int stage) const { return rounds_[stage]; }

  void destroy()
  {
    for (int i = 0; i < kStages; ++i) {
      free_queue(q_[i]);
      free_queue(loop_[i]);
    }
    auto fr = [](void* p) { if (p) cudaFree(p); };
    fr(d_fb_); fr(d_ms_); fr(d_run_); fr(d_ctr_); fr(d_bins_); fr(d_pairs_); fr(d_list_); fr(d_perm_);
    fr(d_iota_); fr(d_ksort_); fr(d_tmp_); fr(d_pixkey_);
    d_fb_ = nullptr; d_ms_ = nullptr; d_run_ = nullptr; d_ctr_ = nullptr; d_bins_ = nullptr;
    d_pairs_ = nullptr; d_list_ = nullptr; d_perm_ = nullptr; d_iota_ = nullptr; d_ksort_ = nullptr;
    d_tmp_ = nullptr; d_pixkey_ = nullptr;
    bins_cap_ = list_cap_ = in_cap_ = tmp_bytes_ = 0;
    if (stream_) cudaStreamDestroy(stream_);
    stream_ = nullptr;
  }

 private:
  // A queue of primitives with their sequential keys.
  struct Queue { void* data = nullptr; unsigned long long* keys = nullptr; size_t cap = 0; };
  // counters: [0..kStages) queue counts, kStages + i: loop queue counts,
  // 2*kStages: pair cursor, +1 status, +2 work counter
  enum { kCtrPairs = 2 * sizeof...(S), kCtrStatus, kCtrWork, kCtrN };

  int links_[sizeof...(S)][kNumPorts];
  ConstantState* cs_ = nullptr;
  ConstantState cs_copy_{};
  MutableState* ms_ = nullptr;
  int W_ = 0, H_ = 0;
  unsigned count_ = 0;
  cudaStream_t stream_ = nullptr;
  Queue q_[sizeof...(S)], loop_[sizeof...(S)];
  unsigned* d_fb_ = nullptr;
  unsigned long long* d_pixkey_ = nullptr;
  MutableState* d_ms_ = nullptr;
  detail::StageRun* d_run_ = nullptr;
  unsigned* d_ctr_ = nullptr;
  unsigned* d_bins_ = nullptr;   // [2 * bins_cap_]: counts, starts
  unsigned long long* d_pairs_ = nullptr;  // [list_cap_] write-pass pairs
  unsigned long long* d_list_ = nullptr;   // [list_cap_] sorted pairs
  unsigned* d_perm_ = nullptr;   // [in_cap_] rank -> queue index
  unsigned* d_iota_ = nullptr;   // [in_cap_]
  unsigned long long* d_ksort_ = nullptr;  // [in_cap_] sorted input keys
  void* d_tmp_ = nullptr;        // radix-sort scratch
  size_t bins_cap_ = 0, list_cap_ = 0, in_cap_ = 0, tmp_bytes_ = 0;
  std::vector<unsigned long long> processed_ = std::vector<unsigned long long>(sizeof...(S), 0);
  int rounds_[sizeof...(S)] = {};

  static void free_queue(Queue& q)
  {
    if (q.data) cudaFree(q.data);
    if (q.keys) cudaFree(q.keys);
    q = Queue();
  }

  void grow(Queue& q, size_t n, size_t elem)
  {
    if (n <= q.cap) return;
    free_queue(q);
    PIKO_STAGE_CHECK(cudaMalloc(&q.data, n * elem));
    PIKO_STAGE_CHECK(cudaMalloc((void**)&q.keys, n * sizeof(unsigned long long)));
    q.cap = n;
  }

  // (re)allocates p for n elements (contents not kept)
  template <class T>
  static void grow_buf(T*& p, size_t& cap, size_t n)
  {
    if (n <= cap && p) return;
    if (p) cudaFree(p);
    p = nullptr;
    PIKO_STAGE_CHECK(cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T)));
    cap = n;
  }

  // the write pass's pairs and the sorted bin lists, n entries each
  void grow_lists(size_t n)
  {
    size_t c = 0;
    grow_buf(d_pairs_, c, n);
    c = 0;
    grow_buf(d_list_, c, n);
    list_cap_ = n;
  }

  void alloc_common()
  {
    if (!d_fb_) PIKO_STAGE_CHECK(cudaMalloc((void**)&d_fb_, sizeof(unsigned) * (size_t)W_ * H_));
    if (!d_pixkey_) PIKO_STAGE_CHECK(cudaMalloc((void**)&d_pixkey_, sizeof(unsigned long long) * (size_t)W_ * H_));
    if (!d_ms_) PIKO_STAGE_CHECK(cudaMalloc((void**)&d_ms_, sizeof(MutableState)));
    if (!d_run_) PIKO_STAGE_CHECK(cudaMalloc((void**)&d_run_, sizeof(detail::StageRun)));
    if (!d_ctr_) PIKO_STAGE_CHECK(cudaMalloc((void**)&d_ctr_, sizeof(unsigned) * kCtrN));
    clearScreen(0xff663313u);   // PikoScreen's initial colour (stage.h:83-85)
  }

  // radix-sort scratch for sorting n keys (the larger of the two sorts' needs)
  void ensure_tmp(size_t n)
  {
    size_t a = 0, b = 0;
    PIKO_STAGE_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, a, (unsigned long long*)nullptr,
                                                     (unsigned long long*)nullptr, (unsigned*)nullptr,
                                                     (unsigned*)nullptr, (int)n, 0, 64, stream_));
    PIKO_STAGE_CHECK(cub::DeviceRadixSort::SortKeys(nullptr, b, (unsigned long long*)nullptr,
                                                    (unsigned long long*)nullptr, (int)n, 0, 64, stream_));
    const size_t need = std::max(a, b);
    if (need > tmp_bytes_ || !d_tmp_) {
      if (d_tmp_) cudaFree(d_tmp_);
      d_tmp_ = nullptr;
      PIKO_STAGE_CHECK(cudaMalloc(&d_tmp_, std::max<size_t>(need, 256)));
      tmp_bytes_ = std::max<size_t>(need, 256);
    }
  }

  // screenSize / binSize, rounded down, as the reference sizes its bin grid
  // (stage.h:273-274): pixels past the last whole bin get no bin (at least one
  // bin per axis here, so that a screen smaller than a bin still has one)
  static int bins_of(int size, int extent) { return size <= 0 ? 1 : std::max(1, extent / size); }

  static int bits_for(unsigned long long v)
  {
    int b = 0;
    while (b < 64 && (v >> b) != 0) ++b;
    return std::max(b, 1);
  }

  template <int I>
  using StageT = typename std::tuple_element<I, std::tuple<S...>>::type;

  // Runs every stage once over its input (a self-looping stage: until its
  // own queue drains).  Returns false after an overflow (capacities grown).
  bool frame()
  {
    PIKO_STAGE_CHECK(cudaMemsetAsync(d_ctr_, 0, sizeof(unsigned) * kCtrN, stream_));
    PIKO_STAGE_CHECK(cudaMemsetAsync(d_pixkey_, 0, sizeof(unsigned long long) * (size_t)W_ * H_, stream_));
    unsigned c0 = count_;
    PIKO_STAGE_CHECK(cudaMemcpyAsync(d_ctr_ + 0, &c0, sizeof(unsigned), cudaMemcpyHostToDevice, stream_));
    for (auto& p : processed_) p = 0;
    bool ok = true;
    run_stages(ok, std::integral_constant<int, 0>());
    return ok;
  }

  void run_stages(bool&, std::integral_constant<int, sizeof...(S)>) {}
  template <int I>
  void run_stages(bool& ok, std::integral_constant<int, I>)
  {
    if (ok) ok = run_stage<I>();
    run_stages(ok, std::integral_constant<int, I + 1>());
  }

  // Where each port of stage I sends its primitives.  A connected stage's
  // input type must be stage I's output type.
  template <int I>
  bool route(detail::StageRun& r)
  {
    bool screen = false;
    for (int p = 0; p < kNumPorts; ++p) {
      const int to = links_[I][p];
      r.outKind[p] = 0;
      r.outData[p] = nullptr;
      r.outKeys[p] = nullptr;
      r.outCount[p] = nullptr;
      r.outCap[p] = 0;
      if (to == kScreen) {
        r.outKind[p] = 2;
        screen = true;
      } else if (to == I) {
        r.outKind[p] = 1;
        r.outData[p] = loop_[I].data;
        r.outKeys[p] = loop_[I].keys;
        r.outCount[p] = d_ctr_ + kStages + I;
        r.outCap[p] = (unsigned)loop_[I].cap;
      } else if (to > I) {
        r.outKind[p] = 1;
        r.outData[p] = q_[to].data;
        r.outKeys[p] = q_[to].keys;
        r.outCount[p] = d_ctr_ + to;
        r.outCap[p] = (unsigned)q_[to].cap;
      }
    }
    return screen;
  }

  template <int I>
  bool run_stage()
  {
    using St = StageT<I>;
    using In = typename St::In;
    St& stage = std::get<I>(stages);
    const int bx = bins_of(St::kBinSizeX, W_), by = bins_of(St::kBinSizeY, H_);
    const size_t bins = (size_t)bx * by;
    if (bins > bins_cap_) {
      if (d_bins_) cudaFree(d_bins_);
      d_bins_ = nullptr;
      PIKO_STAGE_CHECK(cudaMalloc((void**)&d_bins_, sizeof(unsigned) * 2 * bins));
      bins_cap_ = bins;
    }
    unsigned in_count = 0;
    PIKO_STAGE_CHECK(cudaMemcpyAsync(&in_count, d_ctr_ + I, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
    PIKO_STAGE_CHECK(cudaStreamSynchronize(stream_));
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, detail::process_kernel<St>, St::kThreadsPerTile, 0);
    const int ctas = sms * std::max(per_sm, 1);
    const bool loops = links_has_self_loop(I);
    rounds_[I] = 0;
    for (int round = 0; round < kMaxLoopRounds; ++round) {
      if (in_count == 0) break;
      ++rounds_[I];
      processed_[I] += in_count;
      // rank the input by sequential key (the host input is in order already)
      if (in_count > in_cap_ || !d_perm_) {
        size_t c0 = 0, c1 = 0, c2 = 0;
        const size_t n = (size_t)in_count + in_count / 2 + 1024;
        grow_buf(d_perm_, c0, n);
        grow_buf(d_iota_, c1, n);
        grow_buf(d_ksort_, c2, n);
        in_cap_ = n;
      }
      const unsigned iblocks = std::min<unsigned>((in_count + 255) / 256, (unsigned)sms * 8u);
      if (I == 0 && round == 0) {
        detail::iota_kernel<<<iblocks, 256, 0, stream_>>>(d_perm_, in_count);
      } else {
        detail::iota_kernel<<<iblocks, 256, 0, stream_>>>(d_iota_, in_count);
        ensure_tmp(in_count);
        size_t tb = tmp_bytes_;
        PIKO_STAGE_CHECK(cub::DeviceRadixSort::SortPairs(d_tmp_, tb, q_[I].keys, d_ksort_, d_iota_, d_perm_,
                                                         (int)in_count, 0, 64, stream_));
      }
      const size_t want = std::max<size_t>(4 * (size_t)in_count, 1u << 16);
      if (list_cap_ < want) grow_lists(want);
      detail::StageRun r;
      memset(&r, 0, sizeof(r));
      r.numBinsX = bx; r.numBinsY = by;
      r.binSizeX = St::kBinSizeX > 0 ? St::kBinSizeX : W_;
      r.binSizeY = St::kBinSizeY > 0 ? St::kBinSizeY : H_;
      r.binCount = d_bins_;
      r.binStart = d_bins_ + bins;
      r.pairs = d_pairs_;
      r.binList = d_list_;
      r.listCap = (unsigned)list_cap_;
      r.pairCount = d_ctr_ + kCtrPairs;
      r.perm = d_perm_;
      r.stage = I;
      r.fb = d_fb_;
      r.pixKey = d_pixkey_;
      r.W = W_; r.H = H_;
      r.status = d_ctr_ + kCtrStatus;
      const bool screen = route<I>(r);
      PIKO_STAGE_CHECK(cudaMemcpyAsync(d_run_, &r, sizeof(r), cudaMemcpyHostToDevice, stream_));
      PIKO_STAGE_CHECK(cudaMemsetAsync(d_bins_, 0, sizeof(unsigned) * bins, stream_));
      PIKO_STAGE_CHECK(cudaMemsetAsync(d_ctr_ + kCtrPairs, 0, sizeof(unsigned), stream_));
      const In* in = static_cast<const In*>(q_[I].data);
      stage.constState = cs_copy_;
      detail::assign_kernel<St><<<iblocks, 256, 0, stream_>>>(stage, d_run_, in, in_count, 0);
      detail::scan_bins<<<1, 1024, 0, stream_>>>(d_run_);
      detail::assign_kernel<St><<<iblocks, 256, 0, stream_>>>(stage, d_run_, in, in_count, 1);
      unsigned st[2] = {0, 0};
      PIKO_STAGE_CHECK(cudaMemcpyAsync(&st[0], d_ctr_ + kCtrStatus, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
      PIKO_STAGE_CHECK(cudaMemcpyAsync(&st[1], d_ctr_ + kCtrPairs, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
      PIKO_STAGE_CHECK(cudaStreamSynchronize(stream_));
      if (st[0] & detail::kStatusListOverflow) {
        grow_lists((size_t)st[1] + st[1] / 4 + 1024);
        return false;
      }
      // the bin lists: (bin, rank) pairs sorted, bin-major and rank-minor
      const unsigned total = st[1];
      if (total) {
        ensure_tmp(total);
        size_t tb = tmp_bytes_;
        PIKO_STAGE_CHECK(cub::DeviceRadixSort::SortKeys(d_tmp_, tb, d_pairs_, d_list_, (int)total, 0,
                                                        32 + bits_for(bins), stream_));
      }
      // the exact screen resolve (three runs) for a non-looping stage that
      // feeds the screen; otherwise one run with direct screen writes
      const bool exact = screen && !loops;
      const int runs = exact ? 3 : 1;
      for (int pass = 0; pass < runs; ++pass) {
        const int mode = !exact ? detail::kScreenDirect
                                : (pass == 0 ? detail::kScreenDepthOnly
                                             : (pass == 1 ? detail::kScreenKeys : detail::kScreenColour));
        PIKO_STAGE_CHECK(cudaMemsetAsync(d_ctr_ + kCtrWork, 0, sizeof(unsigned), stream_));
        detail::process_kernel<St><<<ctas, St::kThreadsPerTile, 0, stream_>>>(stage, d_run_, in, d_ctr_ + kCtrWork,
                                                                             d_ms_, pass, mode);
      }
      PIKO_STAGE_CHECK(cudaGetLastError());
      PIKO_STAGE_CHECK(cudaMemcpyAsync(&st[0], d_ctr_ + kCtrStatus, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
      PIKO_STAGE_CHECK(cudaStreamSynchronize(stream_));
      if (st[0] & detail::kStatusEmitOverflow)
        throw std::runtime_error("piko::Pipe: a process call emitted more than 2^20 primitives");
      if (st[0]) {
        // grow what overflowed; the caller runs the frame again
        if (st[0] & detail::kStatusQueueOverflow) grow_all_outputs<I>(2);
        return false;
      }
      if (loops) {
        // the primitives the stage sent to itself become its next input
        unsigned next = 0;
        PIKO_STAGE_CHECK(cudaMemcpyAsync(&next, d_ctr_ + kStages + I, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
        PIKO_STAGE_CHECK(cudaStreamSynchronize(stream_));
        std::swap(q_[I], loop_[I]);   // the consumed input becomes the next round's loop queue
        grow(loop_[I], std::max<size_t>(4 * (size_t)std::max(next, 1u), 1u << 16), sizeof(In));
        PIKO_STAGE_CHECK(cudaMemcpyAsync(d_ctr_ + I, &next, sizeof(unsigned), cudaMemcpyHostToDevice, stream_));
        PIKO_STAGE_CHECK(cudaMemsetAsync(d_ctr_ + kStages + I, 0, sizeof(unsigned), stream_));
        in_count = next;
      } else {
        in_count = 0;
      }
    }
    return true;
  }

  bool links_has_self_loop(int i) const
  {
    for (int p = 0; p < kNumPorts; ++p)
      if (links_[i][p] == i) return true;
    return false;
  }

  void grow_target(int to, size_t n) { grow_target_impl(to, n, std::integral_constant<int, 0>()); }
  void grow_target_impl(int, size_t, std::integral_constant<int, sizeof...(S)>) {}
  template <int J>
  void grow_target_impl(int to, size_t n, std::integral_constant<int, J>)
  {
    if (to == J) {
      grow(q_[J], n, sizeof(typename StageT<J>::In));
      return;
    }
    grow_target_impl(to, n, std::integral_constant<int, J + 1>());
  }

  void grow_loop(int j, size_t n) { grow_loop_impl(j, n, std::integral_constant<int, 0>()); }
  void grow_loop_impl(int, size_t, std::integral_constant<int, sizeof...(S)>) {}
  template <int J>
  void grow_loop_impl(int j, size_t n, std::integral_constant<int, J>)
  {
    if (j == J) {
      grow(loop_[J], n, sizeof(typename StageT<J>::In));
      return;
    }
    grow_loop_impl(j, n, std::integral_constant<int, J + 1>());
  }

  // between frames, after an overflow: every queue stage I feeds, doubled
  template <int I>
  void grow_all_outputs(size_t factor)
  {
    for (int p = 0; p < kNumPorts; ++p) {
      const int to = links_[I][p];
      if (to == I) grow_loop(I, loop_[I].cap * factor);
      else if (to > I) grow_target(to, q_[to].cap * factor);
    }
  }
};

#undef PIKO_STAGE_CHECK

}  // namespace piko
