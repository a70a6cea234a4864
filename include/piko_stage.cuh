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
 *     AssignBin   one thread per input primitive calls assignBin(p); its
 *                 assignToBin calls fill per-bin counts, an exclusive scan gives
 *                 each bin its list, and a second pass writes the lists;
 *     Schedule    schedule(binID) names the policy (LOAD_BALANCE: CTAs take bins
 *                 from a queue; ROUND_ROBIN: CTA c takes bins c, c + CTAs, ...;
 *                 SERIAL: one CTA takes every bin in order; ALL: the
 *                 primitives of each bin are split over tileSplitSize CTAs);
 *     Process     a persistent launch of threadsPerTile-thread CTAs; for each
 *                 bin, thread t processes primitives t, t + threadsPerTile, ...
 *                 (the reference's process loop, pikoc/src/pikoc.cpp:236-262);
 *                 emit(p, port) appends p to the input of the stage connected
 *                 to that port, or, for a port connected to the screen, writes
 *                 p.color at p.pos as PikoScreen::assignBin does (stage.h:57-61);
 *     a stage connected to itself runs again on what it emitted to itself until
 *     nothing is left (at most kMaxLoopRounds rounds), like the reference's
 *     Split loop (pikoc/src/pikoc.cpp:294-308).
 *
 * Bin size 0 means one full-screen bin (pikoc/include/PikoSummary.hpp:279); the
 * bin grid is screenSize / binSize rounded down, as in the reference.
 * Queues and bin lists that outgrow their capacity are grown and the frame is
 * run again; device-side work never waits on another CTA.  The two reference
 * pipelines also run as hand-fused kernels behind the C ABI (piko_b200.h); this
 * header is the general path for other pipelines.
 */
#pragma once

#include <cuda_runtime.h>

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

namespace detail {

enum : unsigned { kStatusQueueOverflow = 1u, kStatusListOverflow = 2u };

// Device view of one stage for one launch.
struct StageRun {
  int numBinsX, numBinsY, binSizeX, binSizeY;
  int pass;                 // AssignBin: 0 count, 1 write lists
  unsigned* binCount;       // [bins]
  unsigned* binCursor;      // [bins]
  unsigned* binList;        // [listCap] input indices
  unsigned listCap;
  unsigned* listTotal;      // entries assigned (count pass)
  int policy, split;        // from specifySchedule
  // emit routing, per port
  void* outData[kNumPorts];
  unsigned* outCount[kNumPorts];
  unsigned outCap[kNumPorts];
  int outKind[kNumPorts];   // 0 unconnected, 1 stage input queue, 2 screen
  unsigned* fb;
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

  // set by piko::Pipe before each launch
  detail::StageRun* run_ = nullptr;
  const ConstantState* constState_ = nullptr;
  MutableState* mutableState = nullptr;
  int binID_ = 0;
  unsigned prim_ = 0;   // input index being assigned

 protected:
  __device__ const ConstantState& constState() const { return *constState_; }

  __device__ void assignToBin(const In&, int binID)
  {
    detail::StageRun& r = *run_;
    if (binID < 0 || binID >= r.numBinsX * r.numBinsY) return;
    if (r.pass == 0) {
      atomicAdd(&r.binCount[binID], 1u);
      atomicAdd(r.listTotal, 1u);
    } else {
      const unsigned slot = atomicAdd(&r.binCursor[binID], 1u);
      if (slot < r.listCap) r.binList[slot] = prim_;
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
    if (r.outKind[port] == 2) {
      if constexpr (std::is_same<Out, Pixel>::value) {
        if (p.pos.x >= 0 && p.pos.x < r.W && p.pos.y >= 0 && p.pos.y < r.H)
          r.fb[(size_t)p.pos.y * (size_t)r.W + (size_t)p.pos.x] = p.color;
      }
    } else if (r.outKind[port] == 1) {
      const unsigned slot = atomicAdd(r.outCount[port], 1u);
      if (slot < r.outCap[port]) {
        Out q = p;
        if constexpr (has_bin_id<Out>::value) q.binID = binID_;
        static_cast<Out*>(r.outData[port])[slot] = q;
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

template <class S>
__global__ void assign_kernel(S stage, StageRun* run, const typename S::In* in, const unsigned* count, int pass,
                              const ConstantState* cs)
{
  __shared__ StageRun s_run;
  if (threadIdx.x == 0) {
    s_run = *run;
    s_run.pass = pass;
  }
  __syncthreads();
  stage.run_ = &s_run;
  stage.constState_ = cs;
  const unsigned n = *count;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    stage.prim_ = i;
    stage.assignBin(in[i]);
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
    if (i < bins) run->binCursor[i] = s_carry + s_sum[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) s_carry += s_sum[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0 && s_carry > run->listCap) atomicOr(run->status, (unsigned)kStatusListOverflow);
}

template <class S>
__global__ void process_kernel(S stage, StageRun* run, const typename S::In* in, const unsigned* binOff,
                               unsigned* workNext, const ConstantState* cs, MutableState* ms)
{
  __shared__ StageRun s_run;
  __shared__ int s_bin;
  __shared__ unsigned s_lo, s_hi;
  if (threadIdx.x == 0) s_run = *run;
  __syncthreads();
  stage.run_ = &s_run;
  stage.constState_ = cs;
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
        const unsigned lo = b == 0 ? 0u : binOff[b - 1], hi = binOff[b];
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
    for (unsigned j = s_lo + threadIdx.x; j < s_hi && j < s_run.listCap; j += blockDim.x) stage.process(in[s_run.binList[j]]);
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
    PIKO_STAGE_CHECK(cudaMemcpyAsync(d_cs_, cs_, sizeof(ConstantState), cudaMemcpyHostToDevice, stream_));
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
    for (auto& q : q_) { if (q.data) cudaFree(q.data); q.data = nullptr; q.cap = 0; }
    for (auto& q : loop_) { if (q.data) cudaFree(q.data); q.data = nullptr; q.cap = 0; }
    auto fr = [](void* p) { if (p) cudaFree(p); };
    fr(d_fb_); fr(d_cs_); fr(d_ms_); fr(d_run_); fr(d_ctr_); fr(d_bins_); fr(d_list_);
    d_fb_ = nullptr; d_cs_ = nullptr; d_ms_ = nullptr; d_run_ = nullptr; d_ctr_ = nullptr;
    d_bins_ = nullptr; d_list_ = nullptr;
    bins_cap_ = list_cap_ = 0;
    if (stream_) cudaStreamDestroy(stream_);
    stream_ = nullptr;
  }

 private:
  struct Queue { void* data = nullptr; size_t cap = 0; };
  // counters: [0..kStages) queue counts, kStages + i: loop queue counts,
  // 2*kStages: list total, +1 status, +2 work counter
  enum { kCtrListTotal = 2 * sizeof...(S), kCtrStatus, kCtrWork, kCtrN };

  int links_[sizeof...(S)][kNumPorts];
  ConstantState* cs_ = nullptr;
  MutableState* ms_ = nullptr;
  int W_ = 0, H_ = 0;
  unsigned count_ = 0;
  cudaStream_t stream_ = nullptr;
  Queue q_[sizeof...(S)], loop_[sizeof...(S)];
  unsigned* d_fb_ = nullptr;
  ConstantState* d_cs_ = nullptr;
  MutableState* d_ms_ = nullptr;
  detail::StageRun* d_run_ = nullptr;
  unsigned* d_ctr_ = nullptr;
  unsigned* d_bins_ = nullptr;   // [2 * bins_cap_]: counts, offsets / cursors
  unsigned* d_list_ = nullptr;
  size_t bins_cap_ = 0, list_cap_ = 0;
  std::vector<unsigned long long> processed_ = std::vector<unsigned long long>(sizeof...(S), 0);
  int rounds_[sizeof...(S)] = {};

  void grow(Queue& q, size_t n, size_t elem)
  {
    if (n <= q.cap) return;
    if (q.data) cudaFree(q.data);
    q.data = nullptr;
    q.cap = 0;
    PIKO_STAGE_CHECK(cudaMalloc(&q.data, n * elem));
    q.cap = n;
  }

  void alloc_common()
  {
    if (!d_fb_) PIKO_STAGE_CHECK(cudaMalloc((void**)&d_fb_, sizeof(unsigned) * (size_t)W_ * H_));
    if (!d_cs_) PIKO_STAGE_CHECK(cudaMalloc((void**)&d_cs_, sizeof(ConstantState)));
    if (!d_ms_) PIKO_STAGE_CHECK(cudaMalloc((void**)&d_ms_, sizeof(MutableState)));
    if (!d_run_) PIKO_STAGE_CHECK(cudaMalloc((void**)&d_run_, sizeof(detail::StageRun)));
    if (!d_ctr_) PIKO_STAGE_CHECK(cudaMalloc((void**)&d_ctr_, sizeof(unsigned) * kCtrN));
    clearScreen(0xff663313u);   // PikoScreen's initial colour (stage.h:83-85)
  }

  // screenSize / binSize, rounded down, as the reference sizes its bin grid
  // (stage.h:273-274): pixels past the last whole bin get no bin (at least one
  // bin per axis here, so that a screen smaller than a bin still has one)
  static int bins_of(int size, int extent) { return size <= 0 ? 1 : std::max(1, extent / size); }

  template <int I>
  using StageT = typename std::tuple_element<I, std::tuple<S...>>::type;

  // Runs every stage once over its input (a self-looping stage: until its
  // own queue drains).  Returns false after an overflow (capacities grown).
  bool frame()
  {
    PIKO_STAGE_CHECK(cudaMemsetAsync(d_ctr_, 0, sizeof(unsigned) * kCtrN, stream_));
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
  void route(detail::StageRun& r)
  {
    for (int p = 0; p < kNumPorts; ++p) {
      const int to = links_[I][p];
      r.outKind[p] = 0;
      r.outData[p] = nullptr;
      r.outCount[p] = nullptr;
      r.outCap[p] = 0;
      if (to == kScreen) {
        r.outKind[p] = 2;
      } else if (to == I) {
        r.outKind[p] = 1;
        r.outData[p] = loop_[I].data;
        r.outCount[p] = d_ctr_ + kStages + I;
        r.outCap[p] = (unsigned)loop_[I].cap;
      } else if (to > I) {
        r.outKind[p] = 1;
        r.outData[p] = q_[to].data;
        r.outCount[p] = d_ctr_ + to;
        r.outCap[p] = (unsigned)q_[to].cap;
      }
    }
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
    const size_t want = std::max<size_t>(4 * (size_t)std::max(in_count, 1u), 1u << 16);
    if (list_cap_ < want) {
      if (d_list_) cudaFree(d_list_);
      d_list_ = nullptr;
      PIKO_STAGE_CHECK(cudaMalloc((void**)&d_list_, sizeof(unsigned) * want));
      list_cap_ = want;
    }
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, detail::process_kernel<St>, St::kThreadsPerTile, 0);
    const int ctas = sms * std::max(per_sm, 1);
    rounds_[I] = 0;
    for (int round = 0; round < kMaxLoopRounds; ++round) {
      if (in_count == 0) break;
      ++rounds_[I];
      processed_[I] += in_count;
      detail::StageRun r;
      memset(&r, 0, sizeof(r));
      r.numBinsX = bx; r.numBinsY = by;
      r.binSizeX = St::kBinSizeX > 0 ? St::kBinSizeX : W_;
      r.binSizeY = St::kBinSizeY > 0 ? St::kBinSizeY : H_;
      r.binCount = d_bins_;
      r.binCursor = d_bins_ + bins;
      r.binList = d_list_;
      r.listCap = (unsigned)list_cap_;
      r.listTotal = d_ctr_ + kCtrListTotal;
      r.fb = d_fb_;
      r.W = W_; r.H = H_;
      r.status = d_ctr_ + kCtrStatus;
      route<I>(r);
      PIKO_STAGE_CHECK(cudaMemcpyAsync(d_run_, &r, sizeof(r), cudaMemcpyHostToDevice, stream_));
      PIKO_STAGE_CHECK(cudaMemsetAsync(d_bins_, 0, sizeof(unsigned) * bins, stream_));
      PIKO_STAGE_CHECK(cudaMemsetAsync(d_ctr_ + kCtrListTotal, 0, sizeof(unsigned), stream_));
      PIKO_STAGE_CHECK(cudaMemsetAsync(d_ctr_ + kCtrWork, 0, sizeof(unsigned), stream_));
      const In* in = static_cast<const In*>(q_[I].data);
      const int ablocks = (int)std::min<unsigned>((in_count + 255) / 256, (unsigned)sms * 8u);
      detail::assign_kernel<St><<<ablocks, 256, 0, stream_>>>(stage, d_run_, in, d_ctr_ + I, 0, d_cs_);
      detail::scan_bins<<<1, 1024, 0, stream_>>>(d_run_);
      detail::assign_kernel<St><<<ablocks, 256, 0, stream_>>>(stage, d_run_, in, d_ctr_ + I, 1, d_cs_);
      // bin b's list ends where bin b + 1's cursor started: after the write
      // pass, binCursor[b] is the end of bin b
      detail::process_kernel<St><<<ctas, St::kThreadsPerTile, 0, stream_>>>(stage, d_run_, in, d_bins_ + bins,
                                                                           d_ctr_ + kCtrWork, d_cs_, d_ms_);
      PIKO_STAGE_CHECK(cudaGetLastError());
      unsigned st[2] = {0, 0};
      PIKO_STAGE_CHECK(cudaMemcpyAsync(&st[0], d_ctr_ + kCtrStatus, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
      PIKO_STAGE_CHECK(cudaMemcpyAsync(&st[1], d_ctr_ + kCtrListTotal, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
      PIKO_STAGE_CHECK(cudaStreamSynchronize(stream_));
      if (st[0]) {
        // grow what overflowed; the caller runs the frame again
        if (st[0] & detail::kStatusListOverflow) {
          const size_t need = (size_t)st[1] + st[1] / 4 + 1024;
          if (d_list_) cudaFree(d_list_);
          d_list_ = nullptr;
          PIKO_STAGE_CHECK(cudaMalloc((void**)&d_list_, sizeof(unsigned) * need));
          list_cap_ = need;
        }
        if (st[0] & detail::kStatusQueueOverflow) grow_all_outputs<I>(2);
        return false;
      }
      if (links_has_self_loop(I)) {
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
