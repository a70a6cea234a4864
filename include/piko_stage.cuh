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

#include "piko_stage_device.cuh"

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

namespace piko {
namespace detail {

#define PIKO_STAGE_CHECK(call)                                                         \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string("piko::Pipe: ") + cudaGetErrorString(e_)); \
  } while (0)

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

}  // namespace detail

// One stage as the runtime sees it, without its C++ type: the Stage<>
// arguments, the primitive sizes, the stage object (bytes, StageCommon first)
// and its two kernels, whose parameters are
//   assign (stage object, StageRun*, const In*, unsigned n, int pass)
//   process(stage object, StageRun*, const In*, unsigned* work, MutableState*, int pass, int mode).
// `links[p]` is where output port p goes: a stage index, kScreen, or -2.
struct StageSpec {
  int binX = 0, binY = 0, threads = 0;
  size_t inSize = 0, outSize = 0, objSize = 0;
  void* obj = nullptr;
  const void* assignKernel = nullptr;
  const void* processKernel = nullptr;
  int links[kNumPorts] = {-2, -2, -2, -2, -2};
};

// The pipeline runtime over type-less stages (piko::Pipe wraps it for
// stages known at compile time; piko-public_b200/pikoc.py uses it for stage
// code compiled at run time).
class PipeCore {
 public:
  PipeCore() = default;
  ~PipeCore() { destroy(); }
  PipeCore(const PipeCore&) = delete;
  PipeCore& operator=(const PipeCore&) = delete;

  std::vector<StageSpec> specs;

  void allocate(ConstantState& cs, MutableState& ms, const void* input, int count)
  {
    for (size_t i = 0; i < specs.size(); ++i)
      for (int p = 0; p < kNumPorts; ++p) {
        const int to = specs[i].links[p];
        // allowed: unlinked (-2), kScreen, the stage itself or a later stage
        if (to < -2 || to >= (int)specs.size() || (to >= 0 && to < (int)i))
          throw std::invalid_argument("piko::Pipe: a port may feed only a later stage, the stage itself or the screen");
      }
    const int n = (int)specs.size();
    q_.assign(n, Queue());
    loop_.assign(n, Queue());
    loop2_.assign(n, Queue());
    processed_.assign(n, 0);
    rounds_.assign(n, 0);
    cs_ = &cs;
    ms_ = &ms;
    W_ = cs.screenSizeX;
    H_ = cs.screenSizeY;
    if (W_ <= 0 || H_ <= 0 || count < 0 || n == 0) throw std::invalid_argument("piko::Pipe::allocate");
    if (!stream_) PIKO_STAGE_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    alloc_common();
    count_ = (unsigned)count;
    grow(q_[0], std::max<size_t>(count_, 1), specs[0].inSize);
    // every later stage's input queue and every self loop's queue, sized up
    // front: a queue that earlier stages already wrote must not move during a
    // frame, so queues grow only between frames (after an overflow)
    const size_t initial = std::max<size_t>(4 * (size_t)std::max(count_, 1u), 1u << 16);
    for (int j = 1; j < n; ++j) grow(q_[j], initial, specs[j].inSize);
    for (int j = 0; j < n; ++j)
      if (self_loop(j)) {
        grow(loop_[j], initial, specs[j].inSize);
        grow(loop2_[j], initial, specs[j].inSize);
      }
    if (count)
      PIKO_STAGE_CHECK(cudaMemcpyAsync(q_[0].data, input, specs[0].inSize * count_, cudaMemcpyHostToDevice, stream_));
    PIKO_STAGE_CHECK(cudaStreamSynchronize(stream_));
  }

  // prepare(): the caller's states as they are now.  zBuffer of the caller's
  // MutableState is a device pointer (the nvcc path) or, with host_depth,
  // a host array of W * H floats copied to the device depth buffer.
  void prepare(bool host_depth = false)
  {
    cs_copy_ = *cs_;
    MutableState m = *ms_;
    if (host_depth) {
      if (!d_depth_) PIKO_STAGE_CHECK(cudaMalloc((void**)&d_depth_, sizeof(float) * (size_t)W_ * H_));
      if (m.zBuffer)
        PIKO_STAGE_CHECK(cudaMemcpyAsync(d_depth_, m.zBuffer, sizeof(float) * (size_t)W_ * H_, cudaMemcpyHostToDevice,
                                         stream_));
      m.zBuffer = d_depth_;
    }
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

  unsigned* screen() { return d_fb_; }
  float* device_depth() { return d_depth_; }
  int width() const { return W_; }
  int height() const { return H_; }
  void getData(unsigned* host) const
  {
    PIKO_STAGE_CHECK(cudaMemcpy(host, d_fb_, sizeof(unsigned) * (size_t)W_ * H_, cudaMemcpyDeviceToHost));
  }
  void clearScreen(unsigned color)
  {
    std::vector<unsigned> c((size_t)W_ * H_, color);
    PIKO_STAGE_CHECK(cudaMemcpy(d_fb_, c.data(), sizeof(unsigned) * c.size(), cudaMemcpyHostToDevice));
  }
  const std::vector<unsigned long long>& processed() const { return processed_; }
  int rounds(int stage) const { return rounds_[stage]; }

  void destroy()
  {
    for (auto& q : q_) free_queue(q);
    for (auto& q : loop_) free_queue(q);
    for (auto& q : loop2_) free_queue(q);
    auto fr = [](void* p) { if (p) cudaFree(p); };
    fr(d_fb_); fr(d_ms_); fr(d_run_); fr(d_ctr_); fr(d_bins_); fr(d_pairs_); fr(d_list_); fr(d_perm_);
    fr(d_iota_); fr(d_ksort_); fr(d_tmp_); fr(d_pixkey_); fr(d_depth_);
    d_fb_ = nullptr; d_ms_ = nullptr; d_run_ = nullptr; d_ctr_ = nullptr; d_bins_ = nullptr;
    d_pairs_ = nullptr; d_list_ = nullptr; d_perm_ = nullptr; d_iota_ = nullptr; d_ksort_ = nullptr;
    d_tmp_ = nullptr; d_pixkey_ = nullptr; d_depth_ = nullptr;
    bins_cap_ = list_cap_ = in_cap_ = tmp_bytes_ = 0;
    if (stream_) cudaStreamDestroy(stream_);
    stream_ = nullptr;
  }

 private:
  // A queue of primitives with their sequential keys.
  struct Queue { void* data = nullptr; unsigned long long* keys = nullptr; size_t cap = 0; size_t elem = 0; };
  // counters: [0..n) queue counts, n + i: loop queue counts, 2n: pair cursor,
  // 2n + 1: status, 2n + 2: work counter
  int ctr_pairs() const { return 2 * (int)specs.size(); }
  int ctr_status() const { return ctr_pairs() + 1; }
  int ctr_work() const { return ctr_pairs() + 2; }
  int ctr_n() const { return ctr_pairs() + 3; }

  ConstantState* cs_ = nullptr;
  ConstantState cs_copy_{};
  MutableState* ms_ = nullptr;
  int W_ = 0, H_ = 0;
  unsigned count_ = 0;
  cudaStream_t stream_ = nullptr;
  // q_[i]: stage i's input queue; a self-looping stage's rounds alternate
  // between loop_[i] and loop2_[i], so q_[i] keeps the frame's input for a
  // frame that must run again
  std::vector<Queue> q_, loop_, loop2_;
  unsigned* d_fb_ = nullptr;
  unsigned long long* d_pixkey_ = nullptr;
  float* d_depth_ = nullptr;     // the depth buffer when the caller's is host memory
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
  std::vector<unsigned long long> processed_;
  std::vector<int> rounds_;

  static void free_queue(Queue& q)
  {
    if (q.data) cudaFree(q.data);
    if (q.keys) cudaFree(q.keys);
    q = Queue();
  }

  // (re)allocates a queue for n primitives of elem bytes (contents not kept)
  static void grow(Queue& q, size_t n, size_t elem)
  {
    if (n <= q.cap && q.data) return;
    free_queue(q);
    PIKO_STAGE_CHECK(cudaMalloc(&q.data, n * std::max<size_t>(elem, 1)));
    PIKO_STAGE_CHECK(cudaMalloc((void**)&q.keys, n * sizeof(unsigned long long)));
    q.cap = n;
    q.elem = elem;
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
    if (d_ctr_) cudaFree(d_ctr_);
    PIKO_STAGE_CHECK(cudaMalloc((void**)&d_ctr_, sizeof(unsigned) * ctr_n()));
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
    const size_t need = std::max<size_t>(std::max(a, b), 256);
    if (need > tmp_bytes_ || !d_tmp_) {
      if (d_tmp_) cudaFree(d_tmp_);
      d_tmp_ = nullptr;
      PIKO_STAGE_CHECK(cudaMalloc(&d_tmp_, need));
      tmp_bytes_ = need;
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

  bool self_loop(int i) const
  {
    for (int p = 0; p < kNumPorts; ++p)
      if (specs[i].links[p] == i) return true;
    return false;
  }

  // Runs every stage once over its input (a self-looping stage: until its
  // own queue drains).  Returns false after an overflow (capacities grown).
  bool frame()
  {
    PIKO_STAGE_CHECK(cudaMemsetAsync(d_ctr_, 0, sizeof(unsigned) * ctr_n(), stream_));
    PIKO_STAGE_CHECK(cudaMemsetAsync(d_pixkey_, 0, sizeof(unsigned long long) * (size_t)W_ * H_, stream_));
    unsigned c0 = count_;
    PIKO_STAGE_CHECK(cudaMemcpyAsync(d_ctr_ + 0, &c0, sizeof(unsigned), cudaMemcpyHostToDevice, stream_));
    for (auto& p : processed_) p = 0;
    for (int i = 0; i < (int)specs.size(); ++i)
      if (!run_stage(i)) return false;
    return true;
  }

  // Where each port of stage I sends its primitives; true when a port feeds
  // the screen.
  bool route(int I, detail::StageRun& r, const Queue& self_out)
  {
    bool screen = false;
    const int n = (int)specs.size();
    for (int p = 0; p < kNumPorts; ++p) {
      const int to = specs[I].links[p];
      r.outKind[p] = 0;
      r.outData[p] = nullptr;
      r.outKeys[p] = nullptr;
      r.outCount[p] = nullptr;
      r.outCap[p] = 0;
      r.outSize[p] = (unsigned)specs[I].outSize;
      if (to == kScreen) {
        r.outKind[p] = 2;
        screen = true;
      } else if (to == I) {
        r.outKind[p] = 1;
        r.outData[p] = self_out.data;
        r.outKeys[p] = self_out.keys;
        r.outCount[p] = d_ctr_ + n + I;
        r.outCap[p] = (unsigned)self_out.cap;
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

  void launch(const void* kernel, int grid, int block, void** args)
  {
    PIKO_STAGE_CHECK(cudaLaunchKernel(kernel, dim3((unsigned)grid), dim3((unsigned)block), args, 0, stream_));
  }

  bool run_stage(int I)
  {
    StageSpec& sp = specs[I];
    const int n = (int)specs.size();
    const int bx = bins_of(sp.binX, W_), by = bins_of(sp.binY, H_);
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
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sp.processKernel, sp.threads, 0) != cudaSuccess) {
      cudaGetLastError();
      per_sm = 2;
    }
    const int ctas = sms * std::max(per_sm, 1);
    const bool loops = self_loop(I);
    // the stage object as launched: its copy of the frame's constants
    reinterpret_cast<StageCommon*>(sp.obj)->constState = cs_copy_;
    rounds_[I] = 0;
    Queue* cur = &q_[I];      // this round's input
    Queue* out = &loop_[I];   // this round's self-loop output
    for (int round = 0; round < kMaxLoopRounds; ++round) {
      if (in_count == 0) break;
      ++rounds_[I];
      processed_[I] += in_count;
      // rank the input by sequential key (the host input is in order already)
      if (in_count > in_cap_ || !d_perm_) {
        size_t c0 = 0, c1 = 0, c2 = 0;
        const size_t m = (size_t)in_count + in_count / 2 + 1024;
        grow_buf(d_perm_, c0, m);
        grow_buf(d_iota_, c1, m);
        grow_buf(d_ksort_, c2, m);
        in_cap_ = m;
      }
      const unsigned iblocks = std::min<unsigned>((in_count + 255) / 256, (unsigned)sms * 8u);
      if (I == 0 && round == 0) {
        detail::iota_kernel<<<iblocks, 256, 0, stream_>>>(d_perm_, in_count);
      } else {
        detail::iota_kernel<<<iblocks, 256, 0, stream_>>>(d_iota_, in_count);
        ensure_tmp(in_count);
        size_t tb = tmp_bytes_;
        PIKO_STAGE_CHECK(cub::DeviceRadixSort::SortPairs(d_tmp_, tb, cur->keys, d_ksort_, d_iota_, d_perm_,
                                                         (int)in_count, 0, 64, stream_));
      }
      const size_t want = std::max<size_t>(4 * (size_t)in_count, 1u << 16);
      if (list_cap_ < want) grow_lists(want);
      detail::StageRun r;
      memset(&r, 0, sizeof(r));
      r.numBinsX = bx; r.numBinsY = by;
      r.binSizeX = sp.binX > 0 ? sp.binX : W_;
      r.binSizeY = sp.binY > 0 ? sp.binY : H_;
      r.binCount = d_bins_;
      r.binStart = d_bins_ + bins;
      r.pairs = d_pairs_;
      r.binList = d_list_;
      r.listCap = (unsigned)list_cap_;
      r.pairCount = d_ctr_ + ctr_pairs();
      r.perm = d_perm_;
      r.stage = I;
      r.keyBase = processed_[I] - in_count;
      r.fb = d_fb_;
      r.pixKey = d_pixkey_;
      r.W = W_; r.H = H_;
      r.status = d_ctr_ + ctr_status();
      const bool screen = route(I, r, *out);
      PIKO_STAGE_CHECK(cudaMemcpyAsync(d_run_, &r, sizeof(r), cudaMemcpyHostToDevice, stream_));
      PIKO_STAGE_CHECK(cudaMemsetAsync(d_bins_, 0, sizeof(unsigned) * bins, stream_));
      PIKO_STAGE_CHECK(cudaMemsetAsync(d_ctr_ + ctr_pairs(), 0, sizeof(unsigned), stream_));
      const void* in = cur->data;
      detail::StageRun* run = d_run_;
      unsigned cnt = in_count;
      int pass = 0;
      void* aargs[] = {sp.obj, &run, &in, &cnt, &pass};
      launch(sp.assignKernel, (int)iblocks, 256, aargs);
      detail::scan_bins<<<1, 1024, 0, stream_>>>(d_run_);
      pass = 1;
      launch(sp.assignKernel, (int)iblocks, 256, aargs);
      unsigned st[2] = {0, 0};
      PIKO_STAGE_CHECK(cudaMemcpyAsync(&st[0], d_ctr_ + ctr_status(), sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
      PIKO_STAGE_CHECK(cudaMemcpyAsync(&st[1], d_ctr_ + ctr_pairs(), sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
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
      unsigned* work = d_ctr_ + ctr_work();
      MutableState* ms = d_ms_;
      for (int p = 0; p < runs; ++p) {
        int mode = !exact ? detail::kScreenDirect
                          : (p == 0 ? detail::kScreenDepthOnly : (p == 1 ? detail::kScreenKeys : detail::kScreenColour));
        int pp = p;
        PIKO_STAGE_CHECK(cudaMemsetAsync(work, 0, sizeof(unsigned), stream_));
        void* pargs[] = {sp.obj, &run, &in, &work, &ms, &pp, &mode};
        launch(sp.processKernel, ctas, sp.threads, pargs);
      }
      PIKO_STAGE_CHECK(cudaGetLastError());
      PIKO_STAGE_CHECK(cudaMemcpyAsync(&st[0], d_ctr_ + ctr_status(), sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
      PIKO_STAGE_CHECK(cudaStreamSynchronize(stream_));
      if (st[0] & detail::kStatusEmitOverflow)
        throw std::runtime_error("piko::Pipe: a process call emitted more than 2^20 primitives");
      if (st[0]) {
        // grow every queue this stage feeds; the caller runs the frame again
        for (int p = 0; p < kNumPorts; ++p) {
          const int to = sp.links[p];
          if (to == I) {
            grow(loop_[I], loop_[I].cap * 2, sp.inSize);
            grow(loop2_[I], loop2_[I].cap * 2, sp.inSize);
          }
          else if (to > I) grow(q_[to], q_[to].cap * 2, q_[to].elem);
        }
        return false;
      }
      if (loops) {
        // the primitives the stage sent to itself become its next input
        unsigned next = 0;
        PIKO_STAGE_CHECK(cudaMemcpyAsync(&next, d_ctr_ + n + I, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
        PIKO_STAGE_CHECK(cudaStreamSynchronize(stream_));
        Queue* spare = cur == &q_[I] ? &loop2_[I] : cur;   // never the frame's input queue
        cur = out;
        out = spare;
        grow(*out, std::max<size_t>(4 * (size_t)std::max(next, 1u), 1u << 16), sp.inSize);
        PIKO_STAGE_CHECK(cudaMemcpyAsync(d_ctr_ + I, &next, sizeof(unsigned), cudaMemcpyHostToDevice, stream_));
        PIKO_STAGE_CHECK(cudaMemsetAsync(d_ctr_ + n + I, 0, sizeof(unsigned), stream_));
        in_count = next;
      } else {
        in_count = 0;
      }
    }
    return true;
  }
};

// A pipeline of stages S0..Sn-1 (given in an order where every connection goes
// to a later stage or to the stage itself), drawn into a W x H screen.
template <class... S>
class Pipe {
 public:
  static constexpr int kStages = (int)sizeof...(S);
  using In0 = typename std::tuple_element<0, std::tuple<S...>>::type::In;

  Pipe() { specs_init(std::integral_constant<int, 0>()); }
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
    core_.specs[from].links[port] = to;
  }

  void allocate(ConstantState& cs, MutableState& ms, const In0* input, int count)
  {
    core_.allocate(cs, ms, input, count);
  }
  void prepare() { core_.prepare(false); }
  void run_single() { core_.run_single(); }
  // PikoScreen::getData(): the screen, W*H RGBA8 words (device pointer), and a host copy.
  unsigned* screen() { return core_.screen(); }
  void getData(unsigned* host) const { core_.getData(host); }
  void clearScreen(unsigned color) { core_.clearScreen(color); }
  // primitives each stage processed in the last frame (all rounds)
  const std::vector<unsigned long long>& processed() const { return core_.processed(); }
  int rounds(int stage) const { return core_.rounds(stage); }
  void destroy() { core_.destroy(); }

 private:
  PipeCore core_;

  void specs_init(std::integral_constant<int, sizeof...(S)>) {}
  template <int I>
  void specs_init(std::integral_constant<int, I>)
  {
    using St = typename std::tuple_element<I, std::tuple<S...>>::type;
    if (I == 0) core_.specs.resize(kStages);
    StageSpec& sp = core_.specs[I];
    sp.binX = St::kBinSizeX;
    sp.binY = St::kBinSizeY;
    sp.threads = St::kThreadsPerTile;
    sp.inSize = sizeof(typename St::In);
    sp.outSize = sizeof(typename St::Out);
    sp.objSize = sizeof(St);
    sp.obj = &std::get<I>(stages);
    sp.assignKernel = (const void*)detail::assign_kernel<St>;
    sp.processKernel = (const void*)detail::process_kernel<St>;
    specs_init(std::integral_constant<int, I + 1>());
  }
};

#undef PIKO_STAGE_CHECK

}  // namespace piko
