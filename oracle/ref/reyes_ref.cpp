// TEST INFRASTRUCTURE — part of the oracle, never part of the product path.
//
// Builds the reference's own Reyes renderer (ReyesPipe: SplitStage (self loop)
// -> DiceStage -> ShadeStage -> PikoScreen) for the CPU as `pikoc --target=CPU
// --opt` would.  The stage code is the reference's, compiled in place; this
// file supplies what pikoc generates:
//   * emit routing (Split has two ports)   pikoc/src/pikoc.cpp:69-194
//   * kernels; the pipe has a loop, so every Process kernel fetches with
//     fetchPrimAtomic and skips updatePrimCount  pikoc/src/pikoc.cpp:276-318
//   * run_single with the do { Split.process } while (split.hasPrims) loop
//                                           pikoc/src/Backend/CPUBackend.cpp:428-520
// Deviations are the ones of raster_ref.cpp (GLUT-free entry points, CPU thread
// count as a parameter, depth buffer sized W*H, bin capacity probe), plus
// observation hooks in the generated emit routing that count the leaves Split
// sends to Dice, the micropolygons Dice emits and the Pixels Shade emits.
#include <algorithm>
#include <atomic>
#include <cassert>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#define private public
#define protected public
#include "reyesPipe.h"
#undef private
#undef protected

thread_local int threadIdx_x = 0;
thread_local int blockIdx_x = 0;
int blockDim_x = 0;

static std::atomic<long long> g_leaves(0), g_upolys(0), g_emitted(0);
static bool g_record_leaves = false;
static std::vector<int> g_leaf_rec;

static SplitStage* g_split = nullptr;
static DiceStage* g_dice = nullptr;
static ShadeStage* g_shade = nullptr;

// ---------------------------------------------------------------- emit routing
void SplitStage::emit(piko_patch p, int outPortNum)
{
  if (outPortNum == 0) {
    g_leaves.fetch_add(1, std::memory_order_relaxed);
    if (g_record_leaves) {
      g_leaf_rec.push_back(p.id); g_leaf_rec.push_back(p.numSplits);
      g_leaf_rec.push_back(p.nu); g_leaf_rec.push_back(p.nv);
    }
    ((DiceStage*) d_outPort_[0])->assignBin(p);
  } else {
    ((SplitStage*) d_outPort_[1])->assignBin(p);
  }
}
void DiceStage::emit(piko_upoly p, int outPortNum)
{
  g_upolys.fetch_add(1, std::memory_order_relaxed);
  ((ShadeStage*) d_outPort_[0])->assignBin(p);
}
void ShadeStage::emit(Pixel p, int outPortNum)
{
  g_emitted.fetch_add(1, std::memory_order_relaxed);
  ((PikoScreen*) d_outPort_[0])->assignBin(p);
}

// ---------------------------------------------------------------- kernels
static void kernel0(PikoArray<piko_patch>* input, SplitStage* d_split)
{
  const int gid = getGID();
  if (gid >= input->getNumPrims()) return;
  d_split->assignBin((*input)[gid]);
}

template <class S, class T>
static void process_kernel_loop(S* stg)
{
  overrideBinID = -1;
  const int binID = getBinID();
  Bin<T>* bin = stg->getBin(binID);
  const int numPrims = bin->getNumPrims();
  const int tid = getTID();
  const int numThreads = getNumThreads();
  if (getGID() == 0) stg->hasPrims = false;
  for (int i = tid; i < numPrims; i += numThreads) {
    T prim = bin->fetchPrimAtomic();
    prim.launchIdx = i;
    stg->process(prim);
  }
}

template <class F>
static void run_serial(int numBlocks, int numThreads, F kernel)
{
  blockDim_x = numThreads;
  for (int b = 0; b < numBlocks; ++b) {
    blockIdx_x = b;
    for (threadIdx_x = 0; threadIdx_x < numThreads; ++threadIdx_x) kernel();
  }
}
template <class F>
static void run_parallel(int numBlocks, int numThreads, unsigned numCPUThreads, F kernel)
{
  blockDim_x = numThreads;
  if (numCPUThreads <= 1) { run_serial(numBlocks, numThreads, kernel); return; }
  std::vector<std::thread> cpuThreads;
  int blocksPerThread = (int)ceil(numBlocks / (float)numCPUThreads);
  for (unsigned t = 0; t < numCPUThreads; ++t) {
    cpuThreads.push_back(std::thread([&, t]() {
      int lastBlock = std::min(numBlocks, (int)(t + 1) * blocksPerThread);
      for (int curBlock = t * blocksPerThread; curBlock < lastBlock; ++curBlock) {
        blockIdx_x = curBlock;
        for (threadIdx_x = 0; threadIdx_x < numThreads; ++threadIdx_x) kernel();
      }
    }));
  }
  for (auto& th : cpuThreads) th.join();
}

// ---------------------------------------------------------------- pipe methods
static unsigned g_cpu_threads = 1;
static size_t g_zbytes = 0;
static long long g_levels = 0;
static int g_max_levels = 64;  // the split limit of 20 ends the loop far earlier

void ReyesPipe::allocate(ConstantState& h_constState, MutableState& h_mutableState,
                         piko_patch* inputData, int count)
{
  constState_ = &h_constState;
  mutableState_ = &h_mutableState;
  count_ = count;
  std::map<void*, StageFloor*> stgMap;
  g_split = &split; g_dice = &dice; g_shade = &shade;
  d_split = &split; stgMap[&split] = d_split;
  d_dice = &dice;   stgMap[&dice] = d_dice;
  d_shade = &shade; stgMap[&shade] = d_shade;
  pikoScreen.allocate(constState_);
  d_pikoScreen = &pikoScreen;
  stgMap[&pikoScreen] = d_pikoScreen;
  shade.outPort[0] = &pikoScreen;
  h_input.allocate();
  h_input.copyData(inputData, count);
  d_mutableState = (MutableState*) malloc(std::max(sizeof(MutableState), g_zbytes));
  d_input = &h_input;
  split.allocate(constState_, d_mutableState, stgMap, false);
  dice.allocate(constState_, d_mutableState, stgMap, false);
  shade.allocate(constState_, d_mutableState, stgMap, false);
  for (int i = 0; i < 5; ++i) split.outPortTypes[i] = dice.outPortTypes[i] = shade.outPortTypes[i] = 0;
}

void ReyesPipe::prepare()
{
  memcpy(d_mutableState, mutableState_, std::max(sizeof(MutableState), g_zbytes));
  constState = *constState_;
}

void ReyesPipe::run_single()
{
  int count = count_;
  int numBlocks = (count / 512) + ((count % 512 == 0) ? 0 : 1);
  run_serial(numBlocks, 512, [&]() { kernel0(d_input, d_split); });
  int numBins_split = split.getNumBins();
  int hasPrims_split;
  g_levels = 0;
  do {
    run_parallel(numBins_split, 1, g_cpu_threads,
                 [&]() { process_kernel_loop<SplitStage, piko_patch>(d_split); });
    hasPrims_split = d_split->hasPrims;
    ++g_levels;
  } while (hasPrims_split && g_levels < g_max_levels);
  int numBins_dice = dice.getNumBins();
  run_parallel(numBins_dice, 1, g_cpu_threads,
               [&]() { process_kernel_loop<DiceStage, piko_patch>(d_dice); });
  int numBins_shade = shade.getNumBins();
  run_parallel(numBins_shade, 1, g_cpu_threads,
               [&]() { process_kernel_loop<ShadeStage, piko_upoly>(d_shade); });
}

void ReyesPipe::destroy()
{
  h_input.free();
  split.free();
  dice.free();
  shade.free();
  pikoScreen.free();
  std::free(pikoScreen.h_data_);
  std::free(d_mutableState);
}

template <class S>
static int grow_bins(S& stg)
{
  int grown = 0;
  for (int i = 0; i < stg.numBins_; ++i) {
    auto& b = stg.h_bins_[i];
    if (b.tail_ > b.maxPrims_) {
      int need = b.tail_;
      b.free();
      b.maxPrims_ = need + 64;
      b.allocate();
      ++grown;
    }
  }
  for (int i = 0; i < stg.numBins_; ++i) {
    auto& b = stg.h_bins_[i];
    b.head_ = b.tail_ = b.numPrims_ = 0;
  }
  stg.hasPrims = false;
  return grown;
}

// ---------------------------------------------------------------- C API
struct RefReyes {
  ReyesPipe* pipe = nullptr;
  ConstantState cs;
  std::vector<float> zhost;
  std::vector<piko_patch> input;
  int W = 0, H = 0;
};
static RefReyes* g_ref = nullptr;

extern "C" int piko_ref_reyes_destroy()
{
  if (!g_ref) return 0;
  g_ref->pipe->destroy();
  delete g_ref->pipe;
  delete g_ref;
  g_ref = nullptr;
  return 0;
}

// cps: 16 float4 control points per patch; vp: column-major view-projection.
// Patches are numbered as loadPatchBuffer numbers them (reyesPipe/main.cpp:276-303).
extern "C" int piko_ref_reyes_create(int W, int H, const float* cps, int count, const float* vp)
{
  if (W <= 0 || H <= 0 || count < 0) return -1;
  piko_ref_reyes_destroy();
  g_ref = new RefReyes();
  g_ref->W = W; g_ref->H = H;
  memset(&g_ref->cs, 0, sizeof(ConstantState));
  g_ref->cs.screenSizeX = W;
  g_ref->cs.screenSizeY = H;
  g_ref->cs.halfW = 0.5f * (float)W;
  g_ref->cs.halfH = 0.5f * (float)H;
  memcpy(g_ref->cs.viewProjMatrix, vp, 16 * sizeof(float));
  g_zbytes = (size_t)W * H * sizeof(float);
  g_ref->zhost.assign(std::max(sizeof(MutableState), g_zbytes) / sizeof(float), 1.0f);
  g_ref->input.resize(std::max(count, 1));
  for (int i = 0; i < count; ++i) {
    piko_patch& p = g_ref->input[i];
    memset(&p, 0, sizeof(p));
    for (int j = 0; j < 16; ++j)
      p.CP[j] = gencvec4f(cps[64 * i + 4 * j + 0], cps[64 * i + 4 * j + 1], cps[64 * i + 4 * j + 2], cps[64 * i + 4 * j + 3]);
    p.numSplits = 0;
    p.id = i;
    p.bbmin.x = 99999.0f; p.bbmin.y = 99999.0f;
    p.bbmax.x = -99999.0f; p.bbmax.y = -99999.0f;
  }
  g_ref->pipe = new ReyesPipe();
  g_ref->pipe->allocate(g_ref->cs, *(MutableState*)g_ref->zhost.data(), g_ref->input.data(), count);
  g_cpu_threads = 1;
  std::fill(g_ref->zhost.begin(), g_ref->zhost.end(), 1.0f);
  g_ref->pipe->prepare();
  g_ref->pipe->run_single();
  int grown = grow_bins(*g_split) + grow_bins(*g_dice) + grow_bins(*g_shade);
  for (int i = 0; i < W * H; ++i) g_ref->pipe->pikoScreen.h_data_[i] = 0xff663313;
  g_leaves = 0; g_upolys = 0; g_emitted = 0;
  return grown;
}

extern "C" long long piko_ref_reyes_frame(int cpu_threads, int record_leaves)
{
  if (!g_ref) return -1;
  g_cpu_threads = cpu_threads < 1 ? 1 : (unsigned)cpu_threads;
  g_record_leaves = record_leaves != 0;
  g_leaf_rec.clear();
  timespec a, b;
  clock_gettime(CLOCK_MONOTONIC, &a);
  std::fill(g_ref->zhost.begin(), g_ref->zhost.end(), 1.0f);
  g_ref->pipe->prepare();
  g_ref->pipe->run_single();
  clock_gettime(CLOCK_MONOTONIC, &b);
  g_record_leaves = false;
  return (long long)(b.tv_sec - a.tv_sec) * 1000000000LL + (b.tv_nsec - a.tv_nsec);
}

extern "C" int piko_ref_reyes_read(unsigned* fb, float* depth)
{
  if (!g_ref) return -1;
  size_t n = (size_t)g_ref->W * g_ref->H;
  if (fb) memcpy(fb, g_ref->pipe->pikoScreen.getData(), n * sizeof(unsigned));
  if (depth) memcpy(depth, g_ref->pipe->d_mutableState->zBuffer, n * sizeof(float));
  return 0;
}

// counters: [0] leaves sent to Dice, [1] micropolygons, [2] Pixels emitted,
// [3] split levels of the last frame; reset zeroes them.
extern "C" int piko_ref_reyes_counters(long long* out, int reset)
{
  out[0] = g_leaves.load(); out[1] = g_upolys.load(); out[2] = g_emitted.load(); out[3] = g_levels;
  if (reset) { g_leaves = 0; g_upolys = 0; g_emitted = 0; }
  return 0;
}

// leaves recorded by the last frame run with record_leaves: id, numSplits, nu,
// nv per leaf in the order Split emitted them.
extern "C" long long piko_ref_reyes_leaves(int* out, long long cap)
{
  long long n = (long long)g_leaf_rec.size() / 4;
  for (long long i = 0; i < n && i < cap; ++i)
    for (int k = 0; k < 4; ++k) out[4 * i + k] = g_leaf_rec[4 * i + k];
  return n;
}
