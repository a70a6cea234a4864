// TEST INFRASTRUCTURE — part of the oracle, never part of the product path.
//
// Builds the reference's own binned rasterizer (RasterPipe: VertexShaderStage ->
// RasterStage -> PikoScreen) for the CPU exactly as `pikoc --target=CPU --opt`
// would: the stage code is the reference's, compiled in place from its source
// tree; this file supplies only what pikoc would have generated, which cannot be
// produced here because pikoc needs clang/LLVM 3.2:
//   * emit routing            pikoc/src/pikoc.cpp:69-194
//   * kernel0..kernel2 bodies pikoc/src/pikoc.cpp:196-318
//   * allocate/prepare/run_single/destroy and the std::thread block runner
//                             pikoc/src/Backend/CPUBackend.cpp:272-571
//
// Deliberate deviations from the generated code:
//   1. run() is never used (it ends in glutMainLoop); callers use
//      create -> frame -> read.
//   2. The number of CPU threads of the Process runner is a parameter: 1 gives
//      the deterministic parity run, 64 is what the reference generates.
//   3. MutableState::zBuffer is a fixed 1024x768 array (piko/builtinTypes.h:37);
//      the depth buffer block is allocated with max(sizeof(MutableState), W*H*4)
//      bytes so that larger framebuffers index past the declared bound into
//      owned memory, and prepare() copies W*H floats.
//   4. Bins are fixed-capacity rings that silently wrap (internal/datatypes.h:89,
//      piko/stage.h:281-288).  After allocate() a probe frame measures each
//      bin's fill and any bin that would wrap is re-allocated large enough, so a
//      parity frame never loses primitives.
//   5. Two observation hooks live in the generated emit routing of the drain
//      stage: a counter of emitted Pixels and, for coverage dumps, a record of
//      the emitted pixel positions.
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

// The bins' fill counters and capacities are private members of the reference's
// data structures; the capacity probe (deviation 4) needs to read and resize them.
#define private public
#define protected public
#include "rasterPipe.h"
#undef private
#undef protected

thread_local int threadIdx_x = 0;
thread_local int blockIdx_x = 0;
int blockDim_x = 0;

// ---------------------------------------------------------------- observation
static std::atomic<long long> g_emitted(0);
static bool g_record = false;
static std::vector<int> g_record_xy;

// ---------------------------------------------------------------- emit routing
void __emitSpecializationAssignBinVertexShaderStage__(raster_stri p, void* nextStg, int outPortType)
{
  ((RasterStage*) nextStg)->assignBin(p);
}
void __emitSpecializationProcessVertexShaderStage__(raster_stri p, void* nextStg, int outPortType)
{
  ((RasterStage*) nextStg)->process(p);
}
void VertexShaderStage::emit(raster_stri p, int outPortNum)
{
  __emitSpecializationAssignBinVertexShaderStage__(p, d_outPort_[0], outPortTypes[0]);
}
void __emitSpecializationAssignBinRasterStage__(Pixel p, void* nextStg, int outPortType)
{
  g_emitted.fetch_add(1, std::memory_order_relaxed);
  if (g_record) { g_record_xy.push_back((int)p.pos.x); g_record_xy.push_back((int)p.pos.y); }
  ((PikoScreen*) nextStg)->assignBin(p);
}
void RasterStage::emit(Pixel p, int outPortNum)
{
  __emitSpecializationAssignBinRasterStage__(p, d_outPort_[0], outPortTypes[0]);
}

// ---------------------------------------------------------------- kernels
static void kernel0(PikoArray<raster_wtri>* input, VertexShaderStage* d_vertexShader)
{
  const int gid = getGID();
  if (gid >= input->getNumPrims()) return;
  d_vertexShader->assignBin((*input)[gid]);
}

template <class S, class T>
static void process_kernel(S* stg)
{
  overrideBinID = -1;
  const int binID = getBinID();
  Bin<T>* bin = stg->getBin(binID);
  const int numPrims = bin->getNumPrims();
  const int tid = getTID();
  const int numThreads = getNumThreads();
  if (getGID() == 0) stg->hasPrims = false;
  for (int i = tid; i < numPrims; i += numThreads) {
    T prim = bin->fetchPrim();
    prim.launchIdx = i;
    stg->process(prim);
  }
  piko::BinSynchronize();
  if (tid == 0) bin->updatePrimCount(-numPrims);
}

// Serial runner (AssignBin kernels) and the parallel std::thread runner that the
// CPU backend generates for Process kernels (CPUBackend.cpp:522-571).
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
// RasterPipe keeps its stages as implicitly private members; allocate() (a
// member) publishes them for the capacity probe and the bin queries.
static VertexShaderStage* g_vs = nullptr;
static RasterStage* g_rs = nullptr;

void RasterPipe::allocate(ConstantState& h_constState, MutableState& h_mutableState,
                          raster_wtri* inputData, int count)
{
  constState_ = &h_constState;
  mutableState_ = &h_mutableState;
  count_ = count;
  std::map<void*, StageFloor*> stgMap;
  g_vs = &vertexShader;
  g_rs = &raster;
  d_vertexShader = &vertexShader; stgMap[&vertexShader] = d_vertexShader;
  d_raster = &raster;             stgMap[&raster] = d_raster;
  pikoScreen.allocate(constState_);
  d_pikoScreen = &pikoScreen;
  stgMap[&pikoScreen] = d_pikoScreen;
  raster.outPort[0] = &pikoScreen;
  h_input.allocate();
  h_input.copyData(inputData, count);
  d_mutableState = (MutableState*) malloc(std::max(sizeof(MutableState), g_zbytes));
  d_input = &h_input;
  vertexShader.allocate(constState_, d_mutableState, stgMap, false);
  for (int i = 0; i < 5; ++i) vertexShader.outPortTypes[i] = 0;
  raster.allocate(constState_, d_mutableState, stgMap, false);
  for (int i = 0; i < 5; ++i) raster.outPortTypes[i] = 0;
}

void RasterPipe::prepare()
{
  memcpy(d_mutableState, mutableState_, std::max(sizeof(MutableState), g_zbytes));
  constState = *constState_;
}

void RasterPipe::run_single()
{
  int count = count_;
  int numBlocks = (count / 512) + ((count % 512 == 0) ? 0 : 1);
  run_serial(numBlocks, 512, [&]() { kernel0(d_input, d_vertexShader); });
  int numBins_vertexShader = vertexShader.getNumBins();
  run_parallel(numBins_vertexShader, 1, g_cpu_threads,
               [&]() { process_kernel<VertexShaderStage, raster_wtri>(d_vertexShader); });
  int numBins_raster = raster.getNumBins();
  run_parallel(numBins_raster, 1, g_cpu_threads,
               [&]() { process_kernel<RasterStage, raster_stri>(d_raster); });
}

void RasterPipe::destroy()
{
  h_input.free();
  vertexShader.free();
  raster.free();
  pikoScreen.free();
  std::free(pikoScreen.h_data_);
  std::free(d_mutableState);
}

// ---------------------------------------------------------------- capacity probe
template <class S>
static int grow_bins(S& stg)
{
  int grown = 0;
  for (int i = 0; i < stg.numBins_; ++i) {
    auto& b = stg.h_bins_[i];
    int need = b.tail_;
    if (need > b.maxPrims_) {
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
struct RefRaster {
  RasterPipe* pipe = nullptr;
  ConstantState cs;
  std::vector<float> zhost;  // caller-side MutableState (depth reset to 1.0f per frame)
  std::vector<raster_wtri> input;
  int W = 0, H = 0;
  int grown = 0;
};
static RefRaster* g_ref = nullptr;

static void reset_depth(float value)
{
  std::fill(g_ref->zhost.begin(), g_ref->zhost.end(), value);
}

extern "C" int piko_ref_raster_destroy()
{
  if (!g_ref) return 0;
  g_ref->pipe->destroy();
  delete g_ref->pipe;
  delete g_ref;
  g_ref = nullptr;
  return 0;
}

// xyz: 9 floats per triangle (screen-space x,y and depth z of v0,v1,v2, i.e. the
// pre-transformed raster_wtri::worldPos0..2); icol: 3 packed ABGR colours.
// Triangle ids are their indices, as loadTriangleBuffer assigns them
// (pikoc/samples/rasterPipelineFixPt/main.cpp:396).
static int create_common(int W, int H, int count, const float* xyz, const unsigned* icol, const float* vp);

#ifdef VTX_PRETRANSFORM
extern "C" int piko_ref_raster_create(int W, int H, const float* xyz, const unsigned* icol, int count)
{
  return create_common(W, H, count, xyz, icol, nullptr);
}
#else
// The pipe built without VTX_PRETRANSFORM: xyz holds world positions, which
// the vertex stage transforms with constState.viewProjMatrix
// (vertexShader.pikostage:56-80); vp is that matrix (column-major).  The
// reference sets no vertex colours in this mode (its normals are zero here).
extern "C" int piko_ref_raster_create_world(int W, int H, const float* xyz, const float* vp, int count)
{
  return create_common(W, H, count, xyz, nullptr, vp);
}
#endif

static int create_common(int W, int H, int count, const float* xyz, const unsigned* icol, const float* vp)
{
  if (W <= 0 || H <= 0 || count < 0) return -1;
  piko_ref_raster_destroy();
  g_ref = new RefRaster();
  g_ref->W = W; g_ref->H = H;
  memset(&g_ref->cs, 0, sizeof(ConstantState));
  g_ref->cs.screenSizeX = W;
  g_ref->cs.screenSizeY = H;
  g_ref->cs.halfW = 0.5f * (float)W;
  g_ref->cs.halfH = 0.5f * (float)H;
  g_zbytes = (size_t)W * H * sizeof(float);
  size_t zcount = std::max(sizeof(MutableState), g_zbytes) / sizeof(float);
  g_ref->zhost.assign(zcount, 1.0f);
  g_ref->input.resize(std::max(count, 1));
  for (int i = 0; i < count; ++i) {
    raster_wtri& t = g_ref->input[i];
    t.binID = 0; t.launchIdx = 0; t.id = i;
    t.worldPos0 = gencvec3f(xyz[9 * i + 0], xyz[9 * i + 1], xyz[9 * i + 2]);
    t.worldPos1 = gencvec3f(xyz[9 * i + 3], xyz[9 * i + 4], xyz[9 * i + 5]);
    t.worldPos2 = gencvec3f(xyz[9 * i + 6], xyz[9 * i + 7], xyz[9 * i + 8]);
#ifdef VTX_PRETRANSFORM
    t.icol0 = icol[3 * i + 0]; t.icol1 = icol[3 * i + 1]; t.icol2 = icol[3 * i + 2];
#else
    (void)icol;
    t.normal0 = gencvec2f(0.0f, 0.0f); t.normal1 = t.normal0; t.normal2 = t.normal0;
#endif
  }
  if (vp) memcpy(g_ref->cs.viewProjMatrix, vp, 16 * sizeof(float));
  g_ref->pipe = new RasterPipe();
  g_ref->pipe->allocate(g_ref->cs, *(MutableState*)g_ref->zhost.data(), g_ref->input.data(), count);
  // probe frame (deviation 4): measure bin fills with one thread, grow, reset
  g_cpu_threads = 1;
  reset_depth(1.0f);
  g_ref->pipe->prepare();
  g_ref->pipe->run_single();
  g_ref->grown = grow_bins(*g_vs) + grow_bins(*g_rs);
  for (int i = 0; i < W * H; ++i) g_ref->pipe->pikoScreen.h_data_[i] = 0xff663313;
  g_emitted = 0;
  return g_ref->grown;
}

// One frame as doPerfTest times it (main.cpp:210-222, minus the GL projection
// matrix): resetDepthBuffer + prepare + run_single.  Returns the elapsed ns.
extern "C" long long piko_ref_raster_frame(int cpu_threads)
{
  if (!g_ref) return -1;
  g_cpu_threads = cpu_threads < 1 ? 1 : (unsigned)cpu_threads;
  timespec a, b;
  clock_gettime(CLOCK_MONOTONIC, &a);
  reset_depth(1.0f);
  g_ref->pipe->prepare();
  g_ref->pipe->run_single();
  clock_gettime(CLOCK_MONOTONIC, &b);
  return (long long)(b.tv_sec - a.tv_sec) * 1000000000LL + (b.tv_nsec - a.tv_nsec);
}

// Framebuffer (pikoScreen.getData(), stage.h:108-117) and the depth buffer as
// the Process kernels left it.
extern "C" int piko_ref_raster_read(unsigned* fb, float* depth)
{
  if (!g_ref) return -1;
  size_t n = (size_t)g_ref->W * g_ref->H;
  if (fb) memcpy(fb, g_ref->pipe->pikoScreen.getData(), n * sizeof(unsigned));
  if (depth) memcpy(depth, g_ref->pipe->d_mutableState->zBuffer, n * sizeof(float));
  return 0;
}

extern "C" long long piko_ref_raster_emitted(int reset)
{
  long long v = g_emitted.load();
  if (reset) g_emitted.store(0);
  return v;
}

// Coverage of one triangle, observed through the reference's own Process code:
// the triangle is run alone with the depth buffer set to the largest signed
// integer bit pattern, so every covered sample passes the depth test once and
// is emitted.  Writes up to max_px (x,y) pairs; returns the number covered.
extern "C" int piko_ref_raster_coverage(int tri, int* xy, int max_px)
{
  if (!g_ref || tri < 0 || tri >= g_ref->pipe->count_) return -1;
  RasterPipe* p = g_ref->pipe;
  p->h_input.copyData(&g_ref->input[tri], 1);
  int saved = p->count_;
  p->count_ = 1;
  int bits = INT_MAX;
  float fbits;
  memcpy(&fbits, &bits, 4);
  reset_depth(fbits);
  g_cpu_threads = 1;
  g_record = true;
  g_record_xy.clear();
  p->prepare();
  p->run_single();
  g_record = false;
  p->count_ = saved;
  p->h_input.copyData(g_ref->input.data(), saved);
  int n = (int)g_record_xy.size() / 2;
  for (int i = 0; i < n && i < max_px; ++i) { xy[2 * i] = g_record_xy[2 * i]; xy[2 * i + 1] = g_record_xy[2 * i + 1]; }
  for (int i = 0; i < g_ref->W * g_ref->H; ++i) p->pikoScreen.h_data_[i] = 0xff663313;
  reset_depth(1.0f);
  return n;
}

extern "C" int piko_ref_raster_bins(int* nvs, int* nraster, int* cap_raster)
{
  if (!g_ref) return -1;
  *nvs = g_vs->getNumBins();
  *nraster = g_rs->getNumBins();
  *cap_raster = g_rs->h_bins_[0].maxPrims_;
  return 0;
}
