// An allocation-free way to render one raster frame.
//
// Some programs that would embed this library must not allocate device memory
// while they run: a host application (an engine, a compositor, a training job)
// that reserves all device memory up front in its own pool and gives plug-ins
// none of their own, so a cudaMalloc from the plug-in would fail or fragment
// that pool; or a real-time loop that cannot afford the device-wide
// synchronisation that cudaMalloc/cudaFree may imply.  The regular entry
// points allocate bin queues on first use and grow them on overflow, so those
// callers cannot use them.  piko_raster_frame_noalloc draws one frame of the
// binned raster pipeline with all of its working memory taken from a
// fixed-size array in the library's own device memory; the caller passes
// device pointers for the inputs and the outputs.
//
// The working memory is one file-scope __device__ array, so every GPU that
// loads the library holds it (about 23.5 MB) for the life of the process, and
// every call shares it: calls that may run at the same time on the GPU (on
// different streams, or from different host threads) overwrite each other's
// working memory and must be serialised by the caller.
#include <mutex>

#include "runtime_internal.h"

namespace piko {
cudaError_t launch_raster_frame(const RasterFrameArgs& a, int raster_ctas, cudaStream_t st, cudaEvent_t* ev);
cudaError_t raster_tiles_occupancy(int tile, int* blocks_per_sm);
}  // namespace piko

namespace {

// limits of the allocation-free path
constexpr uint32_t kNaMaxTris = 1u << 16;       // triangles per frame
constexpr uint32_t kNaMaxPixels = 1u << 20;     // width * height
constexpr uint32_t kNaTile = 16;
constexpr uint32_t kNaMaxTiles = 5120;          // 16x16 tiles of any W x H <= 2^20 pixels, sides <= 16384
constexpr uint32_t kNaMaxList = 1u << 20;       // (triangle, tile) queue entries
constexpr uint32_t kNaMaxSegs = 1u << 16;       // 128-tile segments of large triangles
constexpr uint32_t kNaMaxBig = 1u << 13;        // large triangles (more than 32 tiles in their box)

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// layout of the arena (byte offsets)
constexpr size_t kOffScene = 0;
constexpr size_t kOffCtr = align256(kOffScene + sizeof(RasterSceneDev));
constexpr size_t kOffSetup = align256(kOffCtr + sizeof(FrameCounters));
constexpr size_t kOffLargeSeg = align256(kOffSetup + sizeof(TriSetup) * kNaMaxTris);
constexpr size_t kOffLargeWalk = align256(kOffLargeSeg + sizeof(uint2) * kNaMaxSegs);
constexpr size_t kOffCnt = align256(kOffLargeWalk + sizeof(WalkTri) * kNaMaxBig);
constexpr size_t kOffOff = align256(kOffCnt + sizeof(uint32_t) * kNaMaxTiles);
constexpr size_t kOffHeavy = align256(kOffOff + sizeof(uint32_t) * (kNaMaxTiles + 1));
constexpr size_t kOffFlags = align256(kOffHeavy + sizeof(uint32_t) * kNaMaxTiles);
constexpr uint32_t kNaScanBlocks = (kNaMaxTiles + kScanTile - 1) / kScanTile;
constexpr size_t kOffList = align256(kOffFlags + sizeof(unsigned long long) * kNaScanBlocks);
constexpr size_t kOffPairTl = align256(kOffList + sizeof(uint32_t) * kNaMaxList);
constexpr size_t kOffPairG = align256(kOffPairTl + sizeof(unsigned long long) * kNaMaxList);
constexpr size_t kArenaBytes = align256(kOffPairG + sizeof(uint32_t) * kNaMaxList);
static_assert(kArenaBytes < (24u << 20), "the documented arena size");

}  // namespace

// The working memory of piko_raster_frame_noalloc.  In host code this name is
// only a stand-in for the symbol; its device address comes from
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_arena[kArenaBytes];

namespace {

std::mutex g_na_mutex;
void* g_na_base[64] = {};   // device address of the arena, per device ordinal
int g_na_ctas[64] = {};

cudaError_t arena_for_device(int dev, unsigned char** base, int* ctas)
{
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_base[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_arena);
    if (e != cudaSuccess) return e;
    int sms = 0, per_sm = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) return e;
    if ((e = raster_tiles_occupancy((int)kNaTile, &per_sm))) return e;
    g_na_base[dev] = p;
    g_na_ctas[dev] = sms * (per_sm > 0 ? per_sm : 1);
  }
  *base = (unsigned char*)g_na_base[dev];
  *ctas = g_na_ctas[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" piko_status piko_raster_frame_noalloc(const float* d_xyz, const uint32_t* d_icol, int count, int width,
                                                 int height, uint32_t* d_rgba, float* d_depth, void* stream)
{
  if (count < 0 || (count > 0 && (!d_xyz || !d_icol)) || !d_rgba || !d_depth) return PIKO_ERR_INVALID;
  if (width < 32 || height < 32 || width > 16384 || height > 16384) return PIKO_ERR_INVALID;
  if ((uint32_t)count > kNaMaxTris || (uint64_t)width * (uint64_t)height > kNaMaxPixels) return PIKO_ERR_LIMIT;
  int tiles_x = 0, tiles_y = 0;
  const uint32_t n_tiles = (uint32_t)tiles_for(width, height, (int)kNaTile, &tiles_x, &tiles_y);
  if (n_tiles > kNaMaxTiles) return PIKO_ERR_LIMIT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PIKO_ERR_NO_DEVICE;
  unsigned char* base = nullptr;
  int ctas = 0;
  if (arena_for_device(dev, &base, &ctas) != cudaSuccess) return PIKO_ERR_CUDA;
  cudaStream_t st = (cudaStream_t)stream;

  RasterSceneDev sd;
  scene_dev_geometry(sd, width, height, count, (int)kNaTile);
  sd.input_kind = kInputWtri;
  sd.wtri_xyz = d_xyz; sd.wtri_icol = d_icol;
  sd.fb = d_rgba; sd.depth = d_depth;

  // the arena keeps the previous call's contents: zero what must start at zero
  if (cudaMemcpyAsync(base + kOffScene, &sd, sizeof(sd), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemsetAsync(base + kOffCtr, 0, sizeof(FrameCounters), st) != cudaSuccess ||
      cudaMemsetAsync(base + kOffCnt, 0, sizeof(uint32_t) * n_tiles, st) != cudaSuccess ||
      cudaMemsetAsync(base + kOffFlags, 0, sizeof(unsigned long long) * kNaScanBlocks, st) != cudaSuccess)
    return PIKO_ERR_CUDA;

  RasterFrameArgs a;
  memset(&a, 0, sizeof(a));
  a.scenes = reinterpret_cast<const RasterSceneDev*>(base + kOffScene);
  a.n_scenes = 1;
  a.tile = (int)kNaTile;
  a.n_tris_total = (uint32_t)count;
  a.n_tiles_total = n_tiles;
  a.setup = reinterpret_cast<TriSetup*>(base + kOffSetup);
  a.tile_cnt = reinterpret_cast<uint32_t*>(base + kOffCnt);
  a.tile_off = reinterpret_cast<uint32_t*>(base + kOffOff);
  a.tile_list = reinterpret_cast<uint32_t*>(base + kOffList);
  a.pair_tl = reinterpret_cast<unsigned long long*>(base + kOffPairTl);
  a.pair_g = reinterpret_cast<uint32_t*>(base + kOffPairG);
  a.list_cap = kNaMaxList;
  a.heavy = reinterpret_cast<uint32_t*>(base + kOffHeavy);
  a.heavy_cap = kNaMaxTiles;
  a.heavy_threshold = heavy_threshold((int)kNaTile);
  a.large_seg = reinterpret_cast<uint2*>(base + kOffLargeSeg);
  a.seg_cap = kNaMaxSegs;
  a.large_walk = reinterpret_cast<WalkTri*>(base + kOffLargeWalk);
  a.big_cap = kNaMaxBig;
  a.scan_flags = reinterpret_cast<unsigned long long*>(base + kOffFlags);
  a.ctr = reinterpret_cast<FrameCounters*>(base + kOffCtr);
  if (launch_raster_frame(a, ctas, st, nullptr) != cudaSuccess) return PIKO_ERR_CUDA;

  // the queue cannot grow here, so the call waits for the frame and reports
  // an overflow instead of re-rendering
  FrameCounters c;
  if (cudaMemcpyAsync(&c, base + kOffCtr, sizeof(c), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return PIKO_ERR_CUDA;
  if (c.status & kStatusScanTimeout) return PIKO_ERR_TIMEOUT;
  if (c.status & kStatusListOverflow) return PIKO_ERR_QUEUE_OVERFLOW;
  return PIKO_OK;
}
