// Internal host-side types of libpiko_b200.so shared by runtime.cu and
// reyes_kernels.cu (not part of the C ABI).
#pragma once
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <vector>

#include "piko_device.cuh"
#include "../../include/piko_b200.h"

namespace piko {
int raster_scan_blocks(uint32_t n_tiles);
}
using namespace piko;

struct ReyesState;

struct piko_ctx {
  int device = 0;
  int sms = 0;
  bool time_kernels = false;
  cudaStream_t stream = nullptr;
  char err[512] = {0};
};

struct piko_pipe {
  piko_ctx* ctx = nullptr;
  int kind = 0;  // 1 raster, 2 reyes
  int tile = 16;
  int ctas_per_sm = 0;
  uint32_t chunk = 0;
  float split_threshold = 4.0f;
  int max_splits = 20;
  int dice_grid = 0;
  int samples_per_pixel = 1;
  uint32_t sample_seed = 0;
  int phong = 0;
};

enum { kPipeRaster = 1, kPipeReyes = 2 };

// Tile grid of a W x H framebuffer cut into T x T tiles; returns the tile count.
inline int tiles_for(int W, int H, int T, int* tx, int* ty)
{
  *tx = (W + T - 1) / T;
  *ty = (H + T - 1) / T;
  return *tx * *ty;
}

// The fields of a RasterSceneDev that follow from the framebuffer size, the
// triangle count and the tile edge T: the reference's 8x8 and 32x32 bin grids,
// the submission-order constants, the tile grid and the viewport halves.
// Every path that fills a RasterSceneDev starts from this (the rest is zero).
inline void scene_dev_geometry(RasterSceneDev& d, int W, int H, int N, int T)
{
  memset(&d, 0, sizeof(d));
  d.W = W; d.H = H;
  d.nBx = W / kRefBin; d.nBy = H / kRefBin;
  d.nVS = (W / kVsBin) * (H / kVsBin);
  d.N = N;
  scene_vs_consts(d);
  tiles_for(W, H, T, &d.tiles_x, &d.tiles_y);
  d.tiles_x_m = divmod_magic((uint32_t)d.tiles_x);
  d.halfW = 0.5f * (float)W;
  d.halfH = 0.5f * (float)H;
}

inline piko_status set_err(piko_ctx* ctx, piko_status st, const char* fmt, const char* detail = "")
{
  if (ctx) snprintf(ctx->err, sizeof(ctx->err), fmt, detail);
  return st;
}

#define CU(ctx, call)                                                                 \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      return set_err((ctx), e_ == cudaErrorMemoryAllocation ? PIKO_ERR_OOM : PIKO_ERR_CUDA, \
                     "%s", cudaGetErrorString(e_));                                   \
    }                                                                                 \
  } while (0)

template <class T>
inline cudaError_t dalloc(T** p, size_t count)
{
  *p = nullptr;
  if (count == 0) count = 1;
  return cudaMalloc((void**)p, count * sizeof(T));
}
template <class T>
inline void dfree(T*& p)
{
  if (p) cudaFree(p);
  p = nullptr;
}

// Frame scratch shared by every scene drawn in one launch sequence.
struct RasterScratch {
  TriSetup* setup = nullptr;
  uint32_t* tile_cnt = nullptr;
  uint32_t* tile_off = nullptr;
  uint32_t* tile_list = nullptr;
  unsigned long long* pair_tl = nullptr;  // count-pass pair records, [list_cap] each
  uint32_t* pair_g = nullptr;
  uint32_t* heavy = nullptr;
  uint2* large_seg = nullptr;   // large-triangle segment items
  uint32_t seg_cap = 0;
  WalkTri* large_walk = nullptr;  // walk records of the large triangles, [seg_cap]: each has a segment
  uint32_t* chunk_base = nullptr;           // first chunk per heavy tile
  uint32_t* hdone = nullptr;                // finished chunks per heavy tile
  unsigned long long* chunk_keys = nullptr; // tile * tile keys per chunk
  uint32_t* chunk_heavy = nullptr;          // heavy tile of each chunk
  uint32_t heavy_cap = 0, chunk_cap = 0;
  uint32_t chunk_stride = 0;                // keys per chunk (tile * tile)
  unsigned long long* scan_flags = nullptr;
  FrameCounters* ctr = nullptr;
  FrameCounters* h_ctr = nullptr;  // pinned
  RasterSceneDev* d_scenes = nullptr;
  RasterSceneDev* h_scenes = nullptr;  // pinned
  uint32_t tris_cap = 0, tiles_cap = 0, list_cap = 0, scan_cap = 0;
  int scenes_cap = 0;
  uint32_t cov_cap = 0;
  uint32_t* cov_tri = nullptr;
  uint32_t* cov_pix = nullptr;
  cudaEvent_t ev[5] = {};
  bool ev_made = false;

  void release()
  {
    dfree(setup); dfree(tile_cnt); dfree(tile_off); dfree(tile_list); dfree(pair_tl); dfree(pair_g);
    dfree(heavy); dfree(large_seg); dfree(large_walk); dfree(chunk_base); dfree(hdone); dfree(chunk_keys);
    dfree(chunk_heavy);
    dfree(scan_flags); dfree(ctr); dfree(d_scenes); dfree(cov_tri); dfree(cov_pix);
    if (h_ctr) cudaFreeHost(h_ctr);
    if (h_scenes) cudaFreeHost(h_scenes);
    h_ctr = nullptr; h_scenes = nullptr;
    if (ev_made) for (auto& e : ev) cudaEventDestroy(e);
    ev_made = false;
    tris_cap = tiles_cap = list_cap = scan_cap = heavy_cap = chunk_cap = seg_cap = chunk_stride = 0;
    scenes_cap = 0;
    cov_cap = 0;
  }

  // Heavy-tile queue.  16/32-px tiles: any tile may be heavy.  8x8 tiles: a
  // heavy tile has more than `queue_min` list entries, so at most
  // list_cap / (queue_min + 1) of them exist.  Heavy lists are cut into
  // chunks, each with T * T keys in chunk_keys; the key buffers start at an
  // estimate and grow after a frame reports that it needed more (regrow).
  cudaError_t ensure_heavy(uint32_t n_tiles, int T, uint32_t chunk, uint32_t queue_min)
  {
    const bool t8 = T == kRefBin;
    const uint32_t need_h = t8 ? std::min<uint32_t>(n_tiles, list_cap / (queue_min + 1) + 1) : n_tiles;
    cudaError_t e = cudaSuccess;
    if (need_h > heavy_cap || !chunk_base) {
      dfree(heavy); dfree(chunk_base); dfree(hdone);
      heavy_cap = 0;
      if ((e = dalloc(&heavy, need_h))) return e;
      if ((e = dalloc(&chunk_base, need_h))) return e;
      if ((e = dalloc(&hdone, need_h))) return e;
      heavy_cap = need_h;
    }
    const uint32_t stride = (uint32_t)(T * T);
    const uint32_t want = t8 ? need_h / 2 + list_cap / (4 * chunk) + 64 : list_cap / (8 * chunk) + 64;
    if (want > chunk_cap || stride != chunk_stride) {
      if ((e = grow_chunks(std::max(want, stride == chunk_stride ? chunk_cap : 0u), stride))) return e;
    }
    return cudaSuccess;
  }

  // The tile lists and the count passes' pair records (the same number of
  // entries) grow together.
  cudaError_t grow_list(uint32_t n)
  {
    dfree(tile_list); dfree(pair_tl); dfree(pair_g);
    list_cap = 0;
    cudaError_t e = dalloc(&tile_list, n);
    if (!e) e = dalloc(&pair_tl, n);
    if (!e) e = dalloc(&pair_g, n);
    if (!e) list_cap = n;
    return e;
  }

  cudaError_t grow_segs(uint32_t n)
  {
    dfree(large_seg);
    dfree(large_walk);
    seg_cap = 0;
    cudaError_t e = dalloc(&large_seg, n);
    if (!e) e = dalloc(&large_walk, n);
    if (!e) seg_cap = n;
    return e;
  }

  // key buffers of n chunks of `stride` keys each
  cudaError_t grow_chunks(uint32_t n, uint32_t stride)
  {
    dfree(chunk_keys);
    dfree(chunk_heavy);
    chunk_cap = 0;
    cudaError_t e = dalloc(&chunk_keys, (size_t)n * stride);
    if (!e) e = dalloc(&chunk_heavy, n);
    if (!e) { chunk_cap = n; chunk_stride = stride; }
    return e;
  }

  // After a frame whose counters report a queue overflow: grows what
  // overflowed (the tile lists and / or the chunk key buffers) so that the
  // frame can be drawn again.
  cudaError_t regrow(const FrameCounters& c)
  {
    cudaError_t e = cudaSuccess;
    // the lists hold every pair, and each pair partition its share
    const uint32_t need = std::max<uint32_t>(c.list_total, (uint32_t)std::min<unsigned long long>(
                                                               (unsigned long long)c.pair_part_max * kPairParts,
                                                               0xffffffffull));
    if (need > list_cap || c.pair_part_max > list_cap / kPairParts) {
      if ((e = grow_list(need + need / 4 + 1024))) return e;
    }
    const uint32_t chunks = (uint32_t)c.heavy_acc;
    if (chunk_base && chunks > chunk_cap) {
      if ((e = grow_chunks(chunks + chunks / 4 + 64, chunk_stride))) return e;
    }
    // every large triangle has at least one segment: seg_cap bounds both
    const uint32_t segs = std::max((uint32_t)c.large_acc, (uint32_t)(c.large_acc >> 32));
    if (segs > seg_cap) {
      if ((e = grow_segs(segs + segs / 4 + 1024))) return e;
    }
    return cudaSuccess;
  }

  cudaError_t ensure(uint32_t n_tris, uint32_t n_tiles, uint32_t list_need, int n_scenes)
  {
    cudaError_t e = cudaSuccess;
    if (n_tris > tris_cap) {
      dfree(setup);
      if ((e = dalloc(&setup, n_tris))) return e;
      // segment items of large triangles: an estimate, grown after an overflow
      if (n_tris / 8 + 1024 > seg_cap && (e = grow_segs(n_tris / 8 + 1024))) return e;
      tris_cap = n_tris;
    }
    if (n_tiles > tiles_cap) {
      dfree(tile_cnt); dfree(tile_off);
      if ((e = dalloc(&tile_cnt, n_tiles))) return e;
      if ((e = dalloc(&tile_off, (size_t)n_tiles + 1))) return e;
      tiles_cap = n_tiles;
    }
    uint32_t sb = (uint32_t)raster_scan_blocks(n_tiles);
    if (sb > scan_cap) {
      dfree(scan_flags);
      if ((e = dalloc(&scan_flags, sb))) return e;
      scan_cap = sb;
    }
    if (list_need > list_cap) {
      if ((e = grow_list(list_need))) return e;
    }
    if (!ctr) {
      if ((e = dalloc(&ctr, 1))) return e;
      if ((e = cudaMallocHost((void**)&h_ctr, sizeof(FrameCounters)))) return e;
      memset(h_ctr, 0, sizeof(FrameCounters));
    }
    if (n_scenes > scenes_cap) {
      dfree(d_scenes);
      if (h_scenes) cudaFreeHost(h_scenes);
      h_scenes = nullptr;
      if ((e = dalloc(&d_scenes, n_scenes))) return e;
      if ((e = cudaMallocHost((void**)&h_scenes, sizeof(RasterSceneDev) * n_scenes))) return e;
      scenes_cap = n_scenes;
    }
    if (!ev_made) {
      for (auto& ev_ : ev) if ((e = cudaEventCreate(&ev_))) return e;
      ev_made = true;
    }
    return cudaSuccess;
  }
};

struct piko_scene {
  piko_pipe* pipe = nullptr;
  int kind = 0;
  int W = 0, H = 0, N = 0;
  float4* pos = nullptr;
  float4* nrm = nullptr;
  float* pos3 = nullptr;   // packed scenes: float3 positions and normals instead
  float* nrm3 = nullptr;
  int packed = 0;
  float4* col = nullptr;
  float2* uv = nullptr;
  uchar4* tex = nullptr;
  int tex_w = 0, tex_h = 0;
  float* wtri_xyz = nullptr;
  uint32_t* wtri_icol = nullptr;
  float4* patches = nullptr;
  uint32_t* fb = nullptr;
  float* depth = nullptr;
  piko_const_state state{};
  RasterScratch scr;
  cudaStream_t own_stream = nullptr;
  cudaStream_t last_stream = nullptr;
  bool pending = false;
  bool timed = false;
  uint64_t list_total_seen = 0;
  ReyesState* reyes = nullptr;
};

// Launch configuration of a raster launch sequence: tile edge, persistent
// CTAs per SM (0 = the kernel's occupancy) and list entries per chunk of the
// 8x8 tile queue (0 = kDefaultChunk).
struct TuneCfg {
  int tile = 8;
  int ctas_per_sm = 0;
  uint32_t chunk = 0;
  bool operator==(const TuneCfg& o) const { return tile == o.tile && ctas_per_sm == o.ctas_per_sm && chunk == o.chunk; }
};
inline TuneCfg pipe_cfg(const piko_pipe* p) { return TuneCfg{p->tile, p->ctas_per_sm, p->chunk}; }

// Scene-size buckets of the tuner: 4 resolution classes x 4 triangle classes.
constexpr int kTuneBuckets = 16;
int tune_bucket(int W, int H, int N);

struct piko_tuner {
  TuneCfg cfg[kTuneBuckets];
  float ms[kTuneBuckets] = {};
  bool tuned[kTuneBuckets] = {};
};

// Scenes of a batch that share one launch configuration: one launch sequence
// over all of them, on its own branch of the batch's stream fork.
struct BatchGroup {
  TuneCfg cfg;
  std::vector<piko_scene*> scenes;
  RasterScratch scr;
  cudaStream_t stream = nullptr;  // the branch (group 0 runs on the caller's stream)
  cudaEvent_t done = nullptr;
};

struct piko_batch {
  piko_ctx* ctx = nullptr;
  std::vector<piko_scene*> scenes;
  std::vector<BatchGroup*> groups;
  cudaEvent_t fork = nullptr;
  cudaStream_t last_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaStream_t graph_stream = nullptr;
  bool pending = false;
};
piko_status batch_make(piko_ctx* ctx, piko_scene* const* scenes, int n, const TuneCfg* cfgs, piko_batch** out);

// Reyes device path (reyes_kernels.cu)
piko_status piko_reyes_run(piko_scene* s, cudaStream_t st, bool timed);
piko_status piko_reyes_finish(piko_scene* s);
piko_status piko_reyes_stats(piko_scene* s, piko_frame_stats* out);
void piko_reyes_release(piko_scene* s);
// Shared Reyes work buffers: frames on one stream may use one set.
ReyesState* reyes_buffers_new();
void reyes_buffers_free(ReyesState* b);
void reyes_borrow_buffers(piko_scene* s, ReyesState* b);

// One draw of a launch sequence: a resident mesh seen with one camera state,
// rendered into one framebuffer / depth buffer.
struct RasterDraw {
  const piko_scene* mesh;
  const piko_const_state* state;
  uint32_t* fb;
  float* depth;
};
// chunk: list entries per chunk of the 8x8 tile queue (kDefaultChunk when 0);
// lists longer than kQueueMin entries are queued as chunks
constexpr uint32_t kDefaultChunk = 32;
constexpr uint32_t kQueueMin = 8;
piko_status enqueue_raster_draws(piko_ctx* ctx, const RasterDraw* draws, int n, RasterScratch& scr, int T, int ctas,
                                 cudaStream_t st, bool timed, bool coverage, uint32_t chunk = 0);
// One launch sequence over resident scenes drawn with their own camera states.
piko_status enqueue_raster(piko_ctx* ctx, piko_scene* const* scenes, int n, RasterScratch& scr, const TuneCfg& cfg,
                           cudaStream_t st, bool timed, bool coverage);
int raster_ctas(piko_ctx* ctx, int tile, int ctas_per_sm);
uint32_t heavy_threshold(int tile);
