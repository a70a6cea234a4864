// Device-side data layout and scalar helpers shared by the raster and Reyes
// kernels of piko-public_b200.
//
// Arithmetic pinning.  Every kernel file is compiled with --fmad=false and the
// default IEEE division and square root, so each float expression below is the
// sequence of individually rounded operations the reference's CPU backend
// performs (g++ on x86-64, SSE, no contraction).  The conversions the
// reference gets from x86 instructions are spelled out explicitly:
//   (int)f       -> cvt_i32_x86  (cvttss2si: INT_MIN for NaN / out of range)
//   (unsigned)f  -> cvt_u32_x86  (64-bit cvttss2si, low 32 bits kept)
// and the 28.4 fixed-point edge functions use wrapping int32 arithmetic, as the
// reference's int expressions do on the CPU.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace piko {

// --------------------------------------------------------------- constants
constexpr int kVsBin = 32;          // VertexShaderStage bin size (vertexShader.pikostage:18)
constexpr int kVsChunk = 512;       // ids per VS-bin chunk, assignBin (vertexShader.pikostage:27)
constexpr int kRefBinLg2 = 3;       // RasterStage bin size 8 (raster.pikostage:14)
constexpr int kRefBin = 1 << kRefBinLg2;
constexpr int kGuard = 225 << 4;    // guard band (rasterMacros.h:37)
constexpr uint32_t kClearColor = 0xff663313u;  // PikoScreen initial colour (stage.h:83-85)

// tile scan: threads per block and tile counts per thread (scan_tiles)
constexpr int kScanThreads = 256;
constexpr int kScanItems = 2;
constexpr int kScanTile = kScanThreads * kScanItems;

// 8x8 raster queue: short lists (at most kQueueMax entries, so a group's
// entries fit one warp) are handed out kLightGroup tiles per pop
constexpr int kLightGroup = 4;
constexpr uint32_t kQueueMax = 32 / kLightGroup;

// 16/32-px tiles: a heavy tile's list is cut into at most kMaxTileChunks
// chunks of at least `chunk` entries (different warps rasterize them; the last
// one merges their per-pixel keys, so the merge reads a bounded number of
// chunk key buffers).  8x8 tiles use chunks of exactly `chunk` entries.
constexpr uint32_t kMaxTileChunks = 32;
__host__ __device__ __forceinline__ uint32_t tile_chunk_entries(uint32_t cnt, uint32_t chunk, bool t8)
{
  if (t8) return chunk;
  const uint32_t c = (cnt + kMaxTileChunks - 1) / kMaxTileChunks;
  return c > chunk ? c : chunk;
}
__host__ __device__ __forceinline__ uint32_t tile_chunks(uint32_t cnt, uint32_t chunk, bool t8)
{
  const uint32_t c = tile_chunk_entries(cnt, chunk, t8);
  return (cnt + c - 1) / c;
}

// frame status bits (the C ABI maps them to piko_status)
constexpr uint32_t kStatusListOverflow = 1u << 0;
constexpr uint32_t kStatusScanTimeout = 1u << 1;
constexpr uint32_t kStatusUpolyOverflow = 1u << 2;
constexpr uint32_t kStatusPatchOverflow = 1u << 3;
constexpr uint32_t kStatusDepthNeverSettles = 1u << 4;
constexpr uint32_t kStatusBarrierTimeout = 1u << 5;

// ------------------------------------------------- programmatic dependent launch
// A kernel launched with programmatic stream serialisation may start while the
// previous kernel of its stream still runs; pdl_wait() blocks until that
// kernel has completed and its memory is visible, so a kernel that calls it
// before touching global memory behaves exactly as if launched normally (the
// instruction does nothing for a normal launch).  pdl_trigger() lets the next
// such kernel be scheduled once every CTA of this one has started.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// --------------------------------------------------------------- scalar helpers
__device__ __forceinline__ int32_t cvt_i32_x86(float f)
{
  return (f >= -2147483648.0f && f < 2147483648.0f) ? __float2int_rz(f) : INT32_MIN;
}
__device__ __forceinline__ uint32_t cvt_u32_x86(float f)
{
  // |f| < 2^31: the 32-bit truncation has the same low 32 bits as the 64-bit one
  if (fabsf(f) < 2147483648.0f) return (uint32_t)__float2int_rz(f);
  return (f > -9223372036854775808.0f && f < 9223372036854775808.0f) ? (uint32_t)__float2ll_rz(f) : 0u;
}
__device__ __forceinline__ int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
__device__ __forceinline__ int32_t wsub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
__device__ __forceinline__ int32_t wmul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }
__device__ __forceinline__ int32_t wshl(int32_t a, int s) { return (int32_t)((uint32_t)a << s); }
// n / d and n % d for any 32-bit n and d >= 1, given m = 0xffffffff / d: the
// high product is the quotient or one less, fixed by one comparison.
__host__ __device__ __forceinline__ uint32_t divmod_magic(uint32_t d) { return 0xffffffffu / d; }
__device__ __forceinline__ uint32_t fast_divmod(uint32_t n, uint32_t d, uint32_t m, uint32_t& r)
{
  uint32_t q = __umulhi(n, m);
  r = n - q * d;
  if (r >= d) { ++q; r -= d; }
  return q;
}
// std::min / std::max on the CPU (piko/math.h:24-52): NaN handling differs from fminf
__device__ __forceinline__ float std_minf(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float std_maxf(float a, float b) { return (a < b) ? b : a; }

// --------------------------------------------------------------- scenes
// kInputWtriWorld: the raster_wtri payload of the pipe built without
// VTX_PRETRANSFORM (world positions the vertex stage transforms; no colours)
enum : int { kInputSoA = 0, kInputWtri = 1, kInputWtriWorld = 2 };

// One raster scene as the kernels see it.  All device pointers are owned by the
// scene object of the runtime.
struct RasterSceneDev {
  // geometry
  int W, H;
  int nBx, nBy;          // reference 8x8 bin grid (W/8, H/8; floor)
  int nVS;               // VertexShaderStage bins ((W/32)*(H/32))
  int N;                 // triangles
  // submission order constants: C = ceil(N / 512) chunks over nVS bins,
  // C / nVS and C % nVS, the bin of the last chunk, the empty ids of the last chunk
  uint32_t vs_m;         // divmod_magic(nVS)
  uint32_t vs_q, vs_rem, vs_last, vs_deficit, vs_chunks;
  int input_kind;
  int light_mode;
  int tiles_x, tiles_y;  // tile grid of this scene (tile size from RasterFrameArgs)
  uint32_t tiles_x_m;    // divmod_magic(tiles_x)
  uint32_t tile_base;    // first global tile id
  uint32_t tri_base;     // first global triangle-setup slot
  float halfW, halfH;
  float vp[16];
  float light[3];
  float eye[3];
  // inputs (SoA float4 [3][N] per attribute; or the pre-transformed payload)
  const float4* pos;
  const float4* nrm;
  const float* pos3;     // non-null: positions and normals are float3 [3][N] (pos / nrm unused)
  const float* nrm3;
  const float4* col;
  const float2* uv;      // textured variant only ([3][N])
  const float* wtri_xyz; // [N][9] (screen, or world for kInputWtriWorld)
  const uint32_t* wtri_icol;  // [N][3]
  const uchar4* tex;     // [TH][TW], power-of-two sizes
  int tex_w, tex_h;
  // outputs
  uint32_t* fb;          // [H][W] RGBA8 (R in the low byte), row 0 = bottom
  float* depth;          // [H][W]
};

// The submission-order constants of a scene of N triangles and nVS bins.
__host__ __device__ inline void scene_vs_consts(RasterSceneDev& d)
{
  const uint32_t nvs = (uint32_t)d.nVS, n = (uint32_t)d.N;
  const uint32_t C = (n + kVsChunk - 1) / kVsChunk;
  d.vs_m = divmod_magic(nvs);
  d.vs_chunks = C;
  d.vs_q = C / nvs;
  d.vs_rem = C % nvs;
  d.vs_last = C ? (C - 1) % nvs : 0u;
  d.vs_deficit = C * kVsChunk - n;
}

// Per-triangle setup record written by the setup kernel, read by the binning,
// raster and resolve phases.  80 bytes, 16-byte aligned.
struct __align__(16) TriSetup {
  int32_t x[3], y[3];   // 28.4 fixed point
  float z[3];
  uint32_t c[3];        // ABGR vertex colours
  float inv;            // 1.0f / (float)barydenom
  uint32_t bxr, byr;    // clamped reference-bin range: lo | hi << 16
  int32_t hix, hiy;     // pixel bounding box high corner (28.4, rounded up to 16 px)
  uint32_t rank1;       // submission rank + 1 (0 = culled)
  uint32_t flags;       // bit 0: wrapping possible inside the bin range (no tile-level reject)
  uint32_t id;          // triangle index within its scene
};
static_assert(sizeof(TriSetup) == 80, "TriSetup layout");

constexpr uint32_t kTriRisk = 1u;

// Per-frame counters (zeroed before each frame).  The heavy-tile queue and the
// large-triangle queue each reserve slots and work-item ranges with one 64-bit
// atomic, so that slot order and item order agree and an item's slot can be
// found by a search over the slots' first items.
constexpr uint32_t kPairParts = 128;
struct FrameCounters {
  uint32_t status;
  uint32_t scan_ticket;
  uint32_t work_next;
  uint32_t list_total;
  uint32_t kept;
  uint32_t cov_count;
  unsigned long long covered;
  unsigned long long risk;
  unsigned long long heavy_acc;  // heavy tiles << 32 | 8x8 list chunks
  unsigned long long large_acc;  // large triangles << 32 | their box-tile segments
  // The count passes record their (triangle, tile) pairs in kPairParts
  // partitions of list_cap / kPairParts slots each (a warp takes partition
  // (its global warp index) mod kPairParts), so that slot reservations spread
  // over kPairParts counters instead of queueing on one address.
  uint32_t pair_part_max;        // largest partition fill asked for (past its capacity: overflow)
  uint32_t pad[3];
  uint32_t pair_part[kPairParts];
};

// A triangle's box-tile walk: its 28.4 vertices, reference bin range, first
// tile and tiles per row (with the divide-by-tw magic), global setup slot and
// scene tile base, and for 8x8 tiles the reference's trivial-reject value of
// each edge at the first bin with its change per bin in x and y (wrapping
// int32, so equal to evaluating each bin directly).  Large triangles keep
// theirs in memory for the segment walk (112 bytes, 16-byte aligned).
struct __align__(16) WalkTri {
  int32_t x[3], y[3];
  int32_t bx1, bx2, by1, by2;
  int32_t tx1, ty1, tw;
  uint32_t tw_m;          // divmod_magic(tw)
  uint32_t gidx;
  uint32_t tile_base;
  int32_t tiles_x;
  uint32_t flags;
  int32_t tr0[3], trx[3], try_[3];
};
static_assert(sizeof(WalkTri) == 112, "WalkTri layout");

struct RasterFrameArgs {
  const RasterSceneDev* scenes;
  int n_scenes;
  int tile;                 // tile edge in pixels: 8, 16 or 32
  uint32_t n_tris_total;    // sum of N
  uint32_t n_tiles_total;
  TriSetup* setup;          // [n_tris_total]; written only for triangles that reach a bin (rank1 != 0)
  uint32_t* tile_cnt;       // [n_tiles_total]
  uint32_t* tile_off;       // [n_tiles_total + 1]
  uint32_t* tile_list;      // [list_cap]
  uint32_t list_cap;
  uint32_t* heavy;          // [heavy_cap] tiles served first (8x8: tiles split into chunks)
  uint32_t heavy_threshold; // 16/32-px tiles: list entries above which a tile is heavy
  uint32_t heavy_cap;
  // one record per (triangle, tile) pair, written by the count passes: the
  // tile | the pair's index in the tile's list << 32 (the old value of the
  // tile's counter), and the triangle's setup slot; [list_cap] each (pairs
  // and list entries are the same set, so one capacity bounds both)
  unsigned long long* pair_tl;
  uint32_t* pair_g;
  uint2* large_seg;         // [seg_cap] (large triangle, segment index) of every box-tile segment of a large triangle
  uint32_t seg_cap;
  WalkTri* large_walk;      // [big_cap] walk record of each large triangle, written by raster_setup
  uint32_t big_cap;
  // Heavy tiles (8x8: lists longer than queue_min; 16/32 px: longer than
  // heavy_threshold) are split into chunks (tile_chunk_entries) that different
  // warps rasterize.  Each chunk leaves its per-pixel keys (tile * tile of
  // them) in chunk_keys; the warp that completes a tile's last chunk takes the
  // per-pixel minimum over the tile's chunks and resolves the tile.  Without
  // chunk buffers (chunk_base null) heavy tiles are rasterized whole, first.
  uint32_t chunk;
  uint32_t queue_min;       // 8x8 tiles with more entries than this are queued as chunks
  uint32_t* chunk_base;     // [heavy_cap] first chunk of heavy tile h (ascending in h)
  uint32_t* chunk_heavy;    // [chunk_cap] the heavy tile (index h) of each chunk
  uint32_t* hdone;          // [heavy_cap] chunks finished
  unsigned long long* chunk_keys;  // [chunk_cap][tile * tile]
  uint32_t chunk_cap;
  unsigned long long* scan_flags;  // per scan block, epoch-tagged
  uint32_t epoch;
  FrameCounters* ctr;
  // coverage dump (parity tests): one (triangle id, pixel index) record per
  // covered sample, appended in any order; counted in ctr->cov_count
  uint32_t* cov_tri;
  uint32_t* cov_pix;
  uint32_t cov_cap;
};

}  // namespace piko
