// Binned raster pipeline for sm_100a: the reference's RasterPipe
// (VertexShaderStage -> RasterStage -> PikoScreen, pikoc/samples/rasterPipelineFixPt)
// as five kernels per frame, over one scene or a batch of scenes:
//
//   raster_setup    one thread per triangle.  Vertex shading + triangle setup
//                   (R1: main.cpp:299-400 moved on device; R3: vertexShader.pikostage:36-109)
//                   from coalesced SoA loads, then AssignBin (R4,
//                   raster.pikostage:40-117) as a warp-cooperative tile walk: one
//                   counter atomic per (triangle, tile) pair (shared by the
//                   warp's lanes with the same tile at 16/32-px tiles), whose old
//                   value is the pair's index in the tile's list, and a pair
//                   record.  Triangles with more than 32 box tiles are queued
//                   as 128-tile segments for
//   raster_large_count, which walks them the same way over the whole grid.
//   scan_tiles      exclusive prefix sum of the tile counts (single pass,
//                   decoupled look-back) -> per-tile list offsets.  Tiles with
//                   long lists are queued: 16/32-px tiles whole or as chunks,
//                   8x8 tiles as chunks of a fixed number of list entries.
//   raster_scatter  a streaming pass over the pair records: each becomes its
//                   list entry at its tile's offset plus its index (no walk, no
//                   atomics): the compaction.
//   raster_tiles /  persistent CTAs (Schedule).  The 8x8 kernel (one reference
//   raster_frag8    bin per tile) gives each warp a tile or a chunk of one: the
//                   warp tests every list entry against the tile's 64 pixels,
//                   two per lane, and keeps each pixel's winning fragment key in
//                   registers.  The 16/32-px kernel walks each entry's candidate
//                   pixels triangle-parallel with shared-memory key atomics.
//                   Coverage is the reference's 28.4 edge test with its 8x8-bin
//                   trivial reject/accept (R6, raster.pikostage:124-242); the z
//                   test, the shading of each pixel's winner and the composite
//                   are fused in (R7/R8), and every pixel is written once.
//
// Order independence.  The reference's depth test is an atomicMin on the float
// bits compared as signed ints, with ties passing (raster.pikostage:274-285).
// Run sequentially that leaves, per pixel, the minimum depth bits and the
// colour of the LAST fragment, in submission order, that has those bits.  So
// each fragment carries its triangle's submission rank and a pixel keeps the
// fragment with the smallest (depth bits, -rank): the result equals the
// sequential one whatever order the tile lists come in, and no list is sorted.
#include <atomic>

#include "piko_device.cuh"

namespace piko {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kLargeTiles = 32;  // box tiles above which a triangle's walk is spread over the grid
constexpr uint32_t kLargeSeg = 128;   // box tiles per work item of the large-triangle walk

// ------------------------------------------------------------------ helpers
template <class S>
__device__ __forceinline__ int find_base(const S* sc, int n, uint32_t g, bool by_tile)
{
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    uint32_t b = by_tile ? sc[mid].tile_base : sc[mid].tri_base;
    if (b <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// The scenes' first triangles or tiles in shared memory (batches of up to
// CAP scenes; larger ones search the scene records), so that finding a
// triangle's or a tile's scene is a shared-memory search.
constexpr int kSceneTable = 1024;
template <int CAP>
__device__ __forceinline__ void load_scene_table(const RasterFrameArgs& a, uint32_t* tb, bool by_tile)
{
  if (a.n_scenes > CAP) return;
  for (int i = threadIdx.x; i < a.n_scenes; i += blockDim.x) tb[i] = by_tile ? a.scenes[i].tile_base : a.scenes[i].tri_base;
}
template <int CAP>
__device__ __forceinline__ int scene_of(const RasterFrameArgs& a, const uint32_t* tb, uint32_t x, bool by_tile)
{
  if (a.n_scenes > CAP) return find_base(a.scenes, a.n_scenes, x, by_tile);
  int lo = 0, hi = a.n_scenes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tb[mid] <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}
__device__ __forceinline__ int scene_of_tile(const RasterFrameArgs& a, const uint32_t* tb, uint32_t tile)
{
  return scene_of<kSceneTable>(a, tb, tile, true);
}

// The last index i in [0, n) with base[i] <= x, for an ascending base with
// base[0] <= x; the whole warp searches, 32 probes per step.
__device__ __forceinline__ uint32_t warp_search(const uint32_t* base, uint32_t n, uint32_t x, int lane)
{
  uint32_t lo = 0, hi = n;  // answer in [lo, hi)
  while (hi - lo > 1) {
    const uint32_t step = (hi - lo + 31) / 32;
    const uint32_t probe = lo + (uint32_t)lane * step;
    const bool ok = probe < hi && __ldg(&base[probe]) <= x;
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    lo += (uint32_t)(31 - __clz(m)) * step;
    hi = min(hi, lo + step);
  }
  return lo;
}

// Rank of triangle `id` in the order the one-thread CPU backend submits
// triangles to the raster bins: VS bins in index order (kernel1 blocks), and in
// VS bin b the ids with (id/512) % nVS == b ascending (vertexShader.pikostage:25-29).
__device__ __forceinline__ uint32_t submission_rank(uint32_t id, const RasterSceneDev& S)
{
  const uint32_t c = id / kVsChunk;
  uint32_t b;
  const uint32_t cq = fast_divmod(c, (uint32_t)S.nVS, S.vs_m, b);
  const uint32_t start = kVsChunk * (b * S.vs_q + min(b, S.vs_rem)) - (S.vs_last < b ? S.vs_deficit : 0u);
  return start + cq * kVsChunk + (id % kVsChunk);
}

// (depth bits as signed ints ascending, submission rank descending) as one
// unsigned 64-bit key: the smallest key is the sequential depth test's winner.
__device__ __forceinline__ unsigned long long frag_key(float z, uint32_t rank1)
{
  return ((unsigned long long)((uint32_t)__float_as_int(z) ^ 0x80000000u) << 32) | (uint32_t)(~rank1);
}
constexpr unsigned long long kInitKey = ((unsigned long long)(0x3f800000u ^ 0x80000000u) << 32) | 0xffffffffull;

__device__ __forceinline__ TriSetup load_setup(const TriSetup* p)
{
  TriSetup r;
  const uint4* src = reinterpret_cast<const uint4*>(p);
  uint4* dst = reinterpret_cast<uint4*>(&r);
#pragma unroll
  for (int k = 0; k < 5; ++k) dst[k] = __ldg(src + k);
  return r;
}

struct F3 { float x, y, z; };

__device__ __forceinline__ float sat1(float v) { return v > 1.0f ? 1.0f : (v < 0.0f ? 0.0f : v); }

// computeLightingHost + toABGRHost (main.cpp:317-334)
__device__ __forceinline__ uint32_t light_abgr(F3 n, F3 l, F3 m)
{
  float d = n.x * l.x + n.y * l.y + n.z * l.z;
  d = d < 0.0f ? 0.0f : d;
  float r = sat1(d * m.x + 0.15f);
  float g = sat1(d * m.y + 0.15f);
  float b = sat1(d * m.z + 0.30f);
  return 0xff000000u | (cvt_u32_x86(b * 255.0f) << 16) | (cvt_u32_x86(g * 255.0f) << 8) | cvt_u32_x86(r * 255.0f);
}

// E_i(X, Y) = (Y - y_i) * dx_i - (X - x_i) * dy_i  (wrapping int32)
__device__ __forceinline__ int32_t edge_at(int32_t X, int32_t Y, int32_t xi, int32_t yi, int32_t dx, int32_t dy)
{
  return wsub(wmul(wsub(Y, yi), dx), wmul(wsub(X, xi), dy));
}

// Per-lane staging for the warp-cooperative tile walk.

// Conservative tile-level trivial reject (exact int64 arithmetic): the tile,
// clipped to the triangle's bin range, can hold an assigned reference bin only
// if every edge function is >= 0 at the tile corner that maximises it.  Only
// used for triangles whose edge values cannot wrap inside the bin range.
__device__ __forceinline__ bool tile_may_cover(const WalkTri& w, int tx, int ty, int T)
{
  if (T == kRefBin) {
    // the tile is one reference bin: the reference's own trivial reject at the
    // bin corner (raster.pikostage:77-105), stepped from bin (tx1, ty1)
    const int32_t k = tx - w.tx1, m = ty - w.ty1;
    int32_t tr = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) tr |= wadd(wadd(w.tr0[i], wmul(k, w.trx[i])), wmul(m, w.try_[i]));
    return tr >= 0;
  }
  if (w.flags & kTriRisk) return true;
  long long X0 = (long long)max(tx * T, w.bx1 * kRefBin) * 16;
  long long X1 = (long long)min((tx + 1) * T, (w.bx2 + 1) * kRefBin) * 16;
  long long Y0 = (long long)max(ty * T, w.by1 * kRefBin) * 16;
  long long Y1 = (long long)min((ty + 1) * T, (w.by2 + 1) * kRefBin) * 16;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    int j = i == 2 ? 0 : i + 1;
    long long dx = (long long)w.x[j] - w.x[i], dy = (long long)w.y[j] - w.y[i];
    long long X = dy < 0 ? X1 : X0;
    long long Y = dx > 0 ? Y1 : Y0;
    long long e = (Y - w.y[i]) * dx - (X - w.x[i]) * dy;
    if (e < 0) return false;
  }
  return true;
}

// Counts the pairs of R rounds held by the warp's lanes (key = global tile, or
// ~0 for none): one atomicAdd per pair on its tile's counter (per group of
// lanes with the same tile at 16/32-px tiles), whose old value gives the
// pair's index in the tile's list, and one reservation per warp for the
// pair records, which the scatter pass turns into list entries without
// walking again.  Every lane of the warp calls this (ballots).  Records past
// the list capacity are dropped; the scan reports the overflow (the pair
// total equals the list total) and the frame is drawn again.
template <int R>
__device__ __forceinline__ void count_pairs(const RasterFrameArgs& a, const uint32_t (&key)[R],
                                            const uint32_t (&gidx)[R], int lane)
{
  uint32_t local[R];
  if (a.tile == kRefBin) {
#pragma unroll
    for (int q = 0; q < R; ++q) local[q] = key[q] != 0xffffffffu ? atomicAdd(&a.tile_cnt[key[q]], 1u) : 0u;
  } else {
    // 16/32-px tiles: lanes of a round with the same tile share one counter
    // atomic (the group's lowest lane adds the group's size; a lane's index is
    // the old count plus its rank in the group).  (At 8x8 tiles, where fewer
    // of a warp's pairs share a tile, the match costs more than it saves.)
    const unsigned lt0 = (1u << lane) - 1u;
    unsigned grp[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      grp[q] = __match_any_sync(kFull, key[q]);
      local[q] = 0u;
      if (key[q] != 0xffffffffu && (grp[q] & lt0) == 0u)
        local[q] = atomicAdd(&a.tile_cnt[key[q]], (uint32_t)__popc(grp[q]));
    }
#pragma unroll
    for (int q = 0; q < R; ++q)
      local[q] = __shfl_sync(kFull, local[q], __ffs(grp[q]) - 1) + (uint32_t)__popc(grp[q] & lt0);
  }
  unsigned m[R];
  uint32_t n = 0;
#pragma unroll
  for (int q = 0; q < R; ++q) {
    m[q] = __ballot_sync(kFull, key[q] != 0xffffffffu);
    n += (uint32_t)__popc(m[q]);
  }
  if (n == 0) return;
  const uint32_t part = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) & (kPairParts - 1u);
  const uint32_t part_cap = a.list_cap / kPairParts;
  uint32_t base = 0;
  if (lane == 0) {
    base = atomicAdd(&a.ctr->pair_part[part], n);
    if (base + n > part_cap) {
      // the host grows the lists so that every partition fits, and draws again
      atomicMax(&a.ctr->pair_part_max, base + n);
      atomicOr(&a.ctr->status, kStatusListOverflow);
    }
  }
  base = __shfl_sync(kFull, base, 0);
  const unsigned lt = (1u << lane) - 1u;
  const size_t at = (size_t)part * part_cap;
#pragma unroll
  for (int q = 0; q < R; ++q) {
    if (key[q] != 0xffffffffu) {
      const uint32_t slot = base + (uint32_t)__popc(m[q] & lt);
      if (slot < part_cap) {
        a.pair_tl[at + slot] = (unsigned long long)key[q] | ((unsigned long long)local[q] << 32);
        a.pair_g[at + slot] = gidx[q];
      }
    }
    base += (uint32_t)__popc(m[q]);
  }
}

// A frame whose pairs overran the list buffers is drawn again with larger
// ones; its tile lists have entries that no pair filled (a pair counted in
// tile_cnt but past list_cap has no record), so the fragment kernels must not
// read them.  The status is final once the scan has run.
__device__ __forceinline__ bool list_overflowed(const RasterFrameArgs& a)
{
  return (*(volatile uint32_t*)&a.ctr->status & kStatusListOverflow) != 0;
}

// Walks every (triangle, tile) pair of a warp's 32 triangles with all 32 lanes
// busy: pair j belongs to the lane whose inclusive tile-count prefix first
// exceeds j; the pairs that pass the tile-level reject are counted and
// recorded, four rounds of 32 at a time so that four counter atomics per lane
// are in flight together.
__device__ __forceinline__ void walk_tiles(const RasterFrameArgs& a, const WalkTri* wt, uint32_t ntiles)
{
  const int lane = threadIdx.x & 31;
  uint32_t incl = ntiles;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t v = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += v;
  }
  const uint32_t excl = incl - ntiles;
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  constexpr int kRounds = 4;
  for (uint32_t base = 0; base < total; base += 32 * kRounds) {
    uint32_t key[kRounds], gidx[kRounds];
#pragma unroll
    for (int q = 0; q < kRounds; ++q) {
      const uint32_t j = base + (uint32_t)q * 32u + (uint32_t)lane;
      int lo = 0, hi = 31;
#pragma unroll
      for (int st = 0; st < 5; ++st) {
        const int mid = (lo + hi) >> 1;
        const uint32_t v = __shfl_sync(kFull, incl, mid);
        if (v > j) hi = mid; else lo = mid + 1;
      }
      const int owner = lo;
      const uint32_t oexcl = __shfl_sync(kFull, excl, owner);
      key[q] = 0xffffffffu;
      gidx[q] = 0;
      if (j < total) {
        const WalkTri& w = wt[owner];
        uint32_t lx;
        const uint32_t ly = fast_divmod(j - oexcl, (uint32_t)w.tw, w.tw_m, lx);
        const int tx = w.tx1 + (int)lx, ty = w.ty1 + (int)ly;
        if (tile_may_cover(w, tx, ty, a.tile)) {
          key[q] = w.tile_base + (uint32_t)(ty * w.tiles_x + tx);
          gidx[q] = w.gidx;
        }
      }
    }
    count_pairs<kRounds>(a, key, gidx, lane);
  }
}

__device__ __forceinline__ void fill_walk(const RasterFrameArgs& a, const RasterSceneDev& S, const TriSetup& r,
                                          uint32_t g, WalkTri& w, uint32_t& ntiles)
{
  const int tsh = __ffs(a.tile) - 1 - kRefBinLg2;   // tile edge = 8 << tsh
  for (int k = 0; k < 3; ++k) { w.x[k] = r.x[k]; w.y[k] = r.y[k]; }
  w.bx1 = (int)(r.bxr & 0xffff); w.bx2 = (int)(r.bxr >> 16);
  w.by1 = (int)(r.byr & 0xffff); w.by2 = (int)(r.byr >> 16);
  w.tx1 = w.bx1 >> tsh;
  w.ty1 = w.by1 >> tsh;
  const int tx2 = w.bx2 >> tsh, ty2 = w.by2 >> tsh;
  w.tw = tx2 - w.tx1 + 1;
  w.tw_m = divmod_magic((uint32_t)w.tw);
  w.gidx = g;
  w.tile_base = S.tile_base;
  w.tiles_x = S.tiles_x;
  w.flags = r.flags;
  ntiles = (uint32_t)w.tw * (uint32_t)(ty2 - w.ty1 + 1);
  if (tsh == 0) {
    const int32_t BX = w.tx1 * 128, BY = w.ty1 * 128;   // bin corner, 28.4
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int j = i == 2 ? 0 : i + 1;
      const int32_t dx = wsub(r.x[j], r.x[i]), dy = wsub(r.y[j], r.y[i]);
      int32_t off = dy < 0 ? -wshl(dy, 7) : 0;
      off = wadd(off, dx >= 0 ? wshl(dx, 7) : 0);
      w.tr0[i] = wadd(off, wsub(wmul(wsub(BY, r.y[i]), dx), wmul(wsub(BX, r.x[i]), dy)));
      w.trx[i] = -wshl(dy, 7);
      w.try_[i] = wshl(dx, 7);
    }
  }
}

// Vertex attribute i (slot-major index k * N + id): float4, or float3 with w
// 0 in a packed scene (w is never read).
__device__ __forceinline__ float4 load_attr3(const float4* a4, const float* a3, size_t i)
{
  if (a3) return make_float4(__ldg(&a3[3 * i]), __ldg(&a3[3 * i + 1]), __ldg(&a3[3 * i + 2]), 0.0f);
  return __ldg(&a4[i]);
}

// ------------------------------------------------------------------ kernel 1
// 128-thread CTAs: one wave holds the scene's triangle blocks spread nearly
// evenly over the SMs.
constexpr int kSetupThreads = 128;
__global__ void __launch_bounds__(kSetupThreads) raster_setup(RasterFrameArgs a)
{
  pdl_trigger();
  __shared__ WalkTri s_walk[kSetupThreads];
  __shared__ unsigned s_kept[kSetupThreads / 32], s_risk[kSetupThreads / 32];
  __shared__ uint32_t s_tb[kSceneTable];
  load_scene_table<kSceneTable>(a, s_tb, false);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  unsigned nk = 0, nr = 0;
  // one wave of CTAs strides over blocks of kSetupThreads triangles
  for (uint32_t base = blockIdx.x * (uint32_t)kSetupThreads; base < a.n_tris_total;
       base += gridDim.x * (uint32_t)kSetupThreads) {
  const uint32_t g = base + threadIdx.x;
  uint32_t ntiles = 0;
  bool kept_flag = false, risk_flag = false;
  if (g < a.n_tris_total) {
    const int s = scene_of<kSceneTable>(a, s_tb, g, false);
    const RasterSceneDev& S = a.scenes[s];
    const uint32_t id = g - S.tri_base;
    float sx[3], sy[3], sz[3];
    uint32_t ic[3] = {0u, 0u, 0u};
    const bool soa = S.input_kind == kInputSoA;
    if (soa || S.input_kind == kInputWtriWorld) {
      // R1, main.cpp:299-308: vtransform, perspective divide, viewport.  The
      // per-vertex lighting follows the culls: a culled triangle's colours are
      // never read, so only kept triangles load normals and are lit.  World
      // raster_wtri input: the vertex stage's vtxTransform (rasterMacros.h:14-21,
      // matmultfloat4 and rcp_approx = 1.0f / w on the CPU) is the same float
      // sequence; that mode has no colours (left 0).
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        float4 p;
        if (soa) {
          p = load_attr3(S.pos, S.pos3, (size_t)k * S.N + id);
        } else {
          p.x = __ldg(&S.wtri_xyz[(size_t)id * 9 + 3 * k + 0]);
          p.y = __ldg(&S.wtri_xyz[(size_t)id * 9 + 3 * k + 1]);
          p.z = __ldg(&S.wtri_xyz[(size_t)id * 9 + 3 * k + 2]);
          p.w = 1.0f;
        }
        const float* m = S.vp;
        float tx = p.x * m[0] + p.y * m[4] + p.z * m[8] + m[12];
        float ty = p.x * m[1] + p.y * m[5] + p.z * m[9] + m[13];
        float tz = p.x * m[2] + p.y * m[6] + p.z * m[10] + m[14];
        float tw = p.x * m[3] + p.y * m[7] + p.z * m[11] + m[15];
        float onebyw = 1.0f / tw;
        sx[k] = (tx * onebyw + 1.0f) * S.halfW;
        sy[k] = (ty * onebyw + 1.0f) * S.halfH;
        sz[k] = (tz * onebyw);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        sx[k] = S.wtri_xyz[(size_t)id * 9 + 3 * k + 0];
        sy[k] = S.wtri_xyz[(size_t)id * 9 + 3 * k + 1];
        sz[k] = S.wtri_xyz[(size_t)id * 9 + 3 * k + 2];
        ic[k] = S.wtri_icol[(size_t)id * 3 + k];
      }
    }
    // R3: 28.4 quantisation by truncation and the three culls
    TriSetup r;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      r.x[k] = cvt_i32_x86(sx[k] * 16.0f);
      r.y[k] = cvt_i32_x86(sy[k] * 16.0f);
      r.z[k] = sz[k];
      r.c[k] = ic[k];
    }
    r.id = id;
    r.flags = 0;
    r.rank1 = 0;
    r.inv = 0.0f;
    r.bxr = r.byr = 0;
    r.hix = r.hiy = 0;
    bool keep = wsub(wmul(wsub(r.y[2], r.y[0]), wsub(r.x[1], r.x[0])),
                     wmul(wsub(r.x[2], r.x[0]), wsub(r.y[1], r.y[0]))) > 0;
    const int32_t Wf = cvt_i32_x86((float)S.W * 16.0f), Hf = cvt_i32_x86((float)S.H * 16.0f);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      keep = keep && !(r.x[k] < -kGuard || r.x[k] >= wadd(Wf, kGuard));
      keep = keep && !(r.y[k] < -kGuard || r.y[k] >= wadd(Hf, kGuard));
    }
    const int32_t loy0 = min(min(r.y[0], r.y[1]), r.y[2]);
    const int32_t hiy0 = max(max(r.y[0], r.y[1]), r.y[2]);
    keep = keep && !((wsub(loy0, 8) >> 4) == (wsub(hiy0, 8) >> 4));
    kept_flag = keep;
    if (keep && soa) {
      // R1, main.cpp:310-400: per-vertex Gouraud lighting with the normal
      // normalised by HOST::normalize; no colour array: the reference's fixed
      // material colour (main.cpp:380)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float4 n4 = load_attr3(S.nrm, S.nrm3, (size_t)k * S.N + id);
        const float4 c4 = S.col ? __ldg(&S.col[(size_t)k * S.N + id]) : make_float4(0.9f, 0.9f, 0.6f, 1.0f);
        float mag = sqrtf(n4.x * n4.x + n4.y * n4.y + n4.z * n4.z);
        F3 n = {n4.x / mag, n4.y / mag, n4.z / mag};
        F3 l;
        if (S.light_mode == 1) {
          const float4 p = load_attr3(S.pos, S.pos3, (size_t)k * S.N + id);
          l.x = S.eye[0] - p.x; l.y = S.eye[1] - p.y; l.z = S.eye[2] - p.z;
          float mm = sqrtf(l.x * l.x + l.y * l.y + l.z * l.z);
          if (mm != 0.0f) { float rr = 1.0f / mm; l.x = l.x * rr; l.y = l.y * rr; l.z = l.z * rr; }
        } else {
          l.x = S.light[0]; l.y = S.light[1]; l.z = S.light[2];
        }
        r.c[k] = light_abgr(n, l, F3{c4.x, c4.y, c4.z});
      }
    }
    if (keep) {
      // R4: pixel bounding box rounded to 16 px, reference bin range (8x8)
      const int32_t lox = min(min(r.x[0], r.x[1]), r.x[2]) & (int32_t)0xffffff00;
      const int32_t loy = loy0 & (int32_t)0xffffff00;
      const int32_t hix = wadd(max(max(r.x[0], r.x[1]), r.x[2]), 0xff) & (int32_t)0xffffff00;
      const int32_t hiy = wadd(hiy0, 0xff) & (int32_t)0xffffff00;
      const int bits = 4 + kRefBinLg2;
      int bx1 = max(0, lox >> bits), bx2 = min(hix >> bits, S.nBx - 1);
      int by1 = max(0, loy >> bits), by2 = min(hiy >> bits, S.nBy - 1);
      r.hix = hix; r.hiy = hiy;
      const int32_t x1mx0 = wsub(r.x[1], r.x[0]), y1my0 = wsub(r.y[1], r.y[0]);
      const int32_t x0mx2 = wsub(r.x[0], r.x[2]), y0my2 = wsub(r.y[0], r.y[2]);
      const int32_t barydenom = wadd(wmul(-y0my2, x1mx0), wmul(x0mx2, y1my0));
      r.inv = 1.0f / (float)barydenom;
      if (bx1 <= bx2 && by1 <= by2) {
        r.rank1 = submission_rank(id, S) + 1u;
        r.bxr = (uint32_t)bx1 | ((uint32_t)bx2 << 16);
        r.byr = (uint32_t)by1 | ((uint32_t)by2 << 16);
        // can any edge value the reference compares wrap inside the bin range?
        const long long X0 = (long long)bx1 * 128, X1 = (long long)(bx2 + 1) * 128;
        const long long Y0 = (long long)by1 * 128, Y1 = (long long)(by2 + 1) * 128;
        // |e(X, Y)| <= max|Y - y_i| * |dx| + max|X - x_i| * |dy| over the range
        // (a bound at least the largest corner value), plus the trivial-accept
        // offsets
        long long worst = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const int j = i == 2 ? 0 : i + 1;
          const long long dx = llabs((long long)r.x[j] - r.x[i]), dy = llabs((long long)r.y[j] - r.y[i]);
          const long long ax = max(llabs(X0 - r.x[i]), llabs(X1 - r.x[i]));
          const long long ay = max(llabs(Y0 - r.y[i]), llabs(Y1 - r.y[i]));
          worst = max(worst, ay * dx + ax * dy + 512 * (dx + dy));
        }
        if (worst >= 2147483647LL) r.flags |= kTriRisk;
        risk_flag = (r.flags & kTriRisk) != 0;
      }
    }
    // 80-byte record as five 16-byte stores, for the triangles that reach a
    // bin: only tile lists (and the winners they give) lead to a record
    if (r.rank1) {
      const uint4* src = reinterpret_cast<const uint4*>(&r);
      uint4* dst = reinterpret_cast<uint4*>(&a.setup[g]);
#pragma unroll
      for (int k = 0; k < 5; ++k) dst[k] = src[k];
      fill_walk(a, S, r, g, s_walk[threadIdx.x], ntiles);
    }
  }
  // Triangles with many tiles in their box go to raster_large, which walks
  // their box tiles in segments of kLargeSeg: one atomic per warp reserves
  // the warp's segment items.
  const bool is_big = ntiles > kLargeTiles;
  const unsigned big = __ballot_sync(kFull, is_big);
  if (big) {
    const uint32_t nseg = is_big ? (ntiles + kLargeSeg - 1) / kLargeSeg : 0u;
    uint32_t incl = nseg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    unsigned long long old = 0;
    if (lane == 31) old = atomicAdd(&a.ctr->large_acc, ((unsigned long long)__popc(big) << 32) | incl);
    old = __shfl_sync(kFull, old, 31);
    if (is_big) {
      // the triangle's walk record, then one (large triangle, segment) item
      // per segment; records or items past the capacities are reported (the
      // host grows the buffers and draws the frame again)
      const uint32_t bi = (uint32_t)(old >> 32) + (uint32_t)__popc(big & ((1u << lane) - 1u));
      const uint32_t first = (uint32_t)old + incl - nseg;
      if (bi < a.big_cap) {
        a.large_walk[bi] = s_walk[threadIdx.x];
        for (uint32_t k = 0; k < nseg; ++k) {
          if (first + k < a.seg_cap) a.large_seg[first + k] = make_uint2(bi, k);
          else { atomicOr(&a.ctr->status, kStatusListOverflow); break; }
        }
      } else {
        atomicOr(&a.ctr->status, kStatusListOverflow);
      }
      ntiles = 0;
    }
  }
  nk += __popc(__ballot_sync(kFull, kept_flag));
  nr += __popc(__ballot_sync(kFull, risk_flag));
  __syncwarp();
  walk_tiles(a, &s_walk[threadIdx.x & ~31], ntiles);
  __syncwarp();  // the warp's s_walk entries are rewritten by the next block
  }
  // frame counters: one atomic per CTA
  if (lane == 0) {
    s_kept[threadIdx.x >> 5] = nk;
    s_risk[threadIdx.x >> 5] = nr;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned k = 0, rr = 0;
#pragma unroll
    for (int w = 0; w < kSetupThreads / 32; ++w) { k += s_kept[w]; rr += s_risk[w]; }
    if (k) atomicAdd(&a.ctr->kept, k);
    if (rr) atomicAdd(&a.ctr->risk, (unsigned long long)rr);
  }
}

// ------------------------------------------------------------------ kernel 2
// Exclusive scan of tile_cnt (decoupled look-back).  Flags per block hold
// (epoch << 34) | (state << 32) | value, state 1 = aggregate, 2 = inclusive.

__global__ void __launch_bounds__(kScanThreads) scan_tiles(RasterFrameArgs a)
{
  pdl_wait();
  pdl_trigger();
  __shared__ uint32_t s_bid;
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t s_prefix;
  __shared__ unsigned long long s_heavy[kScanThreads / 32];   // per warp: (heavy tiles << 32) | chunks
  if (threadIdx.x == 0) s_bid = atomicAdd(&a.ctr->scan_ticket, 1u);
  __syncthreads();
  const uint32_t bid = s_bid;
  const uint32_t n = a.n_tiles_total;
  const uint32_t base = bid * kScanTile + threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = (base + i < n) ? a.tile_cnt[base + i] : 0u;
    sum += v[i];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  // Heavy tiles (lists longer than the threshold) and their chunks: counted
  // now, reserved below with one atomic per block while warp 0 looks back
  const bool t8 = a.tile == kRefBin;
  const bool chunked = a.chunk_base != nullptr;
  const uint32_t thr = t8 ? a.queue_min : a.heavy_threshold;
  uint32_t nh = 0, nc = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n && v[i] > thr) {
      ++nh;
      if (chunked) nc += tile_chunks(v[i], a.chunk, t8);
    }
  }
  uint32_t hi = nh, ci = nc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t th = __shfl_up_sync(kFull, hi, o), tc = __shfl_up_sync(kFull, ci, o);
    if (lane >= o) { hi += th; ci += tc; }
  }
  if (lane == 31) {
    s_warp[warp] = incl;
    s_heavy[warp] = ((unsigned long long)hi << 32) | ci;
  }
  __syncthreads();
  if (warp == 1 && lane == 0) {
    // the block's reservation; each warp's base replaces its count
    unsigned long long tot = 0;
#pragma unroll
    for (int w = 0; w < kScanThreads / 32; ++w) tot += s_heavy[w];
    unsigned long long run_h = tot ? atomicAdd(&a.ctr->heavy_acc, tot) : 0ull;
#pragma unroll
    for (int w = 0; w < kScanThreads / 32; ++w) {
      const unsigned long long cnt = s_heavy[w];
      s_heavy[w] = run_h;
      run_h += cnt;
    }
  }
  uint32_t warp_excl = 0, agg = 0;
#pragma unroll
  for (int w = 0; w < kScanThreads / 32; ++w) {
    if (w < warp) warp_excl += s_warp[w];
    agg += s_warp[w];
  }
  const unsigned long long ep = (unsigned long long)a.epoch << 34;
  if (warp == 0) {
    // Look-back by the whole warp: lane j reads the flag of block
    // (end - j), so 32 predecessors are examined per step.  The window is
    // summed once every lane up to the nearest inclusive prefix is published.
    uint32_t prefix = 0;
    if (bid == 0) {
      if (lane == 0) atomicExch(&a.scan_flags[0], ep | (2ull << 32) | agg);
    } else {
      if (lane == 0) atomicExch(&a.scan_flags[bid], ep | (1ull << 32) | agg);
      int end = (int)bid - 1;
      uint32_t spins = 0;
      for (;;) {
        const int idx = end - lane;
        uint32_t state = 2, val = 0;  // lanes before block 0 read as an inclusive 0
        if (idx >= 0) {
          const unsigned long long f = __ldcv(&a.scan_flags[idx]);
          state = (f >> 34) == a.epoch ? (uint32_t)(f >> 32) & 3u : 0u;
          val = (uint32_t)f;
        }
        const unsigned pending = __ballot_sync(kFull, state == 0);
        const unsigned inclusive = __ballot_sync(kFull, state == 2);
        const int first = inclusive ? __ffs(inclusive) - 1 : 31;
        const unsigned need = first == 31 ? kFull : ((2u << first) - 1u);
        if (pending & need) {
          if (++spins > (1u << 22)) {
            if (lane == 0) atomicOr(&a.ctr->status, kStatusScanTimeout);
            break;
          }
          __nanosleep(32);
          continue;
        }
        prefix += __reduce_add_sync(kFull, lane <= first ? val : 0u);
        if (inclusive) break;
        end -= 32;
      }
      if (lane == 0) atomicExch(&a.scan_flags[bid], ep | (2ull << 32) | (uint32_t)(prefix + agg));
    }
    if (lane == 0) s_prefix = prefix;
  }
  __syncthreads();
  uint32_t run = s_prefix + warp_excl + (incl - sum);
  // With chunk buffers a heavy list becomes tile_chunks(len) chunks; the
  // tile's first chunk and its finished-chunk counter are all the queue stores
  // per tile.
  const unsigned long long old = s_heavy[warp];
  uint32_t h = (uint32_t)(old >> 32) + hi - nh;
  uint32_t c = (uint32_t)old + ci - nc;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) {
      a.tile_off[base + i] = run;
      if (v[i] > thr) {
        if (h < a.heavy_cap) {
          a.heavy[h] = base + i;
          if (chunked) {
            a.chunk_base[h] = c;
            a.hdone[h] = 0;
            const uint32_t nch = tile_chunks(v[i], a.chunk, t8);
            for (uint32_t j = 0; j < nch && c + j < a.chunk_cap; ++j) a.chunk_heavy[c + j] = h;
            c += nch;
            // chunks past the key buffers are not rasterized: report it
            if (c > a.chunk_cap) atomicOr(&a.ctr->status, kStatusListOverflow);
          }
        } else {
          atomicOr(&a.ctr->status, kStatusListOverflow);
        }
        ++h;
      }
    }
    run += v[i];
  }
  if (base < n && base + kScanItems >= n) {
    // the thread holding the last element publishes the total
    a.tile_off[n] = run;
    a.ctr->list_total = run;
    if (run > a.list_cap) atomicOr(&a.ctr->status, kStatusListOverflow);
  }
}

// ------------------------------------------------------------------ kernel 3
// Large triangles (more than kLargeTiles tiles in their box): their box tiles
// are cut into segments of kLargeSeg, and a warp takes one segment at a time,
// its lanes striding over the segment's tiles (four per lane in flight), so a
// huge triangle spreads over many warps.  The pairs are counted and recorded
// like the small triangles' (count_pairs).
__device__ __forceinline__ void large_segment(const RasterFrameArgs& a, uint32_t it, int lane)
{
  const uint2 sg = a.large_seg[it];
  const uint32_t j0 = sg.y * kLargeSeg;
  const WalkTri w = a.large_walk[sg.x];
  const uint32_t g = w.gidx;
  const int tsh = __ffs(a.tile) - 1 - kRefBinLg2;   // tile edge = 8 << tsh
  const uint32_t ntiles = (uint32_t)w.tw * (uint32_t)((w.by2 >> tsh) - w.ty1 + 1);
  const uint32_t j1 = min(j0 + kLargeSeg, ntiles);
  for (uint32_t jb0 = j0; jb0 < j1; jb0 += 4 * 32) {   // warp-uniform trips
    uint32_t key[4], gidx[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t j = jb0 + (uint32_t)lane + (uint32_t)q * 32u;
      key[q] = 0xffffffffu;
      gidx[q] = g;
      if (j < j1) {
        uint32_t lx;
        const uint32_t ly = fast_divmod(j, (uint32_t)w.tw, w.tw_m, lx);
        const int tx = w.tx1 + (int)lx, ty = w.ty1 + (int)ly;
        if (tile_may_cover(w, tx, ty, a.tile)) key[q] = w.tile_base + (uint32_t)(ty * w.tiles_x + tx);
      }
    }
    count_pairs<4>(a, key, gidx, lane);
  }
}

// The count pass of the large triangles' segments.
__global__ void __launch_bounds__(256, 4) raster_large_count(RasterFrameArgs a)
{
  pdl_wait();
  pdl_trigger();
  const uint32_t items = min((uint32_t)a.ctr->large_acc, a.seg_cap);
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t it = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); it < items; it += warps)
    large_segment(a, it, threadIdx.x & 31);
}

// The scatter pass (the compaction): every recorded pair becomes its list
// entry at tile_off[tile] + its index in the tile, a streaming pass with no
// atomics; four pairs per thread per trip, loads first.
__global__ void __launch_bounds__(256) raster_scatter(RasterFrameArgs a)
{
  pdl_wait();
  pdl_trigger();
  // gridDim.x is a multiple of kPairParts: every partition gets
  // gridDim.x / kPairParts CTAs
  const uint32_t p = blockIdx.x % kPairParts, sub = blockIdx.x / kPairParts;
  const uint32_t part_cap = a.list_cap / kPairParts;
  const uint32_t n = min(a.ctr->pair_part[p], part_cap);
  const unsigned long long* ptl = a.pair_tl + (size_t)p * part_cap;
  const uint32_t* pg = a.pair_g + (size_t)p * part_cap;
  const uint32_t stride = (gridDim.x / kPairParts) * blockDim.x;
  for (uint32_t i0 = sub * blockDim.x + threadIdx.x; i0 < n; i0 += 4 * stride) {
    unsigned long long tl[4];
    uint32_t gi[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t i = i0 + (uint32_t)q * stride;
      tl[q] = i < n ? __ldcs(&ptl[i]) : ~0ull;
      gi[q] = i < n ? __ldcs(&pg[i]) : 0u;
    }
    uint32_t off[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) off[q] = tl[q] != ~0ull ? a.tile_off[(uint32_t)tl[q]] : 0u;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (tl[q] == ~0ull) continue;
      const uint32_t dst = off[q] + (uint32_t)(tl[q] >> 32);
      if (dst < a.list_cap) a.tile_list[dst] = gi[q];
    }
  }
}

// ------------------------------------------------------------------ kernel 4
// A triangle as one tile sees it (tile-local), built by the thread that takes
// the list entry.
struct TileTri {
  int32_t e[3];          // edge values at the centre of the tile's pixel (0, 0)
  int32_t sx[3], sy[3];  // per-pixel steps in x and y
  uint32_t trm, tam;     // per reference bin of the tile: assigned, trivially accepted
  int32_t lxe, lye;      // tile-local pixel limit of the bbox (pixel < limit)
  int32_t ex0, ex1, ey0, ey1;  // candidate pixels, clipped to the tile (inclusive)
  float inv, z2, z0mz2, z1mz2;
  uint32_t rank1;
  uint32_t gidx;         // setup index (coverage dump)
};

__device__ __forceinline__ void build_tile_tri(const TriSetup& r, int X0, int Y0, int T, TileTri& t)
{
  const int32_t Xc = X0 * 16 + 8, Yc = Y0 * 16 + 8;
  int32_t dx[3], dy[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    int j = i == 2 ? 0 : i + 1;
    dx[i] = wsub(r.x[j], r.x[i]);
    dy[i] = wsub(r.y[j], r.y[i]);
    t.e[i] = edge_at(Xc, Yc, r.x[i], r.y[i], dx[i], dy[i]);
    t.sx[i] = -wshl(dy[i], 4);
    t.sy[i] = wshl(dx[i], 4);
  }
  const int bx1 = (int)(r.bxr & 0xffff), bx2 = (int)(r.bxr >> 16);
  const int by1 = (int)(r.byr & 0xffff), by2 = (int)(r.byr >> 16);
  const int BPT = T / kRefBin;
  uint32_t trm = 0, tam = 0;
  for (int bj = 0; bj < BPT; ++bj) {
    const int by = Y0 / kRefBin + bj;
    if (by < by1 || by > by2) continue;
    for (int bi = 0; bi < BPT; ++bi) {
      const int bx = X0 / kRefBin + bi;
      if (bx < bx1 || bx > bx2) continue;
      // trivial reject at the bin corner (raster.pikostage:77-105, 128 = 8 px in 28.4)
      const int32_t BX = bx * 128, BY = by * 128;
      int32_t tr = 0, ta = 0;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        int32_t off = dy[i] < 0 ? -wshl(dy[i], 7) : 0;
        off = wadd(off, dx[i] >= 0 ? wshl(dx[i], 7) : 0);
        tr |= wadd(off, edge_at(BX, BY, r.x[i], r.y[i], dx[i], dy[i]));
        // trivial accept at the first pixel centre (raster.pikostage:201-211)
        int32_t offa = dy[i] >= 0 ? -wshl(dy[i], 4) : 0;
        offa = wadd(offa, dx[i] < 0 ? wshl(dx[i], 4) : 0);
        ta |= wadd(edge_at(BX + 8, BY + 8, r.x[i], r.y[i], dx[i], dy[i]), wshl(offa, kRefBinLg2));
      }
      if (tr >= 0) {
        const uint32_t bit = 1u << (bj * BPT + bi);
        trm |= bit;
        if ((ta & (int32_t)0x80000000) == 0) tam |= bit;
      }
    }
  }
  t.trm = trm;
  t.tam = tam;
  t.lxe = (r.hix >> 4) - X0;
  t.lye = (r.hiy >> 4) - Y0;
  int ex0, ex1, ey0, ey1;
  if (r.flags & kTriRisk) {
    ex0 = bx1 * kRefBin - X0; ex1 = bx2 * kRefBin + kRefBin - 1 - X0;
    ey0 = by1 * kRefBin - Y0; ey1 = by2 * kRefBin + kRefBin - 1 - Y0;
  } else {
    // covered centres lie inside the triangle when no edge value can wrap
    ex0 = (min(min(r.x[0], r.x[1]), r.x[2]) >> 4) - 1 - X0;
    ex1 = (max(max(r.x[0], r.x[1]), r.x[2]) >> 4) - X0;
    ey0 = (min(min(r.y[0], r.y[1]), r.y[2]) >> 4) - 1 - Y0;
    ey1 = (max(max(r.y[0], r.y[1]), r.y[2]) >> 4) - Y0;
  }
  t.ex0 = max(ex0, 0); t.ex1 = min(ex1, T - 1);
  t.ey0 = max(ey0, 0); t.ey1 = min(ey1, T - 1);
  if (!trm) t.ex1 = -1;  // nothing assigned in this tile
  t.inv = r.inv;
  t.z2 = r.z[2];
  t.z0mz2 = r.z[0] - r.z[2];
  t.z1mz2 = r.z[1] - r.z[2];
  t.rank1 = r.rank1;
}

// Inverse of submission_rank: the triangle id with the given rank.
__device__ __forceinline__ uint32_t rank_to_id(uint32_t r, const RasterSceneDev& S)
{
  const uint32_t nVS = (uint32_t)S.nVS;
  if (S.vs_chunks <= nVS) return r;  // at most one chunk per VS bin: ids are submitted in order
  uint32_t lo = 0, hi = nVS - 1;
  while (lo < hi) {
    const uint32_t b = (lo + hi + 1) >> 1;
    const uint32_t start = kVsChunk * (b * S.vs_q + min(b, S.vs_rem)) - (S.vs_last < b ? S.vs_deficit : 0u);
    if (start <= r) lo = b; else hi = b - 1;
  }
  const uint32_t start = kVsChunk * (lo * S.vs_q + min(lo, S.vs_rem)) - (S.vs_last < lo ? S.vs_deficit : 0u);
  const uint32_t pos = r - start;
  return (lo + (pos / kVsChunk) * nVS) * kVsChunk + pos % kVsChunk;
}


// Depth test of one candidate pixel (raster.pikostage:201-285): assigned bin,
// trivial accept or the bbox-limited edge test, barycentric depth, then the
// order-independent keep-the-smaller-key update.  Within one step of a warp no
// two lanes hold the same pixel, and the warp owns its tile, so the update
// needs no atomic.
template <int T>
__device__ __forceinline__ bool frag(const TileTri& t, int lx, int ly, unsigned long long* keys)
{
  constexpr int BPT = T / kRefBin;
  const uint32_t bit = 1u << ((ly >> kRefBinLg2) * BPT + (lx >> kRefBinLg2));
  if (!(t.trm & bit)) return false;
  const int32_t f0 = wadd(wadd(t.e[0], wmul(lx, t.sx[0])), wmul(ly, t.sy[0]));
  const int32_t f1 = wadd(wadd(t.e[1], wmul(lx, t.sx[1])), wmul(ly, t.sy[1]));
  const int32_t f2 = wadd(wadd(t.e[2], wmul(lx, t.sx[2])), wmul(ly, t.sy[2]));
  const bool cov = (t.tam & bit) || ((lx < t.lxe) && (ly < t.lye) && ((f0 | f1 | f2) >= 0));
  if (!cov) return false;
  const float alpha = (float)f1 * t.inv;
  const float beta = (float)f2 * t.inv;
  const float z = t.z2 + alpha * t.z0mz2 + beta * t.z1mz2;
  const unsigned long long key = frag_key(z, t.rank1);
  unsigned long long* k = &keys[ly * T + lx];
  if (key < *k) *k = key;
  return true;
}


// colour of the winning fragment (raster.pikostage:244-309), triangle `id` of
// scene S whose setup records start at `setup`: barycentrics from
// the same edge values, Gouraud interpolation, optional texel, toABGR by
// truncation.  inv255[k] holds (float)k / 255.0f, the exact quotient fromABGR
// computes (piko/math.h:323-330), so no division is repeated per pixel.
__device__ __forceinline__ uint32_t shade_winner(const RasterSceneDev& S, const TriSetup* setup, uint32_t id, int px,
                                                 int py, const float* inv255)
{
  // the texture coordinates are fetched by triangle id, alongside the setup record
  float2 q0 = make_float2(0.0f, 0.0f), q1 = q0, q2 = q0;
  if (S.uv) {
    q0 = __ldg(&S.uv[id]);
    q1 = __ldg(&S.uv[(size_t)S.N + id]);
    q2 = __ldg(&S.uv[2 * (size_t)S.N + id]);
  }
  const TriSetup r = load_setup(&setup[id]);
  const int32_t Xc = px * 16 + 8, Yc = py * 16 + 8;
  const int32_t e1 = edge_at(Xc, Yc, r.x[1], r.y[1], wsub(r.x[2], r.x[1]), wsub(r.y[2], r.y[1]));
  const int32_t e2 = edge_at(Xc, Yc, r.x[2], r.y[2], wsub(r.x[0], r.x[2]), wsub(r.y[0], r.y[2]));
  const float alpha = (float)e1 * r.inv;
  const float beta = (float)e2 * r.inv;
  float vc[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    vc[k][0] = inv255[(r.c[k] >> 0) & 255u];
    vc[k][1] = inv255[(r.c[k] >> 8) & 255u];
    vc[k][2] = inv255[(r.c[k] >> 16) & 255u];
  }
  float col[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float d0 = vc[0][c] - vc[2][c], d1 = vc[1][c] - vc[2][c];
    col[c] = vc[2][c] + alpha * d0 + beta * d1;
  }
  if (S.uv) {
    const float u = q2.x + alpha * (q0.x - q2.x) + beta * (q1.x - q2.x);
    const float v = q2.y + alpha * (q0.y - q2.y) + beta * (q1.y - q2.y);
    const int tx = cvt_i32_x86(floorf(u * (float)S.tex_w)) & (S.tex_w - 1);
    const int ty = cvt_i32_x86(floorf(v * (float)S.tex_h)) & (S.tex_h - 1);
    const uchar4 t = __ldg(&S.tex[(size_t)ty * S.tex_w + tx]);
    col[0] = col[0] * inv255[t.x];
    col[1] = col[1] * inv255[t.y];
    col[2] = col[2] * inv255[t.z];
  }
  return 0xff000000u | (cvt_u32_x86(col[2] * 255.0f) << 16) | (cvt_u32_x86(col[1] * 255.0f) << 8) |
         cvt_u32_x86(col[0] * 255.0f);
}

// Rasterizes list entries [b, e) of the tile at (X0, Y0) of scene S into the
// warp's tile keys (16/32-px tiles): 32 entries at a time each lane builds one
// entry's tile-local form, then the warp takes them one at a time, lanes
// spread over the entry's candidate box in 8x4 blocks.
template <int T>
__device__ __forceinline__ void tiles_entries(const RasterFrameArgs& a, const RasterSceneDev& S, int X0, int Y0,
                                              uint32_t off, uint32_t b, uint32_t e, unsigned long long* keys,
                                              TileTri* st, int lane, unsigned& covered)
{
  // entries past the list capacity are never read (the frame reports the overflow)
  const uint32_t lim = a.list_cap - min(off, a.list_cap);
  e = min(e, lim);
  for (uint32_t b0 = b; b0 < e; b0 += 32) {
    if (b0 + lane < e) {
      const uint32_t gi = a.tile_list[off + b0 + lane];
      build_tile_tri(load_setup(&a.setup[gi]), X0, Y0, T, st[lane]);
      st[lane].gidx = gi;
      if (st[lane].ex1 < st[lane].ex0 || st[lane].ey1 < st[lane].ey0) st[lane].rank1 = 0u;
    }
    __syncwarp();
    const int n = (int)min(32u, e - b0);
    for (int i = 0; i < n; ++i) {
      const TileTri& t = st[i];
      if (t.rank1) {
        const int ex1 = min(t.ex1, T - 1), ey1 = min(t.ey1, T - 1);
        const int lx0 = max(t.ex0, 0) + (lane & 7), ly0 = max(t.ey0, 0) + (lane >> 3);
        for (int ly = ly0; ly <= ey1; ly += 4) {
          for (int lx = lx0; lx <= ex1; lx += 8) {
            if (frag<T>(t, lx, ly, keys)) {
              ++covered;
              if (a.cov_cap) {
                const uint32_t slot = atomicAdd(&a.ctr->cov_count, 1u);
                if (slot < a.cov_cap) {
                  a.cov_tri[slot] = t.gidx - S.tri_base;
                  a.cov_pix[slot] = (uint32_t)((Y0 + ly) * S.W + X0 + lx);
                }
              }
            }
          }
        }
      }
      __syncwarp();  // the next triangle may touch the same pixels
    }
    __syncwarp();    // every lane is done with st[] before it is rebuilt
  }
}

// Resolve of a 16/32-px tile from the warp's keys: each pixel's winner is
// shaded once, the tile written once.
template <int T>
__device__ __forceinline__ void tiles_resolve(const RasterFrameArgs& a, const RasterSceneDev& S, int X0, int Y0,
                                              const unsigned long long* keys, int lane, const float* inv255)
{
  constexpr int PPT = T * T / 32;
#pragma unroll 4
  for (int j = 0; j < PPT; ++j) {
    const int p = j * 32 + lane;
    const int lx = p % T, ly = p / T;
    const int px = X0 + lx, py = Y0 + ly;
    const unsigned long long key = keys[p];
    if (px < S.W && py < S.H) {
      uint32_t c = kClearColor;
      float z = 1.0f;
      if (key != kInitKey) {
        const uint32_t rank = ~(uint32_t)key - 1u;
        z = __uint_as_float((uint32_t)(key >> 32) ^ 0x80000000u);
        const uint32_t id = rank_to_id(rank, S);
        c = shade_winner(S, a.setup + S.tri_base, id, px, py, inv255);
      }
      const size_t idx = (size_t)py * S.W + px;
      S.fb[idx] = c;
      S.depth[idx] = z;
    }
  }
}

// 16/32-px tiles, persistent: warp w of the grid first draws the plain tiles
// w, w + warps, ... (a heavy tile among them is skipped), then takes work items
// from one counter -- the chunks of the heavy tiles' lists (each chunk leaves
// its keys in chunk_keys; the warp finishing a tile's last chunk merges them
// and resolves the tile), or, without chunk buffers, the heavy tiles whole.
template <int T>
__global__ void __launch_bounds__(T == 32 ? 128 : 256) raster_tiles(RasterFrameArgs a)
{
  pdl_wait();
  if (list_overflowed(a)) return;
  constexpr int CTA = T == 32 ? 128 : 256;
  constexpr int NW = CTA / 32;    // warps per CTA, one work item each
  constexpr int NPX = T * T;
  constexpr int PPT = NPX / 32;   // pixels per lane
  __shared__ unsigned long long s_keys[NW][NPX];
  __shared__ TileTri s_tri[NW][32];
  __shared__ float s_inv255[256];
  constexpr int kTb = T == 32 ? 128 : 512;   // scene table (static shared memory stays under 48 KB)
  __shared__ uint32_t s_tb[kTb];
  for (int i = threadIdx.x; i < 256; i += CTA) s_inv255[i] = (float)i / 255.0f;
  load_scene_table<kTb>(a, s_tb, true);
  __syncthreads();
  const int wid = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  unsigned long long* keys = s_keys[wid];
  TileTri* st = s_tri[wid];
  unsigned covered = 0;
  const bool chunked = a.chunk_base != nullptr;
  const unsigned long long hacc = a.ctr->heavy_acc;
  const uint32_t n_heavy = min((uint32_t)(hacc >> 32), a.heavy_cap);
  const uint32_t n_chunks = chunked ? min((uint32_t)hacc, a.chunk_cap) : 0u;
  const uint32_t n_first = chunked ? n_chunks : n_heavy;   // items before the plain tiles

  // The plain tiles first, warp w of the grid taking tiles w, w + warps, ...;
  // then the heavy items (chunks, or whole heavy tiles) from a counter, which
  // also evens out the warps' finishing times.
  uint32_t plain = blockIdx.x * (uint32_t)NW + (uint32_t)wid;
  const uint32_t nwarps = gridDim.x * (uint32_t)NW;
  for (;;) {
    uint32_t w = 0;
    if (plain < a.n_tiles_total) {
      w = n_first + plain;
      plain += nwarps;
    } else {
      if (lane == 0) w = atomicAdd(&a.ctr->work_next, 1u);
      w = __shfl_sync(kFull, w, 0);
      if (w >= n_first) break;
    }
#pragma unroll
    for (int j = 0; j < PPT; ++j) keys[j * 32 + lane] = kInitKey;
    __syncwarp();
    uint32_t tile, b = 0, e = 0, h = 0, c0 = 0, nch = 1;
    bool chunk_item = false;
    if (w < n_first) {
      if (chunked) {
        h = a.chunk_heavy[w];
        if (h >= n_heavy) continue;  // only after a heavy-queue overflow (reported; the frame is redrawn)
        c0 = a.chunk_base[h];
        tile = a.heavy[h];
        const uint32_t cnt = a.tile_off[tile + 1] - a.tile_off[tile];
        const uint32_t ce = tile_chunk_entries(cnt, a.chunk, false);
        nch = (cnt + ce - 1) / ce;
        if (w - c0 >= nch) continue;  // only after a heavy-queue overflow (reported; the frame is redrawn)
        b = (w - c0) * ce;
        e = min(b + ce, cnt);
        chunk_item = true;
      } else {
        tile = a.heavy[w];
        e = a.tile_off[tile + 1] - a.tile_off[tile];
      }
    } else {
      tile = w - n_first;
      e = a.tile_cnt[tile];
      if (e > a.heavy_threshold) continue;  // served from the heavy queue
    }
    const int s = scene_of<kTb>(a, s_tb, tile, true);
    const RasterSceneDev& S = a.scenes[s];
    uint32_t ltx;
    const uint32_t lty = fast_divmod(tile - S.tile_base, (uint32_t)S.tiles_x, S.tiles_x_m, ltx);
    const int X0 = (int)ltx * T, Y0 = (int)lty * T;
    tiles_entries<T>(a, S, X0, Y0, a.tile_off[tile], b, e, keys, st, lane, covered);
    __syncwarp();
    if (chunk_item) {
      // this chunk's keys, then the finished-chunk count of its tile
      unsigned long long* ck = a.chunk_keys + (size_t)w * NPX;
#pragma unroll
      for (int j = 0; j < PPT; ++j) ck[j * 32 + lane] = keys[j * 32 + lane];
      __threadfence();
      __syncwarp();
      uint32_t done = 0;
      if (lane == 0) done = atomicAdd(&a.hdone[h], 1u);
      done = __shfl_sync(kFull, done, 0);
      if (done + 1 != nch) continue;
      // the tile's last chunk: every other chunk's keys are in chunk_keys
      __threadfence();
      for (uint32_t j = 0; j < nch; ++j) {
        if (c0 + j == w) continue;
        const unsigned long long* cj = a.chunk_keys + (size_t)(c0 + j) * NPX;
#pragma unroll
        for (int q = 0; q < PPT; ++q) keys[q * 32 + lane] = min(keys[q * 32 + lane], __ldcg(&cj[q * 32 + lane]));
      }
      __syncwarp();
    }
    tiles_resolve<T>(a, S, X0, Y0, keys, lane, s_inv255);
    __syncwarp();
  }
  // fragment count: one atomic per warp
  covered = __reduce_add_sync(kFull, covered);
  if (lane == 0 && covered) atomicAdd(&a.ctr->covered, (unsigned long long)covered);
}

// 8x8 tiles (one reference bin each): a warp takes a tile, or a chunk of a
// long tile list, and each lane two of the tile's pixels, (lane & 7, lane >> 3)
// and the pixel 4 rows above.  Entries are taken 32 at a time: first every
// lane tests its two pixels against all 32 entries (integer edge functions
// only, independent across entries) and collects one coverage bit per entry
// and pixel; then each lane runs the barycentric depth and the key update for
// its set bits alone, so the float work is not repeated across a warp for
// pixels an entry does not cover.  Each lane keeps its pixels' smallest
// fragment key in registers.  Lists hold exactly the reference's (triangle,
// bin) pairs.
struct __align__(16) BinTri {
  int32_t e0, e1, e2, sx0;      // edge values at the centre of the tile's pixel (0, 0); per-pixel x steps
  int32_t sx1, sx2, sy0, sy1;   // per-pixel y steps
  int32_t sy2, lxe, lye, flags; // bbox limit (pixel < limit), tile-local; kBinDraw | kBinAccept
  float inv, z2, z0mz2, z1mz2;
  uint32_t rank1, gidx, pad0, pad1;
};
constexpr int32_t kBinDraw = 1;    // the entry has pixels to test in this tile
constexpr int32_t kBinAccept = 2;  // trivially accepted bin: all 64 pixels covered

struct Tile8 {
  const RasterSceneDev* S;
  int X0, Y0;
  uint32_t off, cnt;     // list range; cnt as counted (not clamped)
};

// Scene and pixel origin of an 8x8 tile (list range left empty).
__device__ __forceinline__ Tile8 tile8_geom(const RasterFrameArgs& a, const uint32_t* tb, uint32_t tile)
{
  Tile8 t;
  const int s = scene_of_tile(a, tb, tile);
  t.S = &a.scenes[s];
  uint32_t tx;
  const uint32_t ty = fast_divmod(tile - t.S->tile_base, (uint32_t)t.S->tiles_x, t.S->tiles_x_m, tx);
  t.X0 = (int)tx * kRefBin;
  t.Y0 = (int)ty * kRefBin;
  t.off = 0;
  t.cnt = 0;
  return t;
}

__device__ __forceinline__ Tile8 tile8_at(const RasterFrameArgs& a, const uint32_t* tb, uint32_t tile)
{
  Tile8 t;
  const int s = scene_of_tile(a, tb, tile);
  t.S = &a.scenes[s];
  uint32_t tx;
  const uint32_t ty = fast_divmod(tile - t.S->tile_base, (uint32_t)t.S->tiles_x, t.S->tiles_x_m, tx);
  t.X0 = (int)tx * kRefBin;
  t.Y0 = (int)ty * kRefBin;
  t.off = a.tile_off[tile];
  t.cnt = a.tile_off[tile + 1] - t.off;
  return t;
}

// The tile-local form of list entry gi for the 8x8 tile at (X0, Y0).
__device__ __forceinline__ void frag8_build(const RasterFrameArgs& a, uint32_t gi, int X0, int Y0, BinTri& out)
{
  TileTri t;
  build_tile_tri(load_setup(&a.setup[gi]), X0, Y0, kRefBin, t);
  BinTri q;
  q.e0 = t.e[0]; q.e1 = t.e[1]; q.e2 = t.e[2];
  q.sx0 = t.sx[0]; q.sx1 = t.sx[1]; q.sx2 = t.sx[2];
  q.sy0 = t.sy[0]; q.sy1 = t.sy[1]; q.sy2 = t.sy[2];
  q.lxe = t.lxe; q.lye = t.lye;
  const bool draw = (t.trm & 1u) && t.ex1 >= t.ex0 && t.ey1 >= t.ey0 && t.rank1 != 0u;
  q.flags = (draw ? kBinDraw : 0) | ((t.tam & 1u) ? kBinAccept : 0);
  q.inv = t.inv; q.z2 = t.z2; q.z0mz2 = t.z0mz2; q.z1mz2 = t.z1mz2;
  q.rank1 = t.rank1; q.gidx = gi; q.pad0 = 0; q.pad1 = 0;
  out = q;
}

// Entry t's fragment at tile pixel (ox, ly): barycentrics from the edge
// values, z in the reference's operation order, and the order-independent key
// update of that pixel (k, and the winning entry's index w when TRACK).
template <bool TRACK>
__device__ __forceinline__ void frag8_depth(const RasterFrameArgs& a, const Tile8& tl, const BinTri& t, int i, int ox,
                                            int ly, unsigned long long& k, int& w)
{
  const int32_t g1 = wadd(wadd(t.e1, wmul(ox, t.sx1)), wmul(ly, t.sy1));
  const int32_t g2 = wadd(wadd(t.e2, wmul(ox, t.sx2)), wmul(ly, t.sy2));
  const float alpha = (float)g1 * t.inv;
  const float beta = (float)g2 * t.inv;
  const float z = t.z2 + alpha * t.z0mz2 + beta * t.z1mz2;
  const unsigned long long key = frag_key(z, t.rank1);
  if (key < k) { k = key; if (TRACK) w = i; }
  if (a.cov_cap) {
    const uint32_t slot = atomicAdd(&a.ctr->cov_count, 1u);
    if (slot < a.cov_cap) {
      a.cov_tri[slot] = t.gidx - tl.S->tri_base;
      a.cov_pix[slot] = (uint32_t)((tl.Y0 + ly) * tl.S->W + tl.X0 + ox);
    }
  }
}

// Tests the lane's two pixels of tile tl against entries st[0, n) (n <= 32)
// and folds the covered fragments into the lane's keys.  TRACK: w0 / w1 also
// follow the entry index (into st) of each pixel's current winner.
template <bool TRACK>
__device__ __forceinline__ void frag8_test(const RasterFrameArgs& a, const Tile8& tl, const BinTri* st, int n, int lane,
                                           unsigned& covered, unsigned long long& k0, unsigned long long& k1,
                                           int& w0, int& w1)
{
  const int ox = lane & 7, oy = lane >> 3;   // first pixel; the second is (ox, oy + 4)
  // coverage: bit i of m0 / m1 = entry i covers the lane's first / second pixel
  uint32_t m0 = 0, m1 = 0;
#pragma unroll 4
  for (int i = 0; i < n; ++i) {
    const int4 q2 = *reinterpret_cast<const int4*>(&st[i].sy2);
    const bool draw = (q2.w & kBinDraw) != 0, accept = (q2.w & kBinAccept) != 0;
    bool c0 = draw, c1 = draw;
    if (draw && !accept) {   // (one entry for the whole warp: a uniform branch)
      const int4 q0 = *reinterpret_cast<const int4*>(&st[i].e0);
      const int4 q1 = *reinterpret_cast<const int4*>(&st[i].sx1);
      const int32_t f0 = wadd(wadd(q0.x, wmul(ox, q0.w)), wmul(oy, q1.z));
      const int32_t f1 = wadd(wadd(q0.y, wmul(ox, q1.x)), wmul(oy, q1.w));
      const int32_t f2 = wadd(wadd(q0.z, wmul(ox, q1.y)), wmul(oy, q2.x));
      const int32_t g0 = wadd(f0, wshl(q1.z, 2)), g1 = wadd(f1, wshl(q1.w, 2)), g2 = wadd(f2, wshl(q2.x, 2));
      const bool inx = ox < q2.y;
      c0 = inx && oy < q2.z && (f0 | f1 | f2) >= 0;
      c1 = inx && oy + 4 < q2.z && (g0 | g1 | g2) >= 0;
    }
    m0 |= (uint32_t)c0 << i;
    m1 |= (uint32_t)c1 << i;
  }
  covered += __popc(m0) + __popc(m1);
  // depth: barycentrics from the same edge values, z in the reference's
  // operation order, and the order-independent key update
  // one covered entry of each of the lane's two pixels per trip (two
  // independent depth evaluations); each pixel still takes its entries in
  // ascending order
  while (m0 | m1) {
    if (m0) {
      const int i = __ffs(m0) - 1;
      m0 &= m0 - 1u;
      frag8_depth<TRACK>(a, tl, st[i], i, ox, oy, k0, w0);
    }
    if (m1) {
      const int i = __ffs(m1) - 1;
      m1 &= m1 - 1u;
      frag8_depth<TRACK>(a, tl, st[i], i, ox, oy + 4, k1, w1);
    }
  }
}

// Rasterizes list entries [b, e) of tile tl into the lane's two keys, 32
// entries at a time.
__device__ __forceinline__ void frag8_entries(const RasterFrameArgs& a, const Tile8& tl, uint32_t b, uint32_t e,
                                              BinTri* st, int lane, unsigned& covered, unsigned long long& k0,
                                              unsigned long long& k1)
{
  // entries past the list capacity are never read (the frame reports the overflow)
  const uint32_t lim = a.list_cap - min(tl.off, a.list_cap);
  e = min(e, lim);
  for (uint32_t b0 = b; b0 < e; b0 += 32) {
    if (b0 + lane < e) frag8_build(a, a.tile_list[tl.off + b0 + lane], tl.X0, tl.Y0, st[lane]);
    __syncwarp();
    int w0 = 0, w1 = 0;
    frag8_test<false>(a, tl, st, (int)min(32u, e - b0), lane, covered, k0, k1, w0, w1);
    __syncwarp();  // every lane is done with st[] before it is rebuilt
  }
}

// Writes the lane's two pixels: the winner's colour (shaded once per pixel)
// and depth, or the clear colour and 1.0.
__device__ __forceinline__ void resolve8(const RasterFrameArgs& a, const Tile8& tl, int lane, unsigned long long k0,
                                         unsigned long long k1, const float* inv255)
{
  const RasterSceneDev& S = *tl.S;
  const int px = tl.X0 + (lane & 7);
  if (px >= S.W) return;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int py = tl.Y0 + (lane >> 3) + 4 * k;
    if (py >= S.H) continue;
    const unsigned long long key = k ? k1 : k0;
    uint32_t c = kClearColor;
    float z = 1.0f;
    if (key != kInitKey) {
      const uint32_t rank = ~(uint32_t)key - 1u;
      z = __uint_as_float((uint32_t)(key >> 32) ^ 0x80000000u);
      const uint32_t id = rank_to_id(rank, S);
      c = shade_winner(S, a.setup + S.tri_base, id, px, py, inv255);
    }
    const size_t idx = (size_t)py * S.W + px;
    S.fb[idx] = c;
    S.depth[idx] = z;
  }
}

// What the resolve of a light tile needs of an entry besides its BinTri,
// staged in shared memory when the entry is built, so a pixel's winner is
// shaded from shared memory: the vertex colours as floats (byte / 255) and the
// texture coordinates, each as vertex 2's value and vertex 0's and 1's minus
// it -- the differences shade_winner forms for every pixel, formed once.
struct __align__(16) BinShade {
  float c2[3], dc0[3], dc1[3];   // per channel
  float u2, du0, du1;
  float v2, dv0, dv1, pad;
};
static_assert(sizeof(BinShade) == 64, "BinShade layout");

// The colour of entry t / sh at tile pixel (ox, ly): shade_winner's arithmetic
// (raster.pikostage:244-309) from the tile-local edge values, which equal the
// pixel-centre edge values bit for bit (both are the same wrapping int32
// linear function).
__device__ __forceinline__ uint32_t shade_entry(const RasterSceneDev& S, const BinTri& t, const BinShade& sh, int ox,
                                                int ly, const float* inv255)
{
  const int32_t g1 = wadd(wadd(t.e1, wmul(ox, t.sx1)), wmul(ly, t.sy1));
  const int32_t g2 = wadd(wadd(t.e2, wmul(ox, t.sx2)), wmul(ly, t.sy2));
  const float alpha = (float)g1 * t.inv;
  const float beta = (float)g2 * t.inv;
  float col[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) col[c] = sh.c2[c] + alpha * sh.dc0[c] + beta * sh.dc1[c];
  if (S.uv) {
    const float u = sh.u2 + alpha * sh.du0 + beta * sh.du1;
    const float v = sh.v2 + alpha * sh.dv0 + beta * sh.dv1;
    const int tx = cvt_i32_x86(floorf(u * (float)S.tex_w)) & (S.tex_w - 1);
    const int ty = cvt_i32_x86(floorf(v * (float)S.tex_h)) & (S.tex_h - 1);
    const uchar4 tt = __ldg(&S.tex[(size_t)ty * S.tex_w + tx]);
    col[0] = col[0] * inv255[tt.x];
    col[1] = col[1] * inv255[tt.y];
    col[2] = col[2] * inv255[tt.z];
  }
  return 0xff000000u | (cvt_u32_x86(col[2] * 255.0f) << 16) | (cvt_u32_x86(col[1] * 255.0f) << 8) |
         cvt_u32_x86(col[0] * 255.0f);
}

// Writes the lane's two pixels of a light tile from its winners' staged data
// (st / sh indexed by w0 / w1), or the clear colour and 1.0.
__device__ __forceinline__ void resolve8_staged(const Tile8& tl, int lane, unsigned long long k0, unsigned long long k1,
                                                int w0, int w1, const BinTri* st, const BinShade* sh,
                                                const float* inv255)
{
  const RasterSceneDev& S = *tl.S;
  const int ox = lane & 7;
  const int px = tl.X0 + ox;
  if (px >= S.W) return;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int ly = (lane >> 3) + 4 * k;
    const int py = tl.Y0 + ly;
    if (py >= S.H) continue;
    const unsigned long long key = k ? k1 : k0;
    const int w = k ? w1 : w0;
    uint32_t c = kClearColor;
    float z = 1.0f;
    if (key != kInitKey) {
      z = __uint_as_float((uint32_t)(key >> 32) ^ 0x80000000u);
      c = shade_entry(S, st[w], sh[w], ox, ly, inv255);
    }
    const size_t idx = (size_t)py * S.W + px;
    S.fb[idx] = c;
    S.depth[idx] = z;
  }
}

// A group of up to kLightGroup consecutive tiles whose lists hold at most
// queue_min (<= 32 / kLightGroup) entries each: their offsets, list entries
// and setup records are fetched together (one round of loads for the group,
// at most 32 entries, one per lane), then each tile is tested and resolved.
__device__ __forceinline__ void light_group(const RasterFrameArgs& a, const uint32_t* tb, uint32_t t0, uint32_t t1,
                                            uint32_t lim, BinTri* st, BinShade* sh, int lane, unsigned& covered,
                                            const float* inv255)
{
  const int nt = (int)(t1 - t0);
  // lane j <= nt holds tile_off[t0 + j]
  const uint32_t offj = lane <= nt ? a.tile_off[t0 + lane] : 0u;
  uint32_t cnt = 0;     // lane j < nt: entries of tile t0 + j (0 when it is served as chunks)
  bool served = false;  // lane j < nt: tile t0 + j is drawn by this group (its list fits)
  {
    const uint32_t next = __shfl_down_sync(kFull, offj, 1);
    if (lane < nt) {
      cnt = next - offj;
      served = cnt <= lim;
      if (!served) cnt = 0;
    }
  }
  const unsigned served_m = __ballot_sync(kFull, served);
  // inclusive prefix of the counts over the group's tiles
  uint32_t incl = cnt;
#pragma unroll
  for (int o = 1; o < kLightGroup; o <<= 1) {
    const uint32_t v = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += v;
  }
  uint32_t inc[kLightGroup];
#pragma unroll
  for (int q = 0; q < kLightGroup; ++q) inc[q] = __shfl_sync(kFull, incl, q);
  const uint32_t total = inc[kLightGroup - 1];
  // lane l < total builds entry l, of tile j = the first with inc[j] > l
  int j = 0;
#pragma unroll
  for (int q = 0; q < kLightGroup - 1; ++q)
    if ((uint32_t)lane >= inc[q]) j = q + 1;
  const uint32_t off = __shfl_sync(kFull, offj, j);
  if ((uint32_t)lane < total) {
    const Tile8 g = tile8_geom(a, tb, t0 + (uint32_t)j);
    uint32_t first = 0;
#pragma unroll
    for (int q = 0; q < kLightGroup - 1; ++q)
      if (q < j) first = inc[q];
    const uint32_t idx = off + ((uint32_t)lane - first);
    if (idx < a.list_cap) {
      const uint32_t gi = a.tile_list[idx];
      // the entry's colours and texture coordinates, for the resolve (the
      // uv arrays are indexed by triangle id = setup slot - the scene's base)
      const RasterSceneDev& S = *g.S;
      float2 q0 = make_float2(0.0f, 0.0f), q1 = q0, q2 = q0;
      if (S.uv) {
        const uint32_t id = gi - S.tri_base;
        q0 = __ldg(&S.uv[id]);
        q1 = __ldg(&S.uv[(size_t)S.N + id]);
        q2 = __ldg(&S.uv[2 * (size_t)S.N + id]);
      }
      const TriSetup r = load_setup(&a.setup[gi]);
      TileTri t;
      build_tile_tri(r, g.X0, g.Y0, kRefBin, t);
      BinTri bq;
      bq.e0 = t.e[0]; bq.e1 = t.e[1]; bq.e2 = t.e[2];
      bq.sx0 = t.sx[0]; bq.sx1 = t.sx[1]; bq.sx2 = t.sx[2];
      bq.sy0 = t.sy[0]; bq.sy1 = t.sy[1]; bq.sy2 = t.sy[2];
      bq.lxe = t.lxe; bq.lye = t.lye;
      const bool draw = (t.trm & 1u) && t.ex1 >= t.ex0 && t.ey1 >= t.ey0 && t.rank1 != 0u;
      bq.flags = (draw ? kBinDraw : 0) | ((t.tam & 1u) ? kBinAccept : 0);
      bq.inv = t.inv; bq.z2 = t.z2; bq.z0mz2 = t.z0mz2; bq.z1mz2 = t.z1mz2;
      bq.rank1 = t.rank1; bq.gidx = gi; bq.pad0 = 0; bq.pad1 = 0;
      st[lane] = bq;
      BinShade hq;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float v0 = inv255[(r.c[0] >> (8 * c)) & 255u], v1 = inv255[(r.c[1] >> (8 * c)) & 255u];
        const float v2 = inv255[(r.c[2] >> (8 * c)) & 255u];
        hq.c2[c] = v2;
        hq.dc0[c] = v0 - v2;
        hq.dc1[c] = v1 - v2;
      }
      hq.u2 = q2.x; hq.du0 = q0.x - q2.x; hq.du1 = q1.x - q2.x;
      hq.v2 = q2.y; hq.dv0 = q0.y - q2.y; hq.dv1 = q1.y - q2.y;
      hq.pad = 0.0f;
      sh[lane] = hq;
    } else {
      st[lane].flags = 0;  // past the list capacity: the frame reports the overflow
    }
  }
  __syncwarp();
  // one copy of the test and resolve code (the loop stays rolled: the kernel's
  // instruction footprint matters more than the loop overhead)
  uint32_t first = 0;
#pragma unroll 1
  for (int q = 0; q < nt; ++q) {
    const uint32_t iq = __shfl_sync(kFull, incl, q);
    if ((served_m >> q) & 1u) {  // (longer lists are drawn as chunks)
      const Tile8 tl = tile8_geom(a, tb, t0 + (uint32_t)q);
      unsigned long long k0 = kInitKey, k1 = kInitKey;
      int w0 = 0, w1 = 0;
      frag8_test<true>(a, tl, st + first, (int)(iq - first), lane, covered, k0, k1, w0, w1);
      resolve8_staged(tl, lane, k0, k1, w0, w1, st + first, sh + first, inv255);
    }
    first = iq;
  }
  __syncwarp();  // every lane is done with st[] before the next group rebuilds it
}

// Persistent: warp w of the grid first draws the short-list groups w,
// w + warps, ... (light_group), then takes chunks of the long lists (scan_tiles
// queued them) from a counter; each chunk stores its keys, and the warp that
// completes a tile's last chunk takes the per-pixel minimum over the tile's
// chunks and resolves the tile.  The key order makes the result independent of
// which warp merges when.
__global__ void __launch_bounds__(256, 4) raster_frag8(RasterFrameArgs a)
{
  pdl_wait();
  if (list_overflowed(a)) return;
  __shared__ BinTri s_tri[8][32];
  __shared__ BinShade s_shade[8][32];
  __shared__ float s_inv255[256];
  __shared__ unsigned s_cov[8];
  __shared__ uint32_t s_tb[kSceneTable];
  s_inv255[threadIdx.x] = (float)threadIdx.x / 255.0f;
  load_scene_table<kSceneTable>(a, s_tb, true);
  __syncthreads();
  const int wid = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  BinTri* st = s_tri[wid];
  unsigned covered = 0;
  const uint32_t C = a.chunk;
  const unsigned long long hacc = a.ctr->heavy_acc;
  const uint32_t n_heavy = min((uint32_t)(hacc >> 32), a.heavy_cap);
  const uint32_t n_chunks = min((uint32_t)hacc, a.chunk_cap);

  // The short lists first, kLightGroup consecutive tiles per group, warp w
  // of the grid taking groups w, w + warps, ... (no counter: the groups cost
  // about the same); then one counter hands out the heavy tiles' chunks (every
  // list longer than a.queue_min entries, cut into chunks of a.chunk), which
  // also evens out the warps' finishing times.  (Asking for the next item
  // while working on the current one measured slower: a warp busy with a long
  // item holds work that idle warps could take.)
  const uint32_t n_groups = (a.n_tiles_total + kLightGroup - 1) / kLightGroup;
  const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t g = blockIdx.x * (blockDim.x >> 5) + (uint32_t)wid; g < n_groups; g += nwarps) {
    const uint32_t t0 = g * kLightGroup;
    light_group(a, s_tb, t0, min(t0 + kLightGroup, a.n_tiles_total), a.queue_min, st, s_shade[wid], lane, covered,
                s_inv255);
  }
  for (;;) {
    uint32_t ci = 0;
    if (lane == 0) ci = atomicAdd(&a.ctr->work_next, 1u);
    ci = __shfl_sync(kFull, ci, 0);
    if (ci >= n_chunks) break;
    const uint32_t h = a.chunk_heavy[ci];
    if (h >= n_heavy) continue;  // only after a heavy-queue overflow (reported; the frame is redrawn)
    const uint32_t c0 = a.chunk_base[h];
    const Tile8 tl = tile8_at(a, s_tb, a.heavy[h]);
    const uint32_t nch = (tl.cnt + C - 1) / C;
    if (ci - c0 >= nch) continue;  // only after a heavy-queue overflow (reported; the frame is redrawn)
    unsigned long long k0 = kInitKey, k1 = kInitKey;
    frag8_entries(a, tl, (ci - c0) * C, min((ci - c0) * C + C, tl.cnt), st, lane, covered, k0, k1);
    if (nch == 1) {   // the whole list in one chunk: no keys to merge
      resolve8(a, tl, lane, k0, k1, s_inv255);
      continue;
    }
    // pixel p of the tile is key p of the chunk: the lane's pixels are lane and lane + 32
    unsigned long long* ck = a.chunk_keys + (size_t)ci * 64;
    ck[lane] = k0;
    ck[lane + 32] = k1;
    __threadfence();
    __syncwarp();
    uint32_t done = 0;
    if (lane == 0) done = atomicAdd(&a.hdone[h], 1u);
    done = __shfl_sync(kFull, done, 0);
    if (done + 1 == nch) {
      // the tile's last chunk: every other chunk's keys are in chunk_keys
      __threadfence();
      for (uint32_t j = 0; j < nch; ++j) {
        if (c0 + j == ci) continue;
        const unsigned long long* cj = a.chunk_keys + (size_t)(c0 + j) * 64;
        k0 = min(k0, __ldcg(&cj[lane]));
        k1 = min(k1, __ldcg(&cj[lane + 32]));
      }
      resolve8(a, tl, lane, k0, k1, s_inv255);
    }
  }

  // fragment count: one atomic per CTA
  covered = __reduce_add_sync(kFull, covered);
  if (lane == 0) s_cov[wid] = covered;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) t += s_cov[w];
    if (t) atomicAdd(&a.ctr->covered, t);
  }
}

// ------------------------------------------------------------------ launch
struct RasterLaunchInfo {
  int persistent_ctas;
};

int raster_scan_blocks(uint32_t n_tiles) { return (int)((n_tiles + kScanTile - 1) / kScanTile); }

// CTAs of one full wave of a kernel on the current device (cached; every
// launch of this library targets B200s of one kind).  Host threads may launch
// frames concurrently: the cache is an atomic, and two threads that both miss
// it compute and store the same value.
template <class K>
static int wave_ctas(K kernel, std::atomic<int>* cache, int threads = 256)
{
  int v = cache->load(std::memory_order_relaxed);
  if (v <= 0) {
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
    v = sms * (per_sm > 0 ? per_sm : 1);
    cache->store(v, std::memory_order_relaxed);
  }
  return v;
}

// A launch that may begin while the previous kernel of the stream finishes
// (the kernel's pdl_wait() holds it until that kernel's writes are visible).
template <typename K>
static cudaError_t launch_pdl(K kernel, int grid, int block, cudaStream_t st, const RasterFrameArgs& a)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, a);
}

cudaError_t launch_raster_frame(const RasterFrameArgs& a, int raster_ctas, cudaStream_t st, cudaEvent_t* ev)
{
  static std::atomic<int> setup_wave{0}, scatter_wave{0}, large_wave{0};
  const int tri_blocks = (int)((a.n_tris_total + 255) / 256);
  const int setup_blocks = min((int)((a.n_tris_total + kSetupThreads - 1) / kSetupThreads),
                               wave_ctas(raster_setup, &setup_wave, kSetupThreads));
  // the scatter grid covers the list groups of every triangle plus the large
  // triangles' segments (a grid-stride loop takes any excess)
  const int scatter_blocks = std::max(1, wave_ctas(raster_scatter, &scatter_wave) / (int)kPairParts) * (int)kPairParts;
  if (ev) cudaEventRecord(ev[0], st);
  const int large_blocks = wave_ctas(raster_large_count, &large_wave);
  // every launch after the first may start while its predecessor drains
  // (programmatic dependent launch); each waits for it before touching memory
  cudaError_t e = cudaSuccess;
  if (tri_blocks) raster_setup<<<setup_blocks, kSetupThreads, 0, st>>>(a);
  if (tri_blocks && !e) e = launch_pdl(raster_large_count, large_blocks, 256, st, a);
  if (ev) cudaEventRecord(ev[1], st);
  if (!e) e = launch_pdl(scan_tiles, raster_scan_blocks(a.n_tiles_total), kScanThreads, st, a);
  if (ev) cudaEventRecord(ev[2], st);
  if (tri_blocks && !e) e = launch_pdl(raster_scatter, scatter_blocks, 256, st, a);
  if (ev) cudaEventRecord(ev[3], st);
  if (!e) {
    switch (a.tile) {
      case 8: e = launch_pdl(raster_frag8, raster_ctas, 256, st, a); break;
      case 32: e = launch_pdl(raster_tiles<32>, raster_ctas, 128, st, a); break;
      default: e = launch_pdl(raster_tiles<16>, raster_ctas, 256, st, a); break;
    }
  }
  if (ev) cudaEventRecord(ev[4], st);
  if (e) return e;
  return cudaGetLastError();
}

cudaError_t launch_scan_tiles(const RasterFrameArgs& a, cudaStream_t st)
{
  scan_tiles<<<raster_scan_blocks(a.n_tiles_total), kScanThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t raster_tiles_occupancy(int tile, int* blocks_per_sm)
{
  switch (tile) {
    case 8: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, raster_frag8, 256, 0);
    case 32: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, raster_tiles<32>, 128, 0);
    default: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, raster_tiles<16>, 256, 0);
  }
}

}  // namespace piko
