// Binned raster pipeline for sm_100a: the reference's RasterPipe
// (VertexShaderStage -> RasterStage -> PikoScreen, pikoc/samples/rasterPipelineFixPt)
// as four kernels per frame, over one scene or a batch of scenes:
//
//   raster_setup    one thread per triangle.  Vertex shading + triangle setup
//                   (R1: main.cpp:299-400 moved on device; R3: vertexShader.pikostage:36-109)
//                   from coalesced float4 SoA loads, then AssignBin (R4,
//                   raster.pikostage:40-117) as a warp-cooperative tile walk with
//                   warp-aggregated atomic counts per tile.
//   scan_tiles      exclusive prefix sum of the tile counts (single pass,
//                   decoupled look-back) -> per-tile list offsets; tiles with long
//                   lists go to a heavy queue served first.
//   raster_scatter  the same walk again, appending each triangle to its tiles'
//                   lists (warp-aggregated atomic cursors): the compaction.
//   raster_tiles    persistent CTAs pop tiles from a work counter (Schedule).
//                   A tile is rasterized by a thread group; each thread owns a
//                   2x2 quad and keeps its pixels' colour/depth winner in
//                   registers.  Coverage is the reference's 28.4 edge test with
//                   its 8x8-bin trivial reject/accept (R6, raster.pikostage:124-242),
//                   the z test and the composite are fused in (R7/R8).
//
// Order independence.  The reference's depth test is an atomicMin on the float
// bits compared as signed ints, with ties passing (raster.pikostage:274-285).
// Run sequentially that leaves, per pixel, the minimum depth bits and the
// colour of the LAST fragment, in submission order, that has those bits.  So
// each fragment carries its triangle's submission rank and a pixel keeps the
// fragment with the smallest (depth bits, -rank): the result equals the
// sequential one whatever order the tile lists come in, and no list is sorted.
#include "piko_device.cuh"

namespace piko {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kLargeTiles = 32;  // tiles in a triangle's box above which a CTA walks it

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

// Rank of triangle `id` in the order the one-thread CPU backend submits
// triangles to the raster bins: VS bins in index order (kernel1 blocks), and in
// VS bin b the ids with (id/512) % nVS == b ascending (vertexShader.pikostage:25-29).
__device__ __forceinline__ uint32_t submission_rank(uint32_t id, uint32_t N, uint32_t nVS)
{
  uint32_t C = (N + kVsChunk - 1) / kVsChunk;
  uint32_t c = id / kVsChunk;
  uint32_t b = c % nVS;
  uint32_t q = C / nVS, rem = C % nVS;
  uint32_t lastbin = (C - 1) % nVS;
  uint32_t deficit = C * kVsChunk - N;
  uint32_t start = kVsChunk * (b * q + min(b, rem)) - (lastbin < b ? deficit : 0u);
  return start + (c / nVS) * kVsChunk + (id % kVsChunk);
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
struct WalkTri {
  int32_t x[3], y[3];
  int32_t bx1, bx2, by1, by2;
  int32_t tx1, ty1, tw;
  uint32_t gidx;
  uint32_t tile_base;
  int32_t tiles_x;
  uint32_t flags;
};

// Conservative tile-level trivial reject (exact int64 arithmetic): the tile,
// clipped to the triangle's bin range, can hold an assigned reference bin only
// if every edge function is >= 0 at the tile corner that maximises it.  Only
// used for triangles whose edge values cannot wrap inside the bin range.
__device__ __forceinline__ bool tile_may_cover(const WalkTri& w, int tx, int ty, int T)
{
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

// Walks every (triangle, tile) pair of a warp's 32 triangles with all 32 lanes
// busy: pair j belongs to the lane whose inclusive tile-count prefix first
// exceeds j.  COUNT: warp-aggregated atomicAdd on the tile counters.
// SCATTER: warp-aggregated cursor bump, then one list slot per lane.
template <bool SCATTER>
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
  for (uint32_t base = 0; base < total; base += 32) {
    uint32_t j = base + lane;
    int lo = 0, hi = 31;
#pragma unroll
    for (int s = 0; s < 5; ++s) {
      int mid = (lo + hi) >> 1;
      uint32_t v = __shfl_sync(kFull, incl, mid);
      if (v > j) hi = mid; else lo = mid + 1;
    }
    int owner = lo;
    uint32_t oexcl = __shfl_sync(kFull, excl, owner);
    uint32_t key = 0xffffffffu;
    uint32_t gidx = 0;
    if (j < total) {
      const WalkTri& w = wt[owner];
      uint32_t local = j - oexcl;
      int tx = w.tx1 + (int)(local % (uint32_t)w.tw);
      int ty = w.ty1 + (int)(local / (uint32_t)w.tw);
      if (tile_may_cover(w, tx, ty, a.tile)) {
        key = w.tile_base + (uint32_t)(ty * w.tiles_x + tx);
        gidx = w.gidx;
      }
    }
    unsigned peers = __match_any_sync(kFull, key);
    if (key != 0xffffffffu) {
      int leader = __ffs(peers) - 1;
      uint32_t cnt = __popc(peers);
      if (!SCATTER) {
        if (lane == leader) atomicAdd(&a.tile_cnt[key], cnt);
      } else {
        uint32_t b = 0;
        if (lane == leader) b = atomicAdd(&a.tile_cursor[key], cnt);
        b = __shfl_sync(peers, b, leader);
        uint32_t slot = b + __popc(peers & ((1u << lane) - 1u));
        if (slot < a.list_cap) a.tile_list[slot] = gidx;
      }
    }
  }
}

__device__ __forceinline__ void fill_walk(const RasterFrameArgs& a, const RasterSceneDev& S, const TriSetup& r,
                                          uint32_t g, WalkTri& w, uint32_t& ntiles)
{
  const int T = a.tile;
  for (int k = 0; k < 3; ++k) { w.x[k] = r.x[k]; w.y[k] = r.y[k]; }
  w.bx1 = (int)(r.bxr & 0xffff); w.bx2 = (int)(r.bxr >> 16);
  w.by1 = (int)(r.byr & 0xffff); w.by2 = (int)(r.byr >> 16);
  w.tx1 = (w.bx1 * kRefBin) / T;
  w.ty1 = (w.by1 * kRefBin) / T;
  int tx2 = (w.bx2 * kRefBin) / T, ty2 = (w.by2 * kRefBin) / T;
  w.tw = tx2 - w.tx1 + 1;
  w.gidx = g;
  w.tile_base = S.tile_base;
  w.tiles_x = S.tiles_x;
  w.flags = r.flags;
  ntiles = (uint32_t)w.tw * (uint32_t)(ty2 - w.ty1 + 1);
}

// ------------------------------------------------------------------ kernel 1
__global__ void __launch_bounds__(256) raster_setup(RasterFrameArgs a)
{
  __shared__ WalkTri s_walk[256];
  const uint32_t g = blockIdx.x * 256u + threadIdx.x;
  uint32_t ntiles = 0;
  bool kept_flag = false, risk_flag = false;
  if (g < a.n_tris_total) {
    const int s = find_base(a.scenes, a.n_scenes, g, false);
    const RasterSceneDev& S = a.scenes[s];
    const uint32_t id = g - S.tri_base;
    float sx[3], sy[3], sz[3];
    uint32_t ic[3];
    if (S.input_kind == kInputSoA) {
      // R1, main.cpp:299-400: vtransform, perspective divide, viewport; per-vertex
      // Gouraud lighting with the normal normalised by HOST::normalize.
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float4 p = __ldg(&S.pos[(size_t)k * S.N + id]);
        const float4 n4 = __ldg(&S.nrm[(size_t)k * S.N + id]);
        const float4 c4 = __ldg(&S.col[(size_t)k * S.N + id]);
        float mag = sqrtf(n4.x * n4.x + n4.y * n4.y + n4.z * n4.z);
        F3 n = {n4.x / mag, n4.y / mag, n4.z / mag};
        F3 l;
        if (S.light_mode == 1) {
          l.x = S.eye[0] - p.x; l.y = S.eye[1] - p.y; l.z = S.eye[2] - p.z;
          float m = sqrtf(l.x * l.x + l.y * l.y + l.z * l.z);
          if (m != 0.0f) { float rr = 1.0f / m; l.x = l.x * rr; l.y = l.y * rr; l.z = l.z * rr; }
        } else {
          l.x = S.light[0]; l.y = S.light[1]; l.z = S.light[2];
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
        ic[k] = light_abgr(n, l, F3{c4.x, c4.y, c4.z});
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
        r.rank1 = submission_rank(id, (uint32_t)S.N, (uint32_t)S.nVS) + 1u;
        r.bxr = (uint32_t)bx1 | ((uint32_t)bx2 << 16);
        r.byr = (uint32_t)by1 | ((uint32_t)by2 << 16);
        // can any edge value the reference compares wrap inside the bin range?
        const long long X0 = (long long)bx1 * 128, X1 = (long long)(bx2 + 1) * 128;
        const long long Y0 = (long long)by1 * 128, Y1 = (long long)(by2 + 1) * 128;
        long long worst = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          int j = i == 2 ? 0 : i + 1;
          long long dx = (long long)r.x[j] - r.x[i], dy = (long long)r.y[j] - r.y[i];
          long long m = 0;
          long long e;
          e = (Y0 - r.y[i]) * dx - (X0 - r.x[i]) * dy; m = max(m, e < 0 ? -e : e);
          e = (Y0 - r.y[i]) * dx - (X1 - r.x[i]) * dy; m = max(m, e < 0 ? -e : e);
          e = (Y1 - r.y[i]) * dx - (X0 - r.x[i]) * dy; m = max(m, e < 0 ? -e : e);
          e = (Y1 - r.y[i]) * dx - (X1 - r.x[i]) * dy; m = max(m, e < 0 ? -e : e);
          m += 512 * ((dx < 0 ? -dx : dx) + (dy < 0 ? -dy : dy));
          worst = max(worst, m);
        }
        if (worst >= 2147483647LL) r.flags |= kTriRisk;
        risk_flag = (r.flags & kTriRisk) != 0;
      }
    }
    // 80-byte record as five 16-byte stores
    const uint4* src = reinterpret_cast<const uint4*>(&r);
    uint4* dst = reinterpret_cast<uint4*>(&a.setup[g]);
#pragma unroll
    for (int k = 0; k < 5; ++k) dst[k] = src[k];
    if (r.rank1) fill_walk(a, S, r, g, s_walk[threadIdx.x], ntiles);
    if (ntiles > kLargeTiles) {
      a.large[atomicAdd(&a.ctr->large_count, 1u)] = g;
      ntiles = 0;
    }
  }
  const unsigned nk = __popc(__ballot_sync(kFull, kept_flag));
  const unsigned nr = __popc(__ballot_sync(kFull, risk_flag));
  if ((threadIdx.x & 31) == 0) {
    if (nk) atomicAdd(&a.ctr->kept, nk);
    if (nr) atomicAdd(&a.ctr->risk, (unsigned long long)nr);
  }
  __syncwarp();
  walk_tiles<false>(a, &s_walk[threadIdx.x & ~31], ntiles);
}

// ------------------------------------------------------------------ kernel 2
// Exclusive scan of tile_cnt (decoupled look-back).  Flags per block hold
// (epoch << 34) | (state << 32) | value, state 1 = aggregate, 2 = inclusive.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) scan_tiles(RasterFrameArgs a)
{
  __shared__ uint32_t s_bid;
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t s_prefix;
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
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  uint32_t warp_excl = 0, agg = 0;
#pragma unroll
  for (int w = 0; w < kScanThreads / 32; ++w) {
    if (w < warp) warp_excl += s_warp[w];
    agg += s_warp[w];
  }
  const unsigned long long ep = (unsigned long long)a.epoch << 34;
  if (threadIdx.x == 0) {
    uint32_t prefix = 0;
    if (bid == 0) {
      atomicExch(&a.scan_flags[0], ep | (2ull << 32) | agg);
    } else {
      atomicExch(&a.scan_flags[bid], ep | (1ull << 32) | agg);
      int idx = (int)bid - 1;
      uint32_t spins = 0;
      while (idx >= 0) {
        unsigned long long f = atomicAdd(&a.scan_flags[idx], 0ull);
        uint32_t state = (uint32_t)(f >> 32) & 3u;
        if ((f >> 34) != a.epoch || state == 0) {
          if (++spins > (1u << 22)) { atomicOr(&a.ctr->status, kStatusScanTimeout); break; }
          __nanosleep(32);
          continue;
        }
        prefix += (uint32_t)f;
        if (state == 2) break;
        --idx;
      }
      atomicExch(&a.scan_flags[bid], ep | (2ull << 32) | (uint32_t)(prefix + agg));
    }
    s_prefix = prefix;
  }
  __syncthreads();
  uint32_t run = s_prefix + warp_excl + (incl - sum);
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) {
      a.tile_off[base + i] = run;
      a.tile_cursor[base + i] = run;
      if (v[i] > a.heavy_threshold) a.heavy[atomicAdd(&a.ctr->heavy_count, 1u)] = base + i;
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
__global__ void __launch_bounds__(256) raster_scatter(RasterFrameArgs a)
{
  __shared__ WalkTri s_walk[256];
  const uint32_t g = blockIdx.x * 256u + threadIdx.x;
  uint32_t ntiles = 0;
  if (g < a.n_tris_total) {
    const TriSetup r = a.setup[g];
    if (r.rank1) {
      const int s = find_base(a.scenes, a.n_scenes, g, false);
      fill_walk(a, a.scenes[s], r, g, s_walk[threadIdx.x], ntiles);
      if (ntiles > kLargeTiles) ntiles = 0;  // walked by raster_large
    }
  }
  __syncwarp();
  walk_tiles<true>(a, &s_walk[threadIdx.x & ~31], ntiles);
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
};

template <int GS>
__device__ __forceinline__ void group_sync(int grp)
{
  if constexpr (GS == 256) {
    __syncthreads();
  } else if constexpr (GS > 32) {
    asm volatile("bar.sync %0, %1;" ::"r"(grp + 1), "r"(GS) : "memory");
  } else {
    __syncwarp();
  }
}

__device__ __forceinline__ uint32_t next_tile(const RasterFrameArgs& a)
{
  const uint32_t heavy_n = a.ctr->heavy_count;
  for (;;) {
    uint32_t w = atomicAdd(&a.ctr->work_next, 1u);
    if (w < heavy_n) return a.heavy[w];
    uint32_t t = w - heavy_n;
    if (t >= a.n_tiles_total) return 0xffffffffu;
    if (a.tile_cnt[t] > a.heavy_threshold) continue;  // already served from the heavy queue
    return t;
  }
}

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
__device__ __forceinline__ uint32_t rank_to_id(uint32_t r, uint32_t N, uint32_t nVS)
{
  const uint32_t C = (N + kVsChunk - 1) / kVsChunk;
  if (C <= nVS) return r;  // at most one chunk per VS bin: ids are submitted in order
  const uint32_t q = C / nVS, rem = C % nVS;
  const uint32_t lastbin = (C - 1) % nVS;
  const uint32_t deficit = C * kVsChunk - N;
  uint32_t lo = 0, hi = nVS - 1;
  while (lo < hi) {
    const uint32_t b = (lo + hi + 1) >> 1;
    const uint32_t start = kVsChunk * (b * q + min(b, rem)) - (lastbin < b ? deficit : 0u);
    if (start <= r) lo = b; else hi = b - 1;
  }
  const uint32_t start = kVsChunk * (lo * q + min(lo, rem)) - (lastbin < lo ? deficit : 0u);
  const uint32_t pos = r - start;
  return (lo + (pos / kVsChunk) * nVS) * kVsChunk + pos % kVsChunk;
}

// (depth bits as signed ints ascending, submission rank descending) as one
// unsigned 64-bit key: the smallest key is the sequential depth test's winner.
__device__ __forceinline__ unsigned long long frag_key(float z, uint32_t rank1)
{
  return ((unsigned long long)((uint32_t)__float_as_int(z) ^ 0x80000000u) << 32) | (uint32_t)(~rank1);
}
constexpr unsigned long long kInitKey = ((unsigned long long)(0x3f800000u ^ 0x80000000u) << 32) | 0xffffffffull;

// Depth test of one candidate pixel of a triangle (raster.pikostage:201-285):
// assigned bin, trivial accept or the bbox-limited edge test, then the
// barycentric depth.  Returns true when the pixel is covered.
template <int T>
__device__ __forceinline__ bool frag(const TileTri& t, int lx, int ly, int32_t f0, int32_t f1, int32_t f2,
                                     unsigned long long* keys)
{
  constexpr int BPT = T / kRefBin;
  const uint32_t bit = 1u << ((ly >> kRefBinLg2) * BPT + (lx >> kRefBinLg2));
  if (!(t.trm & bit)) return false;
  const bool cov = (t.tam & bit) || ((lx < t.lxe) && (ly < t.lye) && ((f0 | f1 | f2) >= 0));
  if (!cov) return false;
  const float alpha = (float)f1 * t.inv;
  const float beta = (float)f2 * t.inv;
  const float z = t.z2 + alpha * t.z0mz2 + beta * t.z1mz2;
  atomicMin(&keys[ly * T + lx], frag_key(z, t.rank1));
  return true;
}

// colour of the winning fragment (raster.pikostage:244-309): barycentrics from
// the same edge values, Gouraud interpolation, optional texel, toABGR by truncation
__device__ __forceinline__ uint32_t shade_winner(const RasterSceneDev& S, const TriSetup& r, int px, int py)
{
  const int32_t Xc = px * 16 + 8, Yc = py * 16 + 8;
  const int32_t e1 = edge_at(Xc, Yc, r.x[1], r.y[1], wsub(r.x[2], r.x[1]), wsub(r.y[2], r.y[1]));
  const int32_t e2 = edge_at(Xc, Yc, r.x[2], r.y[2], wsub(r.x[0], r.x[2]), wsub(r.y[0], r.y[2]));
  const float alpha = (float)e1 * r.inv;
  const float beta = (float)e2 * r.inv;
  float vc[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    vc[k][0] = (float)((r.c[k] >> 0) & 255u) / 255.0f;
    vc[k][1] = (float)((r.c[k] >> 8) & 255u) / 255.0f;
    vc[k][2] = (float)((r.c[k] >> 16) & 255u) / 255.0f;
  }
  float col[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float d0 = vc[0][c] - vc[2][c], d1 = vc[1][c] - vc[2][c];
    col[c] = vc[2][c] + alpha * d0 + beta * d1;
  }
  if (S.uv) {
    const float2 q0 = __ldg(&S.uv[r.id]);
    const float2 q1 = __ldg(&S.uv[(size_t)S.N + r.id]);
    const float2 q2 = __ldg(&S.uv[2 * (size_t)S.N + r.id]);
    const float u = q2.x + alpha * (q0.x - q2.x) + beta * (q1.x - q2.x);
    const float v = q2.y + alpha * (q0.y - q2.y) + beta * (q1.y - q2.y);
    const int tx = cvt_i32_x86(floorf(u * (float)S.tex_w)) & (S.tex_w - 1);
    const int ty = cvt_i32_x86(floorf(v * (float)S.tex_h)) & (S.tex_h - 1);
    const uchar4 t = __ldg(&S.tex[(size_t)ty * S.tex_w + tx]);
    col[0] = col[0] * ((float)t.x / 255.0f);
    col[1] = col[1] * ((float)t.y / 255.0f);
    col[2] = col[2] * ((float)t.z / 255.0f);
  }
  return 0xff000000u | (cvt_u32_x86(col[2] * 255.0f) << 16) | (cvt_u32_x86(col[1] * 255.0f) << 8) |
         cvt_u32_x86(col[0] * 255.0f);
}

template <int T>
__global__ void __launch_bounds__(256) raster_tiles(RasterFrameArgs a)
{
  constexpr int GS = T == 8 ? 32 : (T == 16 ? 64 : 256);  // threads per tile
  constexpr int NG = 256 / GS;
  constexpr int NPX = T * T;
  constexpr int PPT = NPX / GS;
  constexpr int kBig = 32;   // candidate pixels above which a warp shares one triangle
  __shared__ unsigned long long s_keys[NG][NPX];
  __shared__ uint32_t s_tile[NG];
  const int grp = threadIdx.x / GS;
  const int q = threadIdx.x % GS;
  const int lane = threadIdx.x & 31;
  unsigned long long* keys = s_keys[grp];
  unsigned covered = 0;

  for (;;) {
    if (q == 0) s_tile[grp] = next_tile(a);
#pragma unroll
    for (int j = 0; j < PPT; ++j) keys[j * GS + q] = kInitKey;
    group_sync<GS>(grp);
    const uint32_t tile = s_tile[grp];
    if (tile == 0xffffffffu) break;
    const int s = find_base(a.scenes, a.n_scenes, tile, true);
    const RasterSceneDev& S = a.scenes[s];
    const uint32_t lt = tile - S.tile_base;
    const int X0 = (int)(lt % (uint32_t)S.tiles_x) * T, Y0 = (int)(lt / (uint32_t)S.tiles_x) * T;
    const uint32_t off = a.tile_off[tile];
    uint32_t cnt = a.tile_off[tile + 1] - off;
    if (off + cnt > a.list_cap) cnt = off < a.list_cap ? a.list_cap - off : 0;

    // fragments: one list entry per thread; small triangles walk their own
    // candidate pixels, large ones are shared by the warp
    for (uint32_t b0 = 0; b0 < cnt; b0 += GS) {
      const uint32_t i = b0 + q;
      TileTri t;
      int w = 0, area = 0;
      uint32_t gi = 0;
      if (i < cnt) {
        gi = a.tile_list[off + i];
        build_tile_tri(a.setup[gi], X0, Y0, T, t);
        if (t.ex1 >= t.ex0 && t.ey1 >= t.ey0) {
          w = t.ex1 - t.ex0 + 1;
          area = w * (t.ey1 - t.ey0 + 1);
        }
      }
      const bool big = area > kBig;
      if (area && !big) {
        for (int ly = t.ey0; ly <= t.ey1; ++ly) {
          int32_t f0 = wadd(wadd(t.e[0], wmul(t.ex0, t.sx[0])), wmul(ly, t.sy[0]));
          int32_t f1 = wadd(wadd(t.e[1], wmul(t.ex0, t.sx[1])), wmul(ly, t.sy[1]));
          int32_t f2 = wadd(wadd(t.e[2], wmul(t.ex0, t.sx[2])), wmul(ly, t.sy[2]));
          for (int lx = t.ex0; lx <= t.ex1; ++lx) {
            if (frag<T>(t, lx, ly, f0, f1, f2, keys)) {
              ++covered;
              if (a.cov_cap) {
                const uint32_t slot = atomicAdd(&a.ctr->cov_count, 1u);
                if (slot < a.cov_cap) {
                  a.cov_tri[slot] = gi - S.tri_base;
                  a.cov_pix[slot] = (uint32_t)((Y0 + ly) * S.W + X0 + lx);
                }
              }
            }
            f0 = wadd(f0, t.sx[0]); f1 = wadd(f1, t.sx[1]); f2 = wadd(f2, t.sx[2]);
          }
        }
      }
      unsigned bigs = __ballot_sync(kFull, big);
      while (bigs) {
        const int src = __ffs(bigs) - 1;
        bigs &= bigs - 1;
        TileTri u;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          u.e[k] = __shfl_sync(kFull, t.e[k], src);
          u.sx[k] = __shfl_sync(kFull, t.sx[k], src);
          u.sy[k] = __shfl_sync(kFull, t.sy[k], src);
        }
        u.trm = __shfl_sync(kFull, t.trm, src);
        u.tam = __shfl_sync(kFull, t.tam, src);
        u.lxe = __shfl_sync(kFull, t.lxe, src);
        u.lye = __shfl_sync(kFull, t.lye, src);
        u.ex0 = __shfl_sync(kFull, t.ex0, src);
        u.ey0 = __shfl_sync(kFull, t.ey0, src);
        u.inv = __shfl_sync(kFull, t.inv, src);
        u.z2 = __shfl_sync(kFull, t.z2, src);
        u.z0mz2 = __shfl_sync(kFull, t.z0mz2, src);
        u.z1mz2 = __shfl_sync(kFull, t.z1mz2, src);
        u.rank1 = __shfl_sync(kFull, t.rank1, src);
        const int uw = __shfl_sync(kFull, w, src);
        const int ua = __shfl_sync(kFull, area, src);
        const uint32_t ugi = __shfl_sync(kFull, gi, src);
        for (int p = lane; p < ua; p += 32) {
          const int lx = u.ex0 + p % uw, ly = u.ey0 + p / uw;
          const int32_t f0 = wadd(wadd(u.e[0], wmul(lx, u.sx[0])), wmul(ly, u.sy[0]));
          const int32_t f1 = wadd(wadd(u.e[1], wmul(lx, u.sx[1])), wmul(ly, u.sy[1]));
          const int32_t f2 = wadd(wadd(u.e[2], wmul(lx, u.sx[2])), wmul(ly, u.sy[2]));
          if (frag<T>(u, lx, ly, f0, f1, f2, keys)) {
            ++covered;
            if (a.cov_cap) {
              const uint32_t slot = atomicAdd(&a.ctr->cov_count, 1u);
              if (slot < a.cov_cap) {
                a.cov_tri[slot] = ugi - S.tri_base;
                a.cov_pix[slot] = (uint32_t)((Y0 + ly) * S.W + X0 + lx);
              }
            }
          }
        }
      }
    }
    group_sync<GS>(grp);
    // resolve: each pixel's winner is shaded once; the tile is written once
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      const int p = j * GS + q;
      const int lx = p % T, ly = p / T;
      const int px = X0 + lx, py = Y0 + ly;
      const unsigned long long key = keys[p];
      if (px < S.W && py < S.H) {
        uint32_t c = kClearColor;
        float z = 1.0f;
        if (key != kInitKey) {
          const uint32_t rank = ~(uint32_t)key - 1u;
          z = __uint_as_float((uint32_t)(key >> 32) ^ 0x80000000u);
          const uint32_t id = rank_to_id(rank, (uint32_t)S.N, (uint32_t)S.nVS);
          c = shade_winner(S, a.setup[S.tri_base + id], px, py);
        }
        const size_t idx = (size_t)py * S.W + px;
        S.fb[idx] = c;
        S.depth[idx] = z;
      }
    }
    group_sync<GS>(grp);
  }
  // fragment count: one atomic per warp
  covered = __reduce_add_sync(kFull, covered);
  if (lane == 0 && covered) atomicAdd(&a.ctr->covered, (unsigned long long)covered);
}

// Large triangles (many tiles in their box) are walked by whole CTAs instead
// of one warp lane each.
template <bool SCATTER>
__global__ void __launch_bounds__(256) raster_large(RasterFrameArgs a)
{
  const uint32_t n = min(a.ctr->large_count, a.n_tris_total);
  for (uint32_t li = blockIdx.x; li < n; li += gridDim.x) {
    const uint32_t g = a.large[li];
    const TriSetup r = a.setup[g];
    const int s = find_base(a.scenes, a.n_scenes, g, false);
    WalkTri w;
    uint32_t ntiles = 0;
    fill_walk(a, a.scenes[s], r, g, w, ntiles);
    for (uint32_t j = threadIdx.x; j < ntiles; j += blockDim.x) {
      const int tx = w.tx1 + (int)(j % (uint32_t)w.tw), ty = w.ty1 + (int)(j / (uint32_t)w.tw);
      if (!tile_may_cover(w, tx, ty, a.tile)) continue;
      const uint32_t key = w.tile_base + (uint32_t)(ty * w.tiles_x + tx);
      if (!SCATTER) {
        atomicAdd(&a.tile_cnt[key], 1u);
      } else {
        const uint32_t slot = atomicAdd(&a.tile_cursor[key], 1u);
        if (slot < a.list_cap) a.tile_list[slot] = g;
      }
    }
  }
}

// ------------------------------------------------------------------ launch
struct RasterLaunchInfo {
  int persistent_ctas;
};

int raster_scan_blocks(uint32_t n_tiles) { return (int)((n_tiles + kScanTile - 1) / kScanTile); }

static int raster_ctas_hint(const RasterFrameArgs& a) { return a.large_blocks > 0 ? a.large_blocks : 296; }

cudaError_t launch_raster_frame(const RasterFrameArgs& a, int raster_ctas, cudaStream_t st, cudaEvent_t* ev)
{
  const int tri_blocks = (int)((a.n_tris_total + 255) / 256);
  if (ev) cudaEventRecord(ev[0], st);
  const int large_blocks = raster_ctas_hint(a);
  if (tri_blocks) raster_setup<<<tri_blocks, 256, 0, st>>>(a);
  if (tri_blocks) raster_large<false><<<large_blocks, 256, 0, st>>>(a);
  if (ev) cudaEventRecord(ev[1], st);
  scan_tiles<<<raster_scan_blocks(a.n_tiles_total), kScanThreads, 0, st>>>(a);
  if (ev) cudaEventRecord(ev[2], st);
  if (tri_blocks) raster_scatter<<<tri_blocks, 256, 0, st>>>(a);
  if (tri_blocks) raster_large<true><<<large_blocks, 256, 0, st>>>(a);
  if (ev) cudaEventRecord(ev[3], st);
  switch (a.tile) {
    case 8: raster_tiles<8><<<raster_ctas, 256, 0, st>>>(a); break;
    case 32: raster_tiles<32><<<raster_ctas, 256, 0, st>>>(a); break;
    default: raster_tiles<16><<<raster_ctas, 256, 0, st>>>(a); break;
  }
  if (ev) cudaEventRecord(ev[4], st);
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
    case 8: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, raster_tiles<8>, 256, 0);
    case 32: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, raster_tiles<32>, 256, 0);
    default: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, raster_tiles<16>, 256, 0);
  }
}

}  // namespace piko
