// Reyes pipeline for sm_100a: the reference's ReyesPipe (SplitStage with its
// self loop -> DiceStage -> ShadeStage -> PikoScreen, pikoc/samples/reyesPipe)
// off a device work queue:
//
//   reyes_seed / reyes_split_level  one launch per split level (bounded by the
//       split limit), a thread per patch: project the 16 control points, measure
//       the u/v screen extents, split at the halves (de Casteljau) or emit a
//       leaf with its dice grid (R11, split.pikostage:240-343).  Children and
//       leaves are appended with atomics; no host round trip between levels
//       (the reference copies the Split stage back to the host every level).
//   reyes_dice     a thread per micropolygon: four patch evaluations with
//       normals, projection, the corner-averaged "Phong" colour and the mean
//       depth (R12, dice.pikostage:159-312; R13 colour, shade.pikostage:64-109),
//       then the 64-pixel Shade-bin range of three corners (shade.pikostage:51-56)
//       and a warp-aggregated count per screen tile.
//   scan + reyes_scatter  the raster path's tile-list compaction.
//   reyes_tiles    persistent tile kernel: per pixel the reference's pixel-centre
//       sample (both windings, shade.pikostage:161-235) and depth test.
//
// Order independence.  The reference resolves depth with
//   while (remote > z) remote = atomicMin(bits, z);  pass iff zbuf == z
// in the order Dice bins, leaves and grid points are processed.  Run
// sequentially that keeps, per pixel, the minimum depth m, the depth bits of
// the FIRST fragment with depth == m and the colour of the LAST one.  Every
// micropolygon carries a 64-bit key that sorts like the reference's processing
// order -- (Dice bin, split level, position in the level, grid index) -- so
// the kernels may visit fragments in any order.
#include "runtime_internal.h"

namespace piko {

cudaError_t launch_scan_tiles(const RasterFrameArgs& a, cudaStream_t st);

constexpr unsigned kFullR = 0xffffffffu;

struct __align__(16) PatchRec {
  float4 cp[16];
  uint32_t i0;          // input patch index
  uint32_t level;       // split level = numSplits
  unsigned long long s; // position key inside the level: children of s are 2s, 2s+1
  uint32_t nu, nv;      // dice grid (leaves)
  uint32_t upbase;      // first micropolygon (leaves)
  uint32_t pad;
};
static_assert(sizeof(PatchRec) == 288, "PatchRec layout");

struct __align__(16) UpolyRec {
  float sx[4], sy[4];   // screen x, y of the 4 corners
  float z;              // mean corner depth
  uint32_t color;       // ABGR
  unsigned long long key;  // processing-order key + 1
  uint32_t tx, ty;      // tile rectangle: lo | hi << 16 (empty: lo > hi)
  float bminx, bminy, bmaxx, bmaxy;  // floor/ceil of the 4-corner bounds
  uint32_t pad[2];
};
static_assert(sizeof(UpolyRec) == 80, "UpolyRec layout");

struct ReyesCounters {
  FrameCounters fc;
  uint32_t level_count[40];
  unsigned long long leaf_meta;   // (leaves << 40) | micropolygons
  uint32_t levels_run;
  uint32_t negative_depth;
  uint32_t pad[4];
};

struct ReyesArgs {
  int W, H, nBx, nBy, nDice, tiles_x, tiles_y, tile;
  int P;
  float vp[16];
  float thr;
  int max_splits, grid;
  const float4* in_patches;
  PatchRec* lvl[2];
  uint32_t lvl_cap;
  PatchRec* leaves;
  uint32_t leaf_cap;
  UpolyRec* up;
  uint32_t up_cap;
  uint32_t* tile_cnt;
  uint32_t* tile_off;
  uint32_t* tile_list;
  uint32_t list_cap;
  uint32_t* tile_cursor;
  uint32_t* heavy;
  uint32_t heavy_threshold;
  uint32_t n_tiles;
  ReyesCounters* ctr;
  uint32_t* fb;
  float* depth;
};

__device__ __forceinline__ float4 f4add(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 f4mul(float4 a, float k) { return make_float4(a.x * k, a.y * k, a.z * k, a.w * k); }

// piko::matmultfloat4 with a w component (piko/math.h:395-403)
__device__ __forceinline__ float4 matmul4(const float* m, float4 v)
{
  float4 o;
  o.x = m[0] * v.x + m[4] * v.y + m[8] * v.z + m[12] * v.w;
  o.y = m[1] * v.x + m[5] * v.y + m[9] * v.z + m[13] * v.w;
  o.z = m[2] * v.x + m[6] * v.y + m[10] * v.z + m[14] * v.w;
  o.w = m[3] * v.x + m[7] * v.y + m[11] * v.z + m[15] * v.w;
  return o;
}

__device__ __forceinline__ float dist2(float ax, float ay, float bx, float by)
{
  const float cx = ax - bx, cy = ay - by;
  return sqrtf(cx * cx + cy * cy);
}

__device__ __forceinline__ int pow2roundup(int x)
{
  if (x < 0) return 0;
  --x;
  x |= x >> 1; x |= x >> 2; x |= x >> 4; x |= x >> 8; x |= x >> 16;
  return x + 1;
}

__device__ __forceinline__ int cvt_i32_x86_d(double d)
{
  return (d >= -2147483648.0 && d < 2147483648.0) ? __double2int_rz(d) : INT32_MIN;
}

// splitU / splitV (split.pikostage:95-224)
__device__ __forceinline__ void split_uv(const float4* cp, float4* a, float4* b, bool along_u)
{
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int c0 = along_u ? i * 4 : i, st = along_u ? 1 : 4;
    const int c1 = c0 + st, c2 = c0 + 2 * st, c3 = c0 + 3 * st;
    a[c0] = cp[c0];
    b[c3] = cp[c3];
    a[c1] = f4mul(f4add(cp[c0], cp[c1]), 0.5f);
    b[c2] = f4mul(f4add(cp[c2], cp[c3]), 0.5f);
    const float4 t = f4mul(f4add(cp[c1], cp[c2]), 0.5f);
    a[c2] = f4mul(f4add(a[c1], t), 0.5f);
    b[c1] = f4mul(f4add(b[c2], t), 0.5f);
    a[c3] = f4mul(f4add(a[c2], b[c1]), 0.5f);
    b[c0] = a[c3];
  }
}

__global__ void __launch_bounds__(256) reyes_seed(ReyesArgs a)
{
  const uint32_t i = blockIdx.x * 256u + threadIdx.x;
  if (i == 0) a.ctr->level_count[0] = (uint32_t)min(a.P, (int)a.lvl_cap);
  if (i >= (uint32_t)a.P || i >= a.lvl_cap) return;
  PatchRec& r = a.lvl[0][i];
#pragma unroll
  for (int k = 0; k < 16; ++k) r.cp[k] = a.in_patches[(size_t)i * 16 + k];
  r.i0 = i;
  r.level = 0;
  r.s = i;
  r.nu = r.nv = r.upbase = 0;
}

__global__ void __launch_bounds__(256) reyes_split_level(ReyesArgs a, int L)
{
  const uint32_t count = min(a.ctr->level_count[L], a.lvl_cap);
  const PatchRec* in = a.lvl[L & 1];
  PatchRec* out = a.lvl[(L + 1) & 1];
  if (count && blockIdx.x == 0 && threadIdx.x == 0) atomicMax(&a.ctr->levels_run, (uint32_t)L + 1u);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    float4 cp[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) cp[k] = in[i].cp[k];
    const uint32_t i0 = in[i].i0;
    const unsigned long long s = in[i].s;
    float cx[16], cy[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      float4 c = matmul4(a.vp, cp[k]);
      if (c.w == 0.0f) c.w = 1.0f;
      c.x = c.x / c.w;
      c.y = c.y / c.w;
      cx[k] = (float)(((double)c.x + 1.0) * 0.5 * (double)a.W);
      cy[k] = (float)(((double)c.y + 1.0) * 0.5 * (double)a.H);
    }
    float ue = 0.0f, ve = 0.0f;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const float su = dist2(cx[4 * r], cy[4 * r], cx[4 * r + 1], cy[4 * r + 1]) +
                       dist2(cx[4 * r + 1], cy[4 * r + 1], cx[4 * r + 2], cy[4 * r + 2]) +
                       dist2(cx[4 * r + 2], cy[4 * r + 2], cx[4 * r + 3], cy[4 * r + 3]);
      ue = std_maxf(ue, su);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const float sv = dist2(cx[c], cy[c], cx[c + 4], cy[c + 4]) + dist2(cx[c + 4], cy[c + 4], cx[c + 8], cy[c + 8]) +
                       dist2(cx[c + 8], cy[c + 8], cx[c + 12], cy[c + 12]);
      ve = std_maxf(ve, sv);
    }
    bool split = (ue >= a.thr) || (ve >= a.thr);
    if (L >= a.max_splits) split = false;
    if (split) {
      const uint32_t slot = atomicAdd(&a.ctr->level_count[L + 1], 2u);
      if (slot + 1 < a.lvl_cap) {
        float4 c1[16], c2[16];
        split_uv(cp, c1, c2, ue >= a.thr);
        PatchRec& o1 = out[slot];
        PatchRec& o2 = out[slot + 1];
#pragma unroll
        for (int k = 0; k < 16; ++k) { o1.cp[k] = c1[k]; o2.cp[k] = c2[k]; }
        o1.i0 = o2.i0 = i0;
        o1.level = o2.level = (uint32_t)L + 1;
        o1.s = 2 * s;
        o2.s = 2 * s + 1;
        o1.nu = o1.nv = o1.upbase = o2.nu = o2.nv = o2.upbase = 0;
      } else {
        atomicOr(&a.ctr->fc.status, kStatusPatchOverflow);
      }
    } else {
      int nu = pow2roundup(cvt_i32_x86_d(ceil((double)(ue / a.thr))) + 1);
      int nv = pow2roundup(cvt_i32_x86_d(ceil((double)(ve / a.thr))) + 1);
      nu = nu < 2 ? 2 : (nu > 32 ? 32 : nu);
      nv = nv < 2 ? 2 : (nv > 32 ? 32 : nv);
      if (a.grid > 0) { nu = a.grid; nv = a.grid; }
      const unsigned long long nup = (unsigned long long)(nu + 1) * (unsigned long long)(nv + 1);
      const unsigned long long meta = atomicAdd(&a.ctr->leaf_meta, (1ull << 40) | nup);
      const uint32_t slot = (uint32_t)(meta >> 40);
      if (slot < a.leaf_cap) {
        PatchRec& o = a.leaves[slot];
#pragma unroll
        for (int k = 0; k < 16; ++k) o.cp[k] = cp[k];
        o.i0 = i0;
        o.level = (uint32_t)L;
        o.s = s;
        o.nu = (uint32_t)nu;
        o.nv = (uint32_t)nv;
        o.upbase = (uint32_t)(meta & ((1ull << 40) - 1));
      } else {
        atomicOr(&a.ctr->fc.status, kStatusPatchOverflow);
      }
    }
  }
}

// ------------------------------------------------------------------ dice
__device__ __forceinline__ float B0(float u) { return ((1.0f - u) * (1.0f - u) * (1.0f - u)); }
__device__ __forceinline__ float B1(float u) { return ((3.0f * u) * (1.0f - u) * (1.0f - u)); }
__device__ __forceinline__ float B2(float u) { return ((3.0f * u) * (u - u * u)); }
__device__ __forceinline__ float B3(float u) { return ((u) * (u * u)); }
__device__ __forceinline__ float dB0(float u) { return (-3.0f * (1.0f - u) * (1.0f - u)); }
__device__ __forceinline__ float dB1(float u) { return (3.0f * (1.0f - u) * (1.0f - 3.0f * u)); }
__device__ __forceinline__ float dB2(float u) { return (3.0f * u * (2.0f - 3.0f * u)); }
__device__ __forceinline__ float dB3(float u) { return (3.0f * u * u); }

__device__ __forceinline__ float4 bez(float t, float4 a, float4 b, float4 c, float4 d)
{
  float4 o;
  o.x = B0(t) * a.x + B1(t) * b.x + B2(t) * c.x + B3(t) * d.x;
  o.y = B0(t) * a.y + B1(t) * b.y + B2(t) * c.y + B3(t) * d.y;
  o.z = B0(t) * a.z + B1(t) * b.z + B2(t) * c.z + B3(t) * d.z;
  o.w = B0(t) * a.w + B1(t) * b.w + B2(t) * c.w + B3(t) * d.w;
  return o;
}
__device__ __forceinline__ float4 dbez(float t, float4 a, float4 b, float4 c, float4 d)
{
  float4 o;
  o.x = dB0(t) * a.x + dB1(t) * b.x + dB2(t) * c.x + dB3(t) * d.x;
  o.y = dB0(t) * a.y + dB1(t) * b.y + dB2(t) * c.y + dB3(t) * d.y;
  o.z = dB0(t) * a.z + dB1(t) * b.z + dB2(t) * c.z + dB3(t) * d.z;
  o.w = dB0(t) * a.w + dB1(t) * b.w + dB2(t) * c.w + dB3(t) * d.w;
  return o;
}

// patchEval + normEval + projection of one corner (dice.pikostage:111-146,205-220)
__device__ __forceinline__ void dice_corner(const float4* P, const ReyesArgs& a, float u, float v, float& sx, float& sy,
                                            float& sz, float& nx, float& ny, float& nz)
{
  const float4 r0 = bez(u, P[0], P[1], P[2], P[3]), r1 = bez(u, P[4], P[5], P[6], P[7]);
  const float4 r2 = bez(u, P[8], P[9], P[10], P[11]), r3 = bez(u, P[12], P[13], P[14], P[15]);
  const float4 pt = bez(v, r0, r1, r2, r3);
  const float4 d0 = dbez(u, P[0], P[1], P[2], P[3]), d1 = dbez(u, P[4], P[5], P[6], P[7]);
  const float4 d2 = dbez(u, P[8], P[9], P[10], P[11]), d3 = dbez(u, P[12], P[13], P[14], P[15]);
  const float4 v1 = bez(v, d0, d1, d2, d3);
  const float4 v2 = dbez(v, r0, r1, r2, r3);
  float cx = v1.y * v2.z - v1.z * v2.y;
  float cy = v1.z * v2.x - v1.x * v2.z;
  float cz = v1.x * v2.y - v1.y * v2.x;
  const float mag = sqrtf(cx * cx + cy * cy + cz * cz);
  nx = cx / mag; ny = cy / mag; nz = cz / mag;
  const float4 ss = matmul4(a.vp, pt);
  const float onebyw = 1.0f / ss.w;
  sx = (ss.x * onebyw + 1.0f) * (float)a.W * 0.5f;
  sy = (ss.y * onebyw + 1.0f) * (float)a.H * 0.5f;
  sz = (ss.z * onebyw);
}

// phongShadeReyes + computeLighting as called (shade.pikostage:22-30,64-85):
// negated normal; the dot product takes matcol, the scale takes lightvec
__device__ __forceinline__ float phong_channel(float nx, float ny, float nz, int ch)
{
  nx = -nx; ny = -ny; nz = -nz;
  float d = nx * 0.10f + ny * 0.35f + nz * 0.85f;
  d = d < 0.0f ? 0.0f : d;
  const float lv = ch == 0 ? 0.1773f : (ch == 1 ? 0.5773f : 0.973f);
  const float o = 0.2f + d * lv;
  return o > 1.0f ? 1.0f : (o < 0.0f ? 0.0f : o);
}

__device__ __forceinline__ double std_min_d(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double std_max_d(double a, double b) { return (a < b) ? b : a; }

__device__ __forceinline__ uint32_t find_leaf(const PatchRec* leaves, uint32_t n, uint32_t u)
{
  uint32_t lo = 0, hi = n - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (leaves[mid].upbase <= u) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Tile walk of micropolygons: each lane has a (usually one-tile) rectangle;
// lanes hitting the same tile aggregate their atomic.
template <bool SCATTER>
__device__ __forceinline__ void walk_upoly_tiles(const ReyesArgs& a, uint32_t tx, uint32_t ty, uint32_t uidx)
{
  const int lane = threadIdx.x & 31;
  int x1 = (int)(tx & 0xffff), x2 = (int)(tx >> 16), y1 = (int)(ty & 0xffff), y2 = (int)(ty >> 16);
  const int w = x2 >= x1 ? x2 - x1 + 1 : 0;
  const int n = (y2 >= y1 && w) ? w * (y2 - y1 + 1) : 0;
  const int nmax = __reduce_max_sync(kFullR, (unsigned)n);
  for (int k = 0; k < nmax; ++k) {
    uint32_t key = 0xffffffffu;
    if (k < n) key = (uint32_t)((y1 + k / w) * a.tiles_x + (x1 + k % w));
    const unsigned peers = __match_any_sync(kFullR, key);
    if (key == 0xffffffffu) continue;
    const int leader = __ffs(peers) - 1;
    if (!SCATTER) {
      if (lane == leader) atomicAdd(&a.tile_cnt[key], (uint32_t)__popc(peers));
    } else {
      uint32_t b = 0;
      if (lane == leader) b = atomicAdd(&a.tile_cursor[key], (uint32_t)__popc(peers));
      b = __shfl_sync(peers, b, leader);
      const uint32_t slot = b + __popc(peers & ((1u << lane) - 1u));
      if (slot < a.list_cap) a.tile_list[slot] = uidx;
    }
  }
}

__global__ void __launch_bounds__(256) reyes_dice(ReyesArgs a)
{
  const unsigned long long meta = a.ctr->leaf_meta;
  const uint32_t nleaf = (uint32_t)min((unsigned long long)a.leaf_cap, meta >> 40);
  unsigned long long total = meta & ((1ull << 40) - 1);
  if (total > a.up_cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&a.ctr->fc.status, kStatusUpolyOverflow);
    total = a.up_cap;
  }
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t rounds = (uint32_t)((total + stride - 1) / stride);
  for (uint32_t r = 0; r < rounds; ++r) {
    const uint32_t u = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t tx = 0xffff, ty = 0xffff;  // empty rectangles
    if (u < total && nleaf) {
      const uint32_t li = find_leaf(a.leaves, nleaf, u);
      const PatchRec& p = a.leaves[li];
      const uint32_t local = u - p.upbase;
      const uint32_t nv1 = p.nv + 1;
      if (local < (p.nu + 1) * nv1) {
        const int k = (int)(local / nv1), j = (int)(local % nv1);
        float4 P[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) P[q] = p.cp[q];
        const float du = 1.0f / ((float)p.nu), dv = 1.0f / ((float)p.nv);
        const float myU = (float)k * du, myV = (float)j * dv;
        UpolyRec o;
        float nx[4], ny[4], nz[4], sz[4];
        dice_corner(P, a, myU, myV, o.sx[0], o.sy[0], sz[0], nx[0], ny[0], nz[0]);
        dice_corner(P, a, myU + du, myV, o.sx[1], o.sy[1], sz[1], nx[1], ny[1], nz[1]);
        dice_corner(P, a, myU + du, myV + dv, o.sx[2], o.sy[2], sz[2], nx[2], ny[2], nz[2]);
        dice_corner(P, a, myU, myV + dv, o.sx[3], o.sy[3], sz[3], nx[3], ny[3], nz[3]);
        o.z = ((sz[0] + sz[1] + sz[2] + sz[3])) * 0.25f;
        float col[3];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
          float c = phong_channel(nx[0], ny[0], nz[0], ch) + phong_channel(nx[1], ny[1], nz[1], ch);
          c = c + phong_channel(nx[2], ny[2], nz[2], ch);
          c = c + phong_channel(nx[3], ny[3], nz[3], ch);
          col[ch] = std_minf(c, 4.0f) * 0.25f;
        }
        o.color = (255u << 24) | (cvt_u32_x86(col[2] * 255.0f) << 16) | (cvt_u32_x86(col[1] * 255.0f) << 8) |
                  cvt_u32_x86(col[0] * 255.0f);
        const uint32_t L = p.level;
        const uint32_t id = p.i0 + L * (L + 1) / 2;
        const unsigned long long d = (unsigned long long)((id / 128u) % (uint32_t)a.nDice);
        o.key = ((d << 52) | ((unsigned long long)L << 47) | (p.s << 12) | (unsigned long long)local) + 1ull;
        // Shade bins of corners 0..2 (computeBoundingBox + assignToBB, dice.pikostage:18-43)
        const float lox = floorf((float)std_min_d(o.sx[0], std_min_d(o.sx[1], o.sx[2])));
        const float loy = floorf((float)std_min_d(o.sy[0], std_min_d(o.sy[1], o.sy[2])));
        const float hix = ceilf((float)std_max_d(o.sx[0], std_max_d(o.sx[1], o.sx[2])));
        const float hiy = ceilf((float)std_max_d(o.sy[0], std_max_d(o.sy[1], o.sy[2])));
        int bx1 = cvt_i32_x86(floorf(lox / 64.0f)), bx2 = cvt_i32_x86(floorf(hix / 64.0f));
        int by1 = cvt_i32_x86(floorf(loy / 64.0f)), by2 = cvt_i32_x86(floorf(hiy / 64.0f));
        if (bx1 < 0) bx1 = 0;
        if (by1 < 0) by1 = 0;
        if (bx2 >= a.nBx) bx2 = a.nBx - 1;
        if (by2 >= a.nBy) by2 = a.nBy - 1;
        // 4-corner bounds (shade.pikostage:129-140)
        o.bminx = floorf(std_minf(std_minf(o.sx[0], o.sx[1]), std_minf(o.sx[2], o.sx[3])));
        o.bminy = floorf(std_minf(std_minf(o.sy[0], o.sy[1]), std_minf(o.sy[2], o.sy[3])));
        o.bmaxx = ceilf(std_maxf(std_maxf(o.sx[0], o.sx[1]), std_maxf(o.sx[2], o.sx[3])));
        o.bmaxy = ceilf(std_maxf(std_maxf(o.sy[0], o.sy[1]), std_maxf(o.sy[2], o.sy[3])));
        if (bx1 <= bx2 && by1 <= by2) {
          const float fx0 = (float)(bx1 * 64), fx1 = (float)((bx2 + 1) * 64);
          const float fy0 = (float)(by1 * 64), fy1 = (float)((by2 + 1) * 64);
          int px0 = cvt_i32_x86((o.bminx > fx0) ? o.bminx : fx0);
          int px1 = cvt_i32_x86((o.bmaxx < fx1) ? o.bmaxx : fx1);
          int py0 = cvt_i32_x86((o.bminy > fy0) ? o.bminy : fy0);
          int py1 = cvt_i32_x86((o.bmaxy < fy1) ? o.bmaxy : fy1);
          px0 = max(px0, bx1 * 64); py0 = max(py0, by1 * 64);
          px1 = min(px1, (bx2 + 1) * 64); py1 = min(py1, (by2 + 1) * 64);
          if (px0 < px1 && py0 < py1) {
            tx = (uint32_t)(px0 / a.tile) | ((uint32_t)((px1 - 1) / a.tile) << 16);
            ty = (uint32_t)(py0 / a.tile) | ((uint32_t)((py1 - 1) / a.tile) << 16);
          }
        }
        o.tx = tx;
        o.ty = ty;
        o.pad[0] = o.pad[1] = 0;
        const uint4* src = reinterpret_cast<const uint4*>(&o);
        uint4* dst = reinterpret_cast<uint4*>(&a.up[u]);
#pragma unroll
        for (int q = 0; q < 5; ++q) dst[q] = src[q];
        if (o.z < 0.0f) atomicAdd(&a.ctr->negative_depth, 1u);
      }
    }
    walk_upoly_tiles<false>(a, tx, ty, u);
  }
}

__global__ void __launch_bounds__(256) reyes_scatter(ReyesArgs a)
{
  unsigned long long total = a.ctr->leaf_meta & ((1ull << 40) - 1);
  if (total > a.up_cap) total = a.up_cap;
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t rounds = (uint32_t)((total + stride - 1) / stride);
  for (uint32_t r = 0; r < rounds; ++r) {
    const uint32_t u = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t tx = 0xffff, ty = 0xffff;
    if (u < total) {
      tx = a.up[u].tx;
      ty = a.up[u].ty;
    }
    walk_upoly_tiles<true>(a, tx, ty, u);
  }
}

// ------------------------------------------------------------------ shade tiles
struct TileUpoly {
  float sx[4], sy[4];
  float z;
  uint32_t color;
  unsigned long long key;
  int32_t rx0, rx1, ry0, ry1;   // tile-local pixel rectangle [rx0, rx1) x [ry0, ry1)
};

template <int GS>
__device__ __forceinline__ void rgroup_sync(int grp)
{
  if constexpr (GS == 256) {
    __syncthreads();
  } else if constexpr (GS >= 32) {
    asm volatile("bar.sync %0, %1;" ::"r"(grp + 1), "r"(GS) : "memory");
  } else {
    const unsigned m = ((1u << GS) - 1u) << ((threadIdx.x & 31) & ~(GS - 1));
    __syncwarp(m);
  }
}

__device__ __forceinline__ uint32_t reyes_next_tile(const ReyesArgs& a)
{
  const uint32_t heavy_n = a.ctr->fc.heavy_count;
  for (;;) {
    const uint32_t w = atomicAdd(&a.ctr->fc.work_next, 1u);
    if (w < heavy_n) return a.heavy[w];
    const uint32_t t = w - heavy_n;
    if (t >= a.n_tiles) return 0xffffffffu;
    if (a.tile_cnt[t] > a.heavy_threshold) continue;
    return t;
  }
}

template <int T>
__global__ void __launch_bounds__(256) reyes_tiles(ReyesArgs a)
{
  constexpr int Q = T / 2;
  constexpr int GS = Q * Q;
  constexpr int NG = 256 / GS;
  __shared__ TileUpoly s_up[256];
  __shared__ uint32_t s_tile[NG];
  const int grp = threadIdx.x / GS;
  const int q = threadIdx.x % GS;
  const int ox = 2 * (q % Q), oy = 2 * (q / Q);
  TileUpoly* st = s_up + grp * GS;
  unsigned covered = 0;
  for (;;) {
    if (q == 0) s_tile[grp] = reyes_next_tile(a);
    rgroup_sync<GS>(grp);
    const uint32_t tile = s_tile[grp];
    rgroup_sync<GS>(grp);
    if (tile == 0xffffffffu) break;
    const int X0 = (int)(tile % (uint32_t)a.tiles_x) * T, Y0 = (int)(tile / (uint32_t)a.tiles_x) * T;
    const float bbx = (float)((X0 / 64) * 64), bby = (float)((Y0 / 64) * 64);
    float bz[4];
    uint32_t bits_first[4], col[4];
    unsigned long long kfirst[4], klast[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      bz[k] = 1.0f; bits_first[k] = 0x3f800000u; col[k] = kClearColor; kfirst[k] = 0; klast[k] = 0;
    }
    const uint32_t off = a.tile_off[tile];
    uint32_t cnt = a.tile_off[tile + 1] - off;
    if (off + cnt > a.list_cap) cnt = off < a.list_cap ? a.list_cap - off : 0;
    for (uint32_t b0 = 0; b0 < cnt; b0 += GS) {
      if (b0 + q < cnt) {
        const UpolyRec& u = a.up[a.tile_list[off + b0 + q]];
        TileUpoly& t = st[q];
#pragma unroll
        for (int c = 0; c < 4; ++c) { t.sx[c] = u.sx[c]; t.sy[c] = u.sy[c]; }
        t.z = u.z;
        t.color = u.color;
        t.key = u.key;
        // intersectBBi of the 4-corner bounds with this tile's Shade bin
        t.rx0 = cvt_i32_x86((u.bminx > bbx) ? u.bminx : bbx) - X0;
        t.rx1 = cvt_i32_x86((u.bmaxx < bbx + 64.0f) ? u.bmaxx : bbx + 64.0f) - X0;
        t.ry0 = cvt_i32_x86((u.bminy > bby) ? u.bminy : bby) - Y0;
        t.ry1 = cvt_i32_x86((u.bmaxy < bby + 64.0f) ? u.bmaxy : bby + 64.0f) - Y0;
      }
      rgroup_sync<GS>(grp);
      const int n = (int)min((uint32_t)GS, cnt - b0);
      for (int i = 0; i < n; ++i) {
        const TileUpoly& t = st[i];
        if (ox + 1 < t.rx0 || ox >= t.rx1 || oy + 1 < t.ry0 || oy >= t.ry1) continue;
        const float* X = t.sx;
        const float* Y = t.sy;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int lx = ox + (k & 1), ly = oy + (k >> 1);
          if (lx < t.rx0 || lx >= t.rx1 || ly < t.ry0 || ly >= t.ry1) continue;
          const float px = (float)(X0 + lx) + 0.5f, py = (float)(Y0 + ly) + 0.5f;
          bool r1 = true, r2 = true;
          if (((py - Y[0]) * (X[1] - X[0]) - (px - X[0]) * (Y[1] - Y[0])) <= 0.0f) r1 = false;
          if (((py - Y[1]) * (X[2] - X[1]) - (px - X[1]) * (Y[2] - Y[1])) <= 0.0f) r1 = false;
          if (((py - Y[2]) * (X[3] - X[2]) - (px - X[2]) * (Y[3] - Y[2])) <= 0.0f) r1 = false;
          if (((py - Y[3]) * (X[0] - X[3]) - (px - X[3]) * (Y[0] - Y[3])) <= 0.0f) r1 = false;
          if (((py - Y[0]) * (X[3] - X[0]) - (px - X[0]) * (Y[3] - Y[0])) <= 0.0f) r2 = false;
          if (((py - Y[3]) * (X[2] - X[3]) - (px - X[3]) * (Y[2] - Y[3])) <= 0.0f) r2 = false;
          if (((py - Y[2]) * (X[1] - X[2]) - (px - X[2]) * (Y[1] - Y[2])) <= 0.0f) r2 = false;
          if (((py - Y[1]) * (X[0] - X[1]) - (px - X[1]) * (Y[0] - Y[1])) <= 0.0f) r2 = false;
          if (!(r1 || r2)) continue;
          ++covered;
          const float z = t.z;
          if (!(z <= bz[k])) continue;
          if (z < bz[k]) {
            bz[k] = z; klast[k] = t.key; col[k] = t.color; kfirst[k] = t.key; bits_first[k] = __float_as_uint(z);
          } else {
            if (t.key > klast[k]) { klast[k] = t.key; col[k] = t.color; }
            if (t.key < kfirst[k]) { kfirst[k] = t.key; bits_first[k] = __float_as_uint(z); }
          }
        }
      }
      rgroup_sync<GS>(grp);
    }
#pragma unroll
    for (int ky = 0; ky < 2; ++ky) {
      const int py = Y0 + oy + ky;
      if (py >= a.H) continue;
#pragma unroll
      for (int kx = 0; kx < 2; ++kx) {
        const int px = X0 + ox + kx;
        if (px >= a.W) continue;
        const size_t idx = (size_t)py * a.W + px;
        a.fb[idx] = col[ky * 2 + kx];
        a.depth[idx] = __uint_as_float(bits_first[ky * 2 + kx]);
      }
    }
  }
  covered = __reduce_add_sync(kFullR, covered);
  if ((threadIdx.x & 31) == 0 && covered) atomicAdd(&a.ctr->fc.covered, (unsigned long long)covered);
}

cudaError_t launch_reyes_frame(const ReyesArgs& a, const RasterFrameArgs& scan, int sms, cudaStream_t st,
                               cudaEvent_t* ev)
{
  if (ev) cudaEventRecord(ev[0], st);
  reyes_seed<<<(a.P + 255) / 256 + 1, 256, 0, st>>>(a);
  const int grid = sms * 8;
  for (int L = 0; L <= a.max_splits; ++L) reyes_split_level<<<grid, 256, 0, st>>>(a, L);
  if (ev) cudaEventRecord(ev[1], st);
  reyes_dice<<<grid, 256, 0, st>>>(a);
  if (ev) cudaEventRecord(ev[2], st);
  cudaError_t e = launch_scan_tiles(scan, st);
  if (e) return e;
  reyes_scatter<<<grid, 256, 0, st>>>(a);
  if (ev) cudaEventRecord(ev[3], st);
  int per_sm = 1;
  if (a.tile == 32) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reyes_tiles<32>, 256, 0);
    reyes_tiles<32><<<sms * max(per_sm, 1), 256, 0, st>>>(a);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reyes_tiles<16>, 256, 0);
    reyes_tiles<16><<<sms * max(per_sm, 1), 256, 0, st>>>(a);
  }
  if (ev) cudaEventRecord(ev[4], st);
  return cudaGetLastError();
}

}  // namespace piko

using namespace piko;

// ------------------------------------------------------------------ host state
struct ReyesState {
  PatchRec* lvl[2] = {nullptr, nullptr};
  PatchRec* leaves = nullptr;
  UpolyRec* up = nullptr;
  uint32_t lvl_cap = 0, leaf_cap = 0, up_cap = 0;
  uint32_t* tile_cnt = nullptr;
  uint32_t* tile_off = nullptr;
  uint32_t* tile_cursor = nullptr;
  uint32_t* tile_list = nullptr;
  uint32_t* heavy = nullptr;
  uint32_t list_cap = 0, n_tiles = 0;
  unsigned long long* scan_flags = nullptr;
  ReyesCounters* ctr = nullptr;
  ReyesCounters* h_ctr = nullptr;
  cudaEvent_t ev[5] = {};
  bool ev_made = false;
  int tile = 16;
};

void piko_reyes_release(piko_scene* s)
{
  ReyesState* r = s->reyes;
  if (!r) return;
  dfree(r->lvl[0]); dfree(r->lvl[1]); dfree(r->leaves); dfree(r->up);
  dfree(r->tile_cnt); dfree(r->tile_off); dfree(r->tile_cursor); dfree(r->tile_list); dfree(r->heavy);
  dfree(r->scan_flags); dfree(r->ctr);
  if (r->h_ctr) cudaFreeHost(r->h_ctr);
  if (r->ev_made) for (auto& e : r->ev) cudaEventDestroy(e);
  delete r;
  s->reyes = nullptr;
}

static cudaError_t reyes_alloc(ReyesState* r, uint32_t lvl_cap, uint32_t leaf_cap, uint32_t up_cap, uint32_t list_cap,
                               uint32_t n_tiles)
{
  cudaError_t e = cudaSuccess;
  if (lvl_cap > r->lvl_cap) {
    dfree(r->lvl[0]); dfree(r->lvl[1]);
    if ((e = dalloc(&r->lvl[0], lvl_cap)) || (e = dalloc(&r->lvl[1], lvl_cap))) return e;
    r->lvl_cap = lvl_cap;
  }
  if (leaf_cap > r->leaf_cap) {
    dfree(r->leaves);
    if ((e = dalloc(&r->leaves, leaf_cap))) return e;
    r->leaf_cap = leaf_cap;
  }
  if (up_cap > r->up_cap) {
    dfree(r->up);
    if ((e = dalloc(&r->up, up_cap))) return e;
    r->up_cap = up_cap;
  }
  if (list_cap > r->list_cap) {
    dfree(r->tile_list);
    if ((e = dalloc(&r->tile_list, list_cap))) return e;
    r->list_cap = list_cap;
  }
  if (n_tiles > r->n_tiles) {
    dfree(r->tile_cnt); dfree(r->tile_off); dfree(r->tile_cursor); dfree(r->heavy); dfree(r->scan_flags);
    if ((e = dalloc(&r->tile_cnt, n_tiles)) || (e = dalloc(&r->tile_off, (size_t)n_tiles + 1)) ||
        (e = dalloc(&r->tile_cursor, n_tiles)) || (e = dalloc(&r->heavy, n_tiles)) ||
        (e = dalloc(&r->scan_flags, (size_t)raster_scan_blocks(n_tiles))))
      return e;
    r->n_tiles = n_tiles;
  }
  if (!r->ctr) {
    if ((e = dalloc(&r->ctr, 1))) return e;
    if ((e = cudaMallocHost((void**)&r->h_ctr, sizeof(ReyesCounters)))) return e;
    memset(r->h_ctr, 0, sizeof(ReyesCounters));
  }
  if (!r->ev_made) {
    for (auto& ev : r->ev)
      if ((e = cudaEventCreate(&ev))) return e;
    r->ev_made = true;
  }
  return cudaSuccess;
}

piko_status piko_reyes_run(piko_scene* s, cudaStream_t st, bool timed)
{
  piko_ctx* ctx = s->pipe->ctx;
  piko_pipe* p = s->pipe;
  if (!s->reyes) s->reyes = new ReyesState();
  ReyesState* r = s->reyes;
  const int T = p->tile == 32 ? 32 : 16;   // tiles must divide the 64-pixel Shade bins
  r->tile = T;
  const int tiles_x = (s->W + T - 1) / T, tiles_y = (s->H + T - 1) / T;
  const uint32_t n_tiles = (uint32_t)(tiles_x * tiles_y);
  const uint32_t P = (uint32_t)s->N;
  CU(ctx, reyes_alloc(r, std::max<uint32_t>(1u << 16, 64u * P), std::max<uint32_t>(1u << 16, 64u * P),
                      r->up_cap ? r->up_cap : (1u << 20), r->list_cap ? r->list_cap : (1u << 21), n_tiles));
  CU(ctx, cudaMemsetAsync(r->ctr, 0, sizeof(ReyesCounters), st));
  CU(ctx, cudaMemsetAsync(r->tile_cnt, 0, sizeof(uint32_t) * n_tiles, st));
  CU(ctx, cudaMemsetAsync(r->scan_flags, 0, sizeof(unsigned long long) * raster_scan_blocks(n_tiles), st));
  ReyesArgs a;
  memset(&a, 0, sizeof(a));
  a.W = s->W; a.H = s->H; a.nBx = s->W / 64; a.nBy = s->H / 64;
  a.nDice = std::max(1, a.nBx * a.nBy);
  a.tiles_x = tiles_x; a.tiles_y = tiles_y; a.tile = T;
  a.P = (int)P;
  memcpy(a.vp, s->state.view_proj, sizeof(a.vp));
  a.thr = p->split_threshold;
  a.max_splits = std::min(p->max_splits, 30);
  a.grid = p->dice_grid;
  a.in_patches = s->patches;
  a.lvl[0] = r->lvl[0]; a.lvl[1] = r->lvl[1]; a.lvl_cap = r->lvl_cap;
  a.leaves = r->leaves; a.leaf_cap = r->leaf_cap;
  a.up = r->up; a.up_cap = r->up_cap;
  a.tile_cnt = r->tile_cnt; a.tile_off = r->tile_off; a.tile_list = r->tile_list; a.list_cap = r->list_cap;
  a.tile_cursor = r->tile_cursor; a.heavy = r->heavy; a.heavy_threshold = (uint32_t)(2 * (T / 2) * (T / 2));
  a.n_tiles = n_tiles;
  a.ctr = r->ctr;
  a.fb = s->fb; a.depth = s->depth;
  RasterFrameArgs sc;
  memset(&sc, 0, sizeof(sc));
  sc.n_tiles_total = n_tiles;
  sc.tile_cnt = r->tile_cnt; sc.tile_off = r->tile_off; sc.tile_cursor = r->tile_cursor;
  sc.list_cap = r->list_cap; sc.heavy = r->heavy; sc.heavy_threshold = a.heavy_threshold;
  sc.scan_flags = r->scan_flags; sc.ctr = &r->ctr->fc;
  CU(ctx, launch_reyes_frame(a, sc, ctx->sms, st, timed ? r->ev : nullptr));
  return PIKO_OK;
}

piko_status piko_reyes_finish(piko_scene* s)
{
  piko_ctx* ctx = s->pipe->ctx;
  ReyesState* r = s->reyes;
  if (!r) { s->pending = false; return PIKO_OK; }
  for (int attempt = 0; attempt < 6; ++attempt) {
    CU(ctx, cudaMemcpyAsync(r->h_ctr, r->ctr, sizeof(ReyesCounters), cudaMemcpyDeviceToHost, s->last_stream));
    CU(ctx, cudaStreamSynchronize(s->last_stream));
    const ReyesCounters& c = *r->h_ctr;
    const uint32_t st = c.fc.status;
    if (st & kStatusScanTimeout) return set_err(ctx, PIKO_ERR_TIMEOUT, "%s", "tile scan look-back timed out");
    if (!(st & (kStatusPatchOverflow | kStatusUpolyOverflow | kStatusListOverflow))) {
      s->pending = false;
      return PIKO_OK;
    }
    uint32_t maxlvl = 0;
    for (int i = 0; i < 40; ++i) maxlvl = std::max(maxlvl, c.level_count[i]);
    const uint32_t leaves = (uint32_t)(c.leaf_meta >> 40);
    const unsigned long long ups = c.leaf_meta & ((1ull << 40) - 1);
    uint32_t lvl = r->lvl_cap, lf = r->leaf_cap, up = r->up_cap, lc = r->list_cap;
    if (st & kStatusPatchOverflow) { lvl = std::max(lvl, maxlvl + maxlvl / 2 + 1024); lf = std::max(lf, 2 * leaves + 1024); }
    if (st & kStatusUpolyOverflow) up = (uint32_t)std::min<unsigned long long>(ups + ups / 4 + 4096, 0xffffffffull);
    if (st & kStatusListOverflow) lc = c.fc.list_total + c.fc.list_total / 4 + 4096;
    CU(ctx, reyes_alloc(r, lvl, lf, up, lc, r->n_tiles));
    piko_status rr = piko_reyes_run(s, s->last_stream, s->timed);
    if (rr != PIKO_OK) return rr;
  }
  return set_err(ctx, PIKO_ERR_QUEUE_OVERFLOW, "%s", "Reyes queues kept overflowing");
}

piko_status piko_reyes_stats(piko_scene* s, piko_frame_stats* o)
{
  ReyesState* r = s->reyes;
  if (!r || !r->h_ctr) return PIKO_OK;
  piko_ctx* ctx = s->pipe->ctx;
  CU(ctx, cudaMemcpy(r->h_ctr, r->ctr, sizeof(ReyesCounters), cudaMemcpyDeviceToHost));
  const ReyesCounters& c = *r->h_ctr;
  o->prims_in = (uint64_t)s->N;
  o->prims_kept = c.leaf_meta >> 40;
  o->upolys = c.leaf_meta & ((1ull << 40) - 1);
  o->bin_entries = c.fc.list_total;
  o->covered = c.fc.covered;
  o->status = c.fc.status | (c.negative_depth ? kStatusDepthNeverSettles : 0u);
  o->split_levels = c.levels_run;
  o->n_kernels = 0;
  if (s->timed && r->ev_made) {
    o->n_kernels = 4;
    for (int i = 0; i < 4; ++i) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, r->ev[i], r->ev[i + 1]);
      o->kernel_ms[i] = ms;
    }
  }
  return PIKO_OK;
}
