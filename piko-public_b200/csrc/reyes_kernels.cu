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
//       the 64-pixel Shade-bin range of three corners (shade.pikostage:51-56)
//       cut with the four-corner bounds to one pixel rectangle, then the first
//       fragment pass over that rectangle.
//   reyes_frag<2>, reyes_frag<3>  the other two fragment passes: per pixel the
//       reference's pixel-centre sample (both windings, shade.pikostage:161-235)
//       and its depth resolve, with per-pixel atomics in HBM/L2.  Shade work is
//       spread per micropolygon, not per screen tile, so silhouette tiles where
//       thousands of micropolygons pile up cost no more than anywhere else.
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
  int32_t x0, x1, y0, y1;  // shaded pixel rectangle [x0, x1) x [y0, y1), clipped to the screen
};
static_assert(sizeof(UpolyRec) == 64, "UpolyRec layout");

struct ReyesCounters {
  FrameCounters fc;
  uint32_t level_count[40];
  unsigned long long leaf_meta;   // (leaves << 40) | micropolygons
  uint32_t levels_run;
  uint32_t negative_depth;
  uint32_t big_count;             // micropolygons shaded warp-cooperatively
  uint32_t pad[3];
};

struct ReyesArgs {
  int W, H, nBx, nBy, nDice;
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
  uint32_t* big;                  // indices of micropolygons with more than kSmallPx candidate pixels
  ReyesCounters* ctr;
  uint32_t* fb;
  float* depth;
  uint32_t* zmin;                 // per pixel: order-mapped minimum depth
  unsigned long long* kfirst;     // per pixel: least key among fragments at the minimum
  unsigned long long* klast;      // per pixel: greatest key among fragments at the minimum
};

// Micropolygons whose shaded rectangle holds more pixels than this are shaded
// by a warp (one lane per pixel) instead of by the thread that owns them.
constexpr int kSmallPx = 8;

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

// ------------------------------------------------------------------ shade
// ShadeStage's per-pixel test (shade.pikostage:161-235): the pixel centre is
// inside the micropolygon when all four edge functions are positive for either
// winding.  Every product and difference is rounded separately, as on the CPU.
__device__ __forceinline__ bool upoly_covers(const float* X, const float* Y, float px, float py)
{
  bool r1 = true, r2 = true;
  if (((py - Y[0]) * (X[1] - X[0]) - (px - X[0]) * (Y[1] - Y[0])) <= 0.0f) r1 = false;
  if (((py - Y[1]) * (X[2] - X[1]) - (px - X[1]) * (Y[2] - Y[1])) <= 0.0f) r1 = false;
  if (((py - Y[2]) * (X[3] - X[2]) - (px - X[2]) * (Y[3] - Y[2])) <= 0.0f) r1 = false;
  if (((py - Y[3]) * (X[0] - X[3]) - (px - X[3]) * (Y[0] - Y[3])) <= 0.0f) r1 = false;
  if (((py - Y[0]) * (X[3] - X[0]) - (px - X[0]) * (Y[3] - Y[0])) <= 0.0f) r2 = false;
  if (((py - Y[3]) * (X[2] - X[3]) - (px - X[3]) * (Y[2] - Y[3])) <= 0.0f) r2 = false;
  if (((py - Y[2]) * (X[1] - X[2]) - (px - X[2]) * (Y[1] - Y[2])) <= 0.0f) r2 = false;
  if (((py - Y[1]) * (X[0] - X[1]) - (px - X[1]) * (Y[0] - Y[1])) <= 0.0f) r2 = false;
  return r1 || r2;
}

// Depth order as an unsigned integer: total over non-NaN floats, with -0 and +0
// equal (the CPU compares depths as floats).
__device__ __forceinline__ uint32_t zorder(float z)
{
  uint32_t b = __float_as_uint(z);
  if (b == 0x80000000u) b = 0u;
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float zorder_inv(uint32_t o)
{
  return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}
constexpr uint32_t kZorderClear = 0xbf800000u;  // zorder(1.0f), the cleared depth

// The three fragment passes.  The CPU shades micropolygons in its processing
// order with   while (remote > z) remote = atomicMin(bits, z);  pass iff zbuf == z
// so, per pixel, the surviving depth is the minimum m (the cleared 1.0
// included), its bits come from the FIRST fragment with depth m and the colour
// from the LAST one.  Every fragment carries its micropolygon's order key;
//   pass 1  zmin  <- min over fragments of zorder(z)            (32-bit atomics)
//   pass 2  kfirst / klast <- min / max key over fragments at m  (64-bit atomics)
//   pass 3  the fragment whose key is klast writes the colour, the one whose
//           key is kfirst writes the depth bits.
// A pixel nothing reaches keeps the cleared colour and depth; a fragment at
// exactly 1.0 takes the colour but leaves the (identical) cleared depth bits.
template <int PHASE>
__device__ __forceinline__ void shade_pixel(const ReyesArgs& a, const UpolyRec& u, int x, int y, unsigned& covered)
{
  if (!upoly_covers(u.sx, u.sy, (float)x + 0.5f, (float)y + 0.5f)) return;
  const size_t p = (size_t)y * a.W + x;
  const float z = u.z;
  if (PHASE == 1) {
    ++covered;
    if (z <= 1.0f) atomicMin(&a.zmin[p], zorder(z));
    return;
  }
  if (!(z == zorder_inv(a.zmin[p]))) return;
  if (PHASE == 2) {
    atomicMin(&a.kfirst[p], u.key);
    atomicMax(&a.klast[p], u.key);
  } else {
    if (a.klast[p] == u.key) a.fb[p] = u.color;
    if (a.kfirst[p] == u.key) a.depth[p] = z;
  }
}

template <int PHASE>
__device__ __forceinline__ void shade_small(const ReyesArgs& a, const UpolyRec& u, unsigned& covered)
{
  for (int y = u.y0; y < u.y1; ++y)
    for (int x = u.x0; x < u.x1; ++x) shade_pixel<PHASE>(a, u, x, y, covered);
}

__device__ __forceinline__ void load_upoly(UpolyRec& o, const UpolyRec* src)
{
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* d = reinterpret_cast<uint4*>(&o);
#pragma unroll
  for (int q = 0; q < 4; ++q) d[q] = s[q];
}

__device__ __forceinline__ void add_covered(const ReyesArgs& a, unsigned covered)
{
  covered = __reduce_add_sync(kFullR, covered);
  if ((threadIdx.x & 31) == 0 && covered) atomicAdd(&a.ctr->fc.covered, (unsigned long long)covered);
}

__global__ void __launch_bounds__(256) reyes_clear(ReyesArgs a, uint32_t npx)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npx; i += gridDim.x * blockDim.x) {
    a.fb[i] = kClearColor;
    a.depth[i] = 1.0f;
    a.zmin[i] = kZorderClear;
    a.kfirst[i] = ~0ull;
    a.klast[i] = 0ull;
  }
}

// Dice (R12, R13) and fragment pass 1 of the micropolygons with at most
// kSmallPx candidate pixels; larger ones are queued for the warp passes.
__global__ void __launch_bounds__(256) reyes_dice(ReyesArgs a)
{
  const unsigned long long meta = a.ctr->leaf_meta;
  const uint32_t nleaf = (uint32_t)min((unsigned long long)a.leaf_cap, meta >> 40);
  unsigned long long total = meta & ((1ull << 40) - 1);
  if (total > a.up_cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&a.ctr->fc.status, kStatusUpolyOverflow);
    total = a.up_cap;
  }
  unsigned covered = 0;
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < total && nleaf; u += gridDim.x * blockDim.x) {
    const uint32_t li = find_leaf(a.leaves, nleaf, u);
    const PatchRec& p = a.leaves[li];
    const uint32_t local = u - p.upbase;
    const uint32_t nv1 = p.nv + 1;
    UpolyRec o;
    o.x0 = o.x1 = o.y0 = o.y1 = 0;
    if (local < (p.nu + 1) * nv1) {
      const int k = (int)(local / nv1), j = (int)(local % nv1);
      float4 P[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) P[q] = p.cp[q];
      const float du = 1.0f / ((float)p.nu), dv = 1.0f / ((float)p.nv);
      const float myU = (float)k * du, myV = (float)j * dv;
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
      // 4-corner bounds (shade.pikostage:129-140) intersected with each Shade
      // bin; the bins are adjacent, so the union is one rectangle
      const float bminx = floorf(std_minf(std_minf(o.sx[0], o.sx[1]), std_minf(o.sx[2], o.sx[3])));
      const float bminy = floorf(std_minf(std_minf(o.sy[0], o.sy[1]), std_minf(o.sy[2], o.sy[3])));
      const float bmaxx = ceilf(std_maxf(std_maxf(o.sx[0], o.sx[1]), std_maxf(o.sx[2], o.sx[3])));
      const float bmaxy = ceilf(std_maxf(std_maxf(o.sy[0], o.sy[1]), std_maxf(o.sy[2], o.sy[3])));
      if (bx1 <= bx2 && by1 <= by2) {
        const float fx0 = (float)(bx1 * 64), fx1 = (float)((bx2 + 1) * 64);
        const float fy0 = (float)(by1 * 64), fy1 = (float)((by2 + 1) * 64);
        int px0 = cvt_i32_x86((bminx > fx0) ? bminx : fx0);
        int px1 = cvt_i32_x86((bmaxx < fx1) ? bmaxx : fx1);
        int py0 = cvt_i32_x86((bminy > fy0) ? bminy : fy0);
        int py1 = cvt_i32_x86((bmaxy < fy1) ? bmaxy : fy1);
        px0 = max(px0, bx1 * 64); py0 = max(py0, by1 * 64);
        px1 = min(min(px1, (bx2 + 1) * 64), a.W);
        py1 = min(min(py1, (by2 + 1) * 64), a.H);
        if (px0 < px1 && py0 < py1) { o.x0 = px0; o.x1 = px1; o.y0 = py0; o.y1 = py1; }
      }
      const uint4* src = reinterpret_cast<const uint4*>(&o);
      uint4* dst = reinterpret_cast<uint4*>(&a.up[u]);
#pragma unroll
      for (int q = 0; q < 4; ++q) dst[q] = src[q];
      if (o.z < 0.0f) atomicAdd(&a.ctr->negative_depth, 1u);
      const int area = (o.x1 - o.x0) * (o.y1 - o.y0);
      if (area > kSmallPx) {
        a.big[atomicAdd(&a.ctr->big_count, 1u)] = u;
      } else {
        shade_small<1>(a, o, covered);
      }
    } else {
      reinterpret_cast<uint4*>(&a.up[u])[3] = make_uint4(0u, 0u, 0u, 0u);
    }
  }
  add_covered(a, covered);
}

// Fragment pass PHASE.  SMALL: a thread per micropolygon with at most kSmallPx
// pixels; then, every pass, a warp per queued larger micropolygon, a lane per
// pixel.
template <int PHASE, bool SMALL>
__global__ void __launch_bounds__(256) reyes_frag(ReyesArgs a)
{
  unsigned covered = 0;
  if (SMALL) {
    unsigned long long total = a.ctr->leaf_meta & ((1ull << 40) - 1);
    if (total > a.up_cap) total = a.up_cap;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
      UpolyRec u;
      load_upoly(u, &a.up[i]);
      const int area = (u.x1 - u.x0) * (u.y1 - u.y0);
      if (area > 0 && area <= kSmallPx) shade_small<PHASE>(a, u, covered);
    }
  }
  const uint32_t nbig = a.ctr->big_count;
  const int lane = threadIdx.x & 31;
  const uint32_t nwarps = gridDim.x * (blockDim.x / 32);
  for (uint32_t w = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; w < nbig; w += nwarps) {
    UpolyRec u;
    load_upoly(u, &a.up[a.big[w]]);
    const int bw = u.x1 - u.x0;
    const int n = bw * (u.y1 - u.y0);
    for (int k = lane; k < n; k += 32) shade_pixel<PHASE>(a, u, u.x0 + k % bw, u.y0 + k / bw, covered);
  }
  if (PHASE == 1) add_covered(a, covered);
}

cudaError_t launch_reyes_frame(const ReyesArgs& a, uint32_t npx, int sms, cudaStream_t st, cudaEvent_t* ev)
{
  if (ev) cudaEventRecord(ev[0], st);
  const int grid = sms * 8;
  reyes_clear<<<sms * 4, 256, 0, st>>>(a, npx);
  reyes_seed<<<(a.P + 255) / 256 + 1, 256, 0, st>>>(a);
  for (int L = 0; L <= a.max_splits; ++L) reyes_split_level<<<grid, 256, 0, st>>>(a, L);
  if (ev) cudaEventRecord(ev[1], st);
  reyes_dice<<<grid, 256, 0, st>>>(a);
  reyes_frag<1, false><<<grid, 256, 0, st>>>(a);
  if (ev) cudaEventRecord(ev[2], st);
  reyes_frag<2, true><<<grid, 256, 0, st>>>(a);
  if (ev) cudaEventRecord(ev[3], st);
  reyes_frag<3, true><<<grid, 256, 0, st>>>(a);
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
  uint32_t* big = nullptr;
  uint32_t lvl_cap = 0, leaf_cap = 0, up_cap = 0;
  uint32_t* zmin = nullptr;
  unsigned long long* kfirst = nullptr;
  unsigned long long* klast = nullptr;
  size_t npx_cap = 0;
  ReyesCounters* ctr = nullptr;
  ReyesCounters* h_ctr = nullptr;
  cudaEvent_t ev[5] = {};
  bool ev_made = false;
};

void piko_reyes_release(piko_scene* s)
{
  ReyesState* r = s->reyes;
  if (!r) return;
  dfree(r->lvl[0]); dfree(r->lvl[1]); dfree(r->leaves); dfree(r->up); dfree(r->big);
  dfree(r->zmin); dfree(r->kfirst); dfree(r->klast); dfree(r->ctr);
  if (r->h_ctr) cudaFreeHost(r->h_ctr);
  if (r->ev_made) for (auto& e : r->ev) cudaEventDestroy(e);
  delete r;
  s->reyes = nullptr;
}

static cudaError_t reyes_alloc(ReyesState* r, uint32_t lvl_cap, uint32_t leaf_cap, uint32_t up_cap, size_t npx)
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
    dfree(r->up); dfree(r->big);
    if ((e = dalloc(&r->up, up_cap)) || (e = dalloc(&r->big, up_cap))) return e;
    r->up_cap = up_cap;
  }
  if (npx > r->npx_cap) {
    dfree(r->zmin); dfree(r->kfirst); dfree(r->klast);
    if ((e = dalloc(&r->zmin, npx)) || (e = dalloc(&r->kfirst, npx)) || (e = dalloc(&r->klast, npx))) return e;
    r->npx_cap = npx;
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
  const uint32_t P = (uint32_t)s->N;
  const size_t npx = (size_t)s->W * (size_t)s->H;
  CU(ctx, reyes_alloc(r, std::max<uint32_t>(1u << 16, 64u * P), std::max<uint32_t>(1u << 16, 64u * P),
                      r->up_cap ? r->up_cap : (1u << 20), npx));
  CU(ctx, cudaMemsetAsync(r->ctr, 0, sizeof(ReyesCounters), st));
  ReyesArgs a;
  memset(&a, 0, sizeof(a));
  a.W = s->W; a.H = s->H; a.nBx = s->W / 64; a.nBy = s->H / 64;
  a.nDice = std::max(1, a.nBx * a.nBy);
  a.P = (int)P;
  memcpy(a.vp, s->state.view_proj, sizeof(a.vp));
  a.thr = p->split_threshold;
  a.max_splits = std::min(p->max_splits, 30);
  a.grid = p->dice_grid;
  a.in_patches = s->patches;
  a.lvl[0] = r->lvl[0]; a.lvl[1] = r->lvl[1]; a.lvl_cap = r->lvl_cap;
  a.leaves = r->leaves; a.leaf_cap = r->leaf_cap;
  a.up = r->up; a.up_cap = r->up_cap; a.big = r->big;
  a.ctr = r->ctr;
  a.fb = s->fb; a.depth = s->depth;
  a.zmin = r->zmin; a.kfirst = r->kfirst; a.klast = r->klast;
  CU(ctx, launch_reyes_frame(a, (uint32_t)npx, ctx->sms, st, timed ? r->ev : nullptr));
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
    if (!(st & (kStatusPatchOverflow | kStatusUpolyOverflow))) {
      s->pending = false;
      return PIKO_OK;
    }
    uint32_t maxlvl = 0;
    for (int i = 0; i < 40; ++i) maxlvl = std::max(maxlvl, c.level_count[i]);
    const uint32_t leaves = (uint32_t)(c.leaf_meta >> 40);
    const unsigned long long ups = c.leaf_meta & ((1ull << 40) - 1);
    uint32_t lvl = r->lvl_cap, lf = r->leaf_cap, up = r->up_cap;
    if (st & kStatusPatchOverflow) { lvl = std::max(lvl, maxlvl + maxlvl / 2 + 1024); lf = std::max(lf, 2 * leaves + 1024); }
    if (st & kStatusUpolyOverflow) up = (uint32_t)std::min<unsigned long long>(ups + ups / 4 + 4096, 0xffffffffull);
    CU(ctx, reyes_alloc(r, lvl, lf, up, r->npx_cap));
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
  o->bin_entries = c.big_count;   // micropolygons shaded a warp per micropolygon
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
