// Reyes pipeline for sm_100a: the reference's ReyesPipe (SplitStage with its
// self loop -> DiceStage -> ShadeStage -> PikoScreen, pikoc/samples/reyesPipe)
// off a device work queue:
//
//   reyes_split    one cooperative launch (one CTA per SM), sixteen lanes per
//       patch: project the 16 control points, measure the u/v screen extents,
//       split at the halves (de Casteljau) or emit a leaf with its dice grid
//       (R11, split.pikostage:240-343).  Each CTA expands its patches level
//       after level in shared memory; children past what a CTA keeps go to a
//       global frontier that the next step spreads over all CTAs, after a grid
//       barrier; leaves are staged and written out in batches.  No host round
//       trip between levels (the reference copies the Split stage back to the
//       host every level).
//   reyes_dice     every CTA an equal range of dice rows; per group of rows,
//       the control rows at each u once, each grid point once into shared
//       memory: patch position and normal, projection, the corner-averaged
//       "Phong" colour and the mean depth (R12, dice.pikostage:159-312; R13
//       colour, shade.pikostage:64-109), the 64-pixel Shade-bin range of three
//       corners (shade.pikostage:51-56) cut with the four-corner bounds to one
//       pixel rectangle, then a sample-parallel coverage pass and the first
//       fragment pass (depth minimum) over that rectangle.
//   reyes_big      the first fragment pass for micropolygons with more than
//       kSmallPx candidate pixels, a warp each.
//   reyes_keys, reyes_resolve  the other two fragment passes over the fragment
//       list; reyes_pixels writes the pixels no fragment reached (averages a
//       pixel's samples with 4 samples per pixel) and sets the per-sample
//       state of the reached samples back to empty for the next frame.
//       Shade work is spread per micropolygon and per fragment, not per
//       screen tile, so silhouette tiles where thousands of micropolygons pile
//       up cost no more than anywhere else.  The per-sample test is the
//       reference's (both windings, shade.pikostage:161-235).
//
// Order independence.  The reference resolves depth with
//   while (remote > z) remote = atomicMin(bits, z);  pass iff zbuf == z
// in the order Dice bins, leaves and grid points are processed.  Run
// sequentially that keeps, per pixel, the minimum depth m, the depth bits of
// the FIRST fragment with depth == m and the colour of the LAST one.  Every
// micropolygon carries a 64-bit key that sorts like the reference's processing
// order -- (Dice bin, split level, position in the level, grid index) -- so
// the kernels may visit fragments in any order.
#include <mutex>

#include "runtime_internal.h"

namespace piko {

constexpr unsigned kFullR = 0xffffffffu;

struct __align__(16) PatchRec {
  float4 cp[16];
  uint32_t i0;          // input patch index
  uint32_t level;       // split level = numSplits
  unsigned long long s; // position key inside the level: children of s are 2s, 2s+1
  uint32_t nu, nv;      // dice grid (leaves)
  uint32_t rowbase;     // first dice row (leaves): leaf rows are numbered in slot order
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

// The frame status and fragment count of a Reyes frame (status bits as the
// raster path's).
struct ReyesFrameCounters {
  uint32_t status;
  uint32_t pad;
  unsigned long long covered;
};

struct ReyesCounters {
  ReyesFrameCounters fc;
  uint32_t level_count[40];
  unsigned long long leaf_meta;   // (leaves << 40) | dice rows (nu + 1 per leaf)
  unsigned long long upolys;      // micropolygons of all leaves
  uint32_t levels_run;
  uint32_t negative_depth;
  uint32_t big_count;             // micropolygons queued for reyes_big
  uint32_t frag_count;            // fragments appended by pass 1
  unsigned long long bar_arrive;  // grid barrier of reyes_split: (arrivals << 40) | children
  unsigned long long bar_release; // (barriers passed << 32) | next level's patch count
};

struct FragRec;

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
  UpolyRec* up;                   // micropolygons with more than kSmallPx candidate pixels
  uint32_t up_cap;
  FragRec* frags;                 // covered samples with depth <= 1 (pass 1 output)
  uint32_t frag_cap;
  ReyesCounters* ctr;
  uint32_t* fb;
  float* depth;
  uint32_t* zmin;                 // per sample: order-mapped minimum depth
  unsigned long long* kfirst;     // per sample: least key among fragments at the minimum
  unsigned long long* klast;      // per sample: greatest key among fragments at the minimum
  // Multi-sample / Phong variant (no reference counterpart).  spp samples per
  // pixel (1: the reference's pixel centre; 4: one jittered sample per pixel
  // quadrant, seeded); phong = 1 lights the micropolygon's interpolated normal.
  // With spp > 1 the resolve writes samples (scol, sdep) and reyes_pixels
  // averages them into the pixel.
  int spp;
  uint32_t seed;
  int phong;
  uint32_t* scol;                 // per sample colour (spp > 1)
  float* sdep;                    // per sample depth (spp > 1)
};

// Micropolygons whose shaded rectangle holds more pixels than this are shaded
// by a warp (one lane per pixel) instead of by the thread that owns them.
constexpr int kSmallPx = 16;

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
// The cleared per-sample minimum: above zorder(z) of every depth z <= 1 (the
// only fragments kept), so a sample's minimum stays kZminEmpty exactly when no
// fragment reached it.
constexpr uint32_t kZminEmpty = 0xffffffffu;

// Sample s of pixel (x, y): the centre for one sample per pixel; otherwise
// quadrant (s & 1, s >> 1) of the pixel at a jitter from an integer hash of
// (seed, x, y, 2s + axis), 24 bits per axis.  The oracle's restatement uses the
// same function, operation for operation.
__device__ __forceinline__ uint32_t sample_hash(uint32_t seed, uint32_t x, uint32_t y, uint32_t k)
{
  uint32_t h = seed * 0x9E3779B1u;
  h ^= x * 0x85EBCA77u;
  h ^= y * 0xC2B2AE3Du;
  h ^= k * 0x27D4EB2Fu;
  h ^= h >> 16; h *= 0x7FEB352Du;
  h ^= h >> 15; h *= 0x846CA68Bu;
  h ^= h >> 16;
  return h;
}
__device__ __forceinline__ void sample_pos(int spp, uint32_t seed, int x, int y, int s, float& px, float& py)
{
  if (spp == 1) { px = (float)x + 0.5f; py = (float)y + 0.5f; return; }
  const float jx = (float)(sample_hash(seed, (uint32_t)x, (uint32_t)y, 2u * (uint32_t)s) >> 8) * 5.9604644775390625e-8f;
  const float jy = (float)(sample_hash(seed, (uint32_t)x, (uint32_t)y, 2u * (uint32_t)s + 1u) >> 8) * 5.9604644775390625e-8f;
  px = (float)x + ((float)(s & 1) + jx) * 0.5f;
  py = (float)y + ((float)(s >> 1) + jy) * 0.5f;
}

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

// One row (or column) of splitU / splitV (split.pikostage:95-224): de Casteljau
// at t = 1/2 of the four points p0..p3; a0..a3 is the first half, b0..b3 the
// second.  Returns the j-th point of half `second`.
__device__ __forceinline__ float4 casteljau_half(float4 p0, float4 p1, float4 p2, float4 p3, int j, bool second)
{
  const float4 a1 = f4mul(f4add(p0, p1), 0.5f);
  const float4 b2 = f4mul(f4add(p2, p3), 0.5f);
  const float4 t = f4mul(f4add(p1, p2), 0.5f);
  const float4 a2 = f4mul(f4add(a1, t), 0.5f);
  const float4 b1 = f4mul(f4add(b2, t), 0.5f);
  const float4 a3 = f4mul(f4add(a2, b1), 0.5f);
  if (!second) return j == 0 ? p0 : (j == 1 ? a1 : (j == 2 ? a2 : a3));
  return j == 0 ? a3 : (j == 1 ? b1 : (j == 2 ? b2 : p3));
}

__device__ __forceinline__ float4 shfl4(unsigned mask, float4 v, int src)
{
  return make_float4(__shfl_sync(mask, v.x, src, 16), __shfl_sync(mask, v.y, src, 16), __shfl_sync(mask, v.z, src, 16),
                     __shfl_sync(mask, v.w, src, 16));
}

// Grid-wide barrier between split levels that also carries the next level's
// patch count: every CTA arrives with the children it reserved; the last
// arrival sums them and releases barrier k with (k + 1) << 32 | count, so no
// CTA reads the count back afterwards.  It comes in two halves (arrive, wait).
// The wait is bounded: after 1 s without a release (the
// globaltimer; an iteration cap besides) the CTA records kStatusBarrierTimeout
// and goes on (the host reports PIKO_ERR_TIMEOUT).
constexpr unsigned long long kBarrierWaitNs = 1000000000ull;

__device__ __forceinline__ unsigned long long global_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void barrier_arrive(ReyesCounters* c, uint32_t k, uint32_t* s_children)
{
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t children = *s_children;   // settled: every lane has passed the sync
    *s_children = 0;                         // next level's adds come after barrier_wait
    __threadfence();
    const unsigned long long old = atomicAdd(&c->bar_arrive, (1ull << 40) | children);
    if ((uint32_t)(old >> 40) == gridDim.x - 1) {
      const unsigned long long total = (old & ((1ull << 40) - 1)) + children;
      c->bar_arrive = 0;
      __threadfence();
      atomicExch(&c->bar_release, ((unsigned long long)(k + 1) << 32) | min(total, 0xffffffffull));
    }
  }
}

__device__ __forceinline__ uint32_t barrier_wait(ReyesCounters* c, uint32_t k, uint32_t* s_count)
{
  if (threadIdx.x == 0) {
    volatile unsigned long long* rel = &c->bar_release;
    volatile uint32_t* status = &c->fc.status;
    uint32_t spins = 0;
    unsigned long long v;
    const unsigned long long t0 = global_ns();
    while ((uint32_t)((v = *rel) >> 32) != k + 1) {
      // the time limit and another CTA's timeout are checked every 16 polls
      if ((++spins & 15u) != 0u) continue;
      __nanosleep(32);
      if (*status & kStatusBarrierTimeout) { v = 0; break; }
      if (global_ns() - t0 > kBarrierWaitNs || spins > (1u << 28)) {
        atomicOr(&c->fc.status, kStatusBarrierTimeout);
        v = 0;
        break;
      }
    }
    __threadfence();
    *s_count = (uint32_t)v;
  }
  __syncthreads();
  return *s_count;
}

// The per-sample state (depth minimum, key bounds) starts every frame empty:
// the buffers are set so when allocated, and reyes_pixels, which visits every
// sample after the fragment passes, sets a reached sample back.  The split
// clears nothing.

// One patch of one split level (R11, split.pikostage:240-343), sixteen lanes
// per patch: lane c holds control point c; the u and v polyline lengths are
// summed over shuffles in the reference's order.  split_measure decides split
// or leaf (and the leaf's dice grid); split_write then writes control point c
// of both children (split along u or v at the halves, de Casteljau) or copies
// it into the leaf.
struct SplitDecision {
  float ue, ve;
  bool split;
  int nu, nv;
};

__device__ __forceinline__ SplitDecision split_measure(const ReyesArgs& a, int L, float4 cp, int c, unsigned hmask)
{
  float4 q = matmul4(a.vp, cp);
  if (q.w == 0.0f) q.w = 1.0f;
  q.x = q.x / q.w;
  q.y = q.y / q.w;
  // (x + 1.0) * 0.5 * W in double, rounded to float, is one fma of floats:
  // the double sequence is exact wherever the value lies near a float
  // rounding boundary, so both round the exact value x * W/2 + W/2 once
  const float hw = 0.5f * (float)a.W, hh = 0.5f * (float)a.H;
  const float cx = __fmaf_rn(q.x, hw, hw);
  const float cy = __fmaf_rn(q.y, hh, hh);
  // distance to the next point along u (same row) and along v (same column)
  const float ux = __shfl_sync(hmask, cx, c + 1, 16), uy = __shfl_sync(hmask, cy, c + 1, 16);
  const float vx = __shfl_sync(hmask, cx, c + 4, 16), vy = __shfl_sync(hmask, cy, c + 4, 16);
  const float du = dist2(cx, cy, ux, uy);
  const float dv = dist2(cx, cy, vx, vy);
  SplitDecision d;
  d.ue = 0.0f;
  d.ve = 0.0f;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    float su = __shfl_sync(hmask, du, 4 * r, 16) + __shfl_sync(hmask, du, 4 * r + 1, 16);
    su = su + __shfl_sync(hmask, du, 4 * r + 2, 16);
    d.ue = std_maxf(d.ue, su);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float sv = __shfl_sync(hmask, dv, k, 16) + __shfl_sync(hmask, dv, k + 4, 16);
    sv = sv + __shfl_sync(hmask, dv, k + 8, 16);
    d.ve = std_maxf(d.ve, sv);
  }
  d.split = (d.ue >= a.thr) || (d.ve >= a.thr);
  if (L >= a.max_splits) d.split = false;
  d.nu = d.nv = 0;
  if (!d.split) {
    if (a.grid > 0) {   // a fixed dice grid replaces the extent-derived one
      d.nu = d.nv = a.grid;
    } else {
      int nu = pow2roundup(cvt_i32_x86_d(ceil((double)(d.ue / a.thr))) + 1);
      int nv = pow2roundup(cvt_i32_x86_d(ceil((double)(d.ve / a.thr))) + 1);
      d.nu = nu < 2 ? 2 : (nu > 32 ? 32 : nu);
      d.nv = nv < 2 ? 2 : (nv > 32 ? 32 : nv);
    }
  }
  return d;
}

// The split runs as one cooperative launch of kSplitThreads-thread CTAs, one
// per SM, sixteen lanes per patch (a 16-lane group takes two patches of a
// level), so a CTA works on up to kSplitKeep patches per level.  A CTA expands
// its patches level after level in shared memory: the children of a level
// stay in the CTA (up to kSplitKeep of them; the rest go to a global frontier
// for the next step, spread evenly over the CTAs), and leaves are staged and
// written out in batches.  A step ends with a grid barrier; the split ends at
// the first step whose frontier is empty.  Patches of a step's frontier are at
// least at level `step`, so there are at most max_splits + 1 steps.  Nothing
// depends on which CTA or pass handles a patch: every leaf carries its input
// index, level and in-level position (children of s are 2s and 2s + 1), which
// give the order key.
constexpr int kSplitThreads = 512;
constexpr int kSplitKeep = 2 * (kSplitThreads / 16);   // patches a CTA keeps per level (two per 16-lane group)
constexpr int kSplitStage = 128;
struct SplitSmem {
  PatchRec buf[2][2 * kSplitKeep];    // current level, children of the current level
  PatchRec stage[kSplitStage];        // leaves not yet written out
  uint32_t nnext, nleaf, ncur, maxlevel;
  uint32_t children;                  // patches this CTA pushed to the frontier in this step
  uint32_t word[4];
};
constexpr size_t kSplitSmem = sizeof(SplitSmem);

// Copies n patch records (18 float4 each) with the whole CTA.
__device__ __forceinline__ void copy_patches(PatchRec* dst, const PatchRec* src, uint32_t n, bool from_l2)
{
  constexpr uint32_t kQ = sizeof(PatchRec) / 16;
  const float4* s4 = reinterpret_cast<const float4*>(src);
  float4* d4 = reinterpret_cast<float4*>(dst);
  for (uint32_t i = threadIdx.x; i < n * kQ; i += blockDim.x) d4[i] = from_l2 ? __ldcg(&s4[i]) : s4[i];
}

// Input patch i of a step: an input patch at level 0 (i0 = s = i) or a record
// of the global frontier.
__device__ __forceinline__ void load_inputs(const ReyesArgs& a, int step, uint32_t first, uint32_t n, PatchRec* dst)
{
  if (step == 0) {
    for (uint32_t q = threadIdx.x; q < n * 16u; q += blockDim.x) {
      const uint32_t i = q >> 4, c = q & 15u;
      dst[i].cp[c] = __ldcg(&a.in_patches[(size_t)(first + i) * 16 + c]);
      if (c == 0) {
        dst[i].i0 = first + i;
        dst[i].level = 0;
        dst[i].s = first + i;
      }
    }
  } else {
    copy_patches(dst, a.lvl[step & 1] + first, n, true);
  }
}

// Writes the staged leaves out: one 64-bit atomic reserves their slots and
// dice rows together (so rows stay contiguous in slot order), and their
// micropolygon count is added.  Called by every thread of the CTA.
__device__ __forceinline__ void flush_leaves(const ReyesArgs& a, SplitSmem& S)
{
  __syncthreads();
  const uint32_t nl = S.nleaf;
  if (nl == 0) return;   // uniform
  if (threadIdx.x < 32) {
    const uint32_t lane = threadIdx.x;
    const uint32_t per = (nl + 31u) / 32u;
    const uint32_t b0 = min(lane * per, nl), b1 = min(b0 + per, nl);
    uint32_t rows = 0, ups = 0;
    for (uint32_t i = b0; i < b1; ++i) {
      rows += S.stage[i].nu + 1u;
      ups += (S.stage[i].nu + 1u) * (S.stage[i].nv + 1u);
    }
    uint32_t incl = rows;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(kFullR, incl, o);
      if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t total = __shfl_sync(kFullR, incl, 31);
    const uint32_t up_total = __reduce_add_sync(kFullR, ups);
    unsigned long long old = 0;
    if (lane == 0) {
      old = atomicAdd(&a.ctr->leaf_meta, ((unsigned long long)nl << 40) | total);
      atomicAdd(&a.ctr->upolys, (unsigned long long)up_total);
    }
    old = __shfl_sync(kFullR, old, 0);
    uint32_t r = (uint32_t)(old & ((1ull << 40) - 1)) + incl - rows;
    for (uint32_t i = b0; i < b1; ++i) {
      S.stage[i].rowbase = r;
      r += S.stage[i].nu + 1u;
    }
    if (lane == 0) S.word[3] = (uint32_t)(old >> 40);
  }
  __syncthreads();
  const uint32_t base = S.word[3];
  if (base + nl <= a.leaf_cap) {
    copy_patches(a.leaves + base, S.stage, nl, false);
  } else if (threadIdx.x == 0) {
    atomicOr(&a.ctr->fc.status, kStatusPatchOverflow);   // the host grows the buffer and runs again
  }
  __syncthreads();
  if (threadIdx.x == 0) S.nleaf = 0;
}

// One level of the CTA's current patches (at most kSplitKeep; 16-lane group
// q takes patches q, q + 32): split ones put their children in nxt, leaves
// go to the stage.
__device__ __forceinline__ void split_one(const ReyesArgs& a, SplitSmem& S, const PatchRec* cur, PatchRec* nxt,
                                          uint32_t p)
{
  const int c = threadIdx.x & 15;
  const unsigned hmask = 0xffffu << (threadIdx.x & 16);
  const float4 cp = cur[p].cp[c];
  const uint32_t i0 = cur[p].i0, L = cur[p].level;
  const unsigned long long s = cur[p].s;
  const SplitDecision d = split_measure(a, (int)L, cp, c, hmask);
  uint32_t slot = 0;
  if (c == 0) slot = d.split ? atomicAdd(&S.nnext, 2u) : atomicAdd(&S.nleaf, 1u);
  slot = __shfl_sync(hmask, slot, 0, 16);
  if (d.split) {
    const bool along_u = d.ue >= a.thr;
    // the four points of this lane's row (split along u) or column (along v)
    const int base = along_u ? (c & ~3) : (c & 3), st = along_u ? 1 : 4, j = along_u ? (c & 3) : (c >> 2);
    const float4 p0 = shfl4(hmask, cp, base), p1 = shfl4(hmask, cp, base + st);
    const float4 p2 = shfl4(hmask, cp, base + 2 * st), p3 = shfl4(hmask, cp, base + 3 * st);
    nxt[slot].cp[c] = casteljau_half(p0, p1, p2, p3, j, false);
    nxt[slot + 1].cp[c] = casteljau_half(p0, p1, p2, p3, j, true);
    if (c < 2) {
      PatchRec& o = nxt[slot + c];
      o.i0 = i0;
      o.level = L + 1;
      o.s = 2 * s + (unsigned long long)c;
    }
    if (c == 0) atomicMax(&S.maxlevel, L + 1);
  } else {
    PatchRec& o = S.stage[slot];
    o.cp[c] = cp;
    if (c == 0) {
      o.i0 = i0;
      o.level = L;
      o.s = s;
      o.nu = (uint32_t)d.nu;
      o.nv = (uint32_t)d.nv;
    }
  }
}

__device__ __forceinline__ void split_pass(const ReyesArgs& a, SplitSmem& S, const PatchRec* cur, PatchRec* nxt,
                                           uint32_t ncur)
{
  for (uint32_t p = threadIdx.x >> 4; p < ncur; p += kSplitThreads / 16)   // whole 16-lane groups
    split_one(a, S, cur, nxt, p);
}

__global__ void __launch_bounds__(kSplitThreads, 1) reyes_split(ReyesArgs a)
{
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char split_smem[];
  SplitSmem& S = *reinterpret_cast<SplitSmem*>(split_smem);
  if (threadIdx.x == 0) {
    S.nleaf = 0;
    S.maxlevel = 0;
    S.children = 0;
  }
  uint32_t n_in = (uint32_t)a.P;
  for (int step = 0; n_in > 0; ++step) {   // n_in is uniform
    // This CTA's share of the step's frontier.  With fewer patches than
    // CTAs, 2^d CTAs share a patch: each takes the patch's descendants along
    // its own d-bit path (the first d levels of the patch are computed by
    // all of them), so every CTA has a subtree; a leaf met on the way is
    // emitted by the group's CTA whose remaining path bits are all 0.
    uint32_t d = 0;
    while (d < 16 && ((unsigned long long)n_in << (d + 1)) <= gridDim.x) ++d;
    uint32_t r0, r1, path = 0, dr = 0;
    if (d > 0) {
      const uint32_t owner = blockIdx.x >> d;
      r0 = min(owner, n_in);
      r1 = min(owner + 1, n_in);
      path = blockIdx.x & ((1u << d) - 1u);
      dr = d;
    } else {
      r0 = (uint32_t)((unsigned long long)n_in * blockIdx.x / gridDim.x);
      r1 = (uint32_t)((unsigned long long)n_in * (blockIdx.x + 1) / gridDim.x);
    }
    PatchRec* frontier = a.lvl[(step + 1) & 1];
    uint32_t pos = r0, ncur = 0;
    int cb = 0;   // buf[cb] holds the current patches
    __syncthreads();
    while (ncur > 0 || pos < r1) {   // uniform
      // top up the current patches from the share
      const uint32_t take = min((uint32_t)kSplitKeep - ncur, r1 - pos);
      if (take) load_inputs(a, step, pos, take, &S.buf[cb][ncur]);
      pos += take;
      ncur += take;
      if (S.nleaf + (uint32_t)kSplitKeep > (uint32_t)kSplitStage) flush_leaves(a, S);
      if (threadIdx.x == 0) S.nnext = 0;
      __syncthreads();
      split_pass(a, S, S.buf[cb], S.buf[cb ^ 1], ncur);
      __syncthreads();
      uint32_t nn = S.nnext;
      if (dr > 0) {
        // one patch on the CTA's path (ncur == 1): keep the child the path
        // names, or drop a leaf that another CTA of the group emits
        if (nn == 0) {
          if ((path & ((1u << dr) - 1u)) != 0u && threadIdx.x == 0) S.nleaf -= 1;
        } else {
          if ((path >> (dr - 1)) & 1u) {
            float4* dst = reinterpret_cast<float4*>(&S.buf[cb ^ 1][0]);
            const float4* src = reinterpret_cast<const float4*>(&S.buf[cb ^ 1][1]);
            if (threadIdx.x < sizeof(PatchRec) / 16) dst[threadIdx.x] = src[threadIdx.x];
          }
          nn = 1;
        }
        --dr;
      } else if (nn > (uint32_t)kSplitKeep) {
        // children past kSplitKeep go to the frontier of the next step
        const uint32_t extra = nn - (uint32_t)kSplitKeep;
        if (threadIdx.x == 0) {
          S.word[3] = atomicAdd(&a.ctr->level_count[min(step + 1, 39)], extra);
          S.children += extra;
        }
        __syncthreads();
        const uint32_t at = S.word[3];
        if (at + extra <= a.lvl_cap) {
          copy_patches(frontier + at, &S.buf[cb ^ 1][kSplitKeep], extra, false);
        } else if (threadIdx.x == 0) {
          atomicOr(&a.ctr->fc.status, kStatusPatchOverflow);
        }
      }
      ncur = min(nn, (uint32_t)kSplitKeep);
      cb ^= 1;
      __syncthreads();
    }
    // grid barrier: the frontier written by every CTA is read after it.  The
    // staged leaves go out between arriving and waiting: only later launches
    // read them, so the arrival need not wait for their stores.
    barrier_arrive(a.ctr, (uint32_t)step, &S.children);
    flush_leaves(a, S);
    n_in = min(barrier_wait(a.ctr, (uint32_t)step, &S.word[1]), a.lvl_cap);
  }
  if (threadIdx.x == 0 && a.P > 0) atomicMax(&a.ctr->levels_run, S.maxlevel + 1u);
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

// patchEval + normEval + projection of one corner (dice.pikostage:111-146,205-220),
// in two parts: dice_row evaluates the four control rows and their u
// derivatives at u, which every corner at that u shares; dice_corner finishes
// one corner at v.  Splitting changes no operation or its order.
struct DiceRow {
  float4 r[4], d[4];
};

__device__ __forceinline__ void dice_row(const float4* P, float u, DiceRow& R)
{
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    R.r[k] = bez(u, P[4 * k], P[4 * k + 1], P[4 * k + 2], P[4 * k + 3]);
    R.d[k] = dbez(u, P[4 * k], P[4 * k + 1], P[4 * k + 2], P[4 * k + 3]);
  }
}

__device__ __forceinline__ void dice_corner(const DiceRow& R, const ReyesArgs& a, float v, float& sx, float& sy,
                                            float& sz, float& nx, float& ny, float& nz)
{
  const float4 pt = bez(v, R.r[0], R.r[1], R.r[2], R.r[3]);
  const float4 v1 = bez(v, R.d[0], R.d[1], R.d[2], R.d[3]);
  const float4 v2 = dbez(v, R.r[0], R.r[1], R.r[2], R.r[3]);
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


// ------------------------------------------------------------------ shade
// ShadeStage's per-pixel test (shade.pikostage:161-235): the sample is inside
// the micropolygon when all four edge functions are positive for either
// winding.  Every product and difference is rounded separately, as on the CPU.
// The reversed winding's edges are written with the forward deltas negated:
// b - a == -(a - b), x * -y == -(x * y) and -p - -q == -(p - q) hold exactly
// in round-to-nearest, so "reversed edge > 0" is "the same products with the
// forward delta, difference < 0", bit for bit.
__device__ __forceinline__ bool upoly_covers(float4 X4, float4 Y4, float px, float py)
{
  const float X[4] = {X4.x, X4.y, X4.z, X4.w}, Y[4] = {Y4.x, Y4.y, Y4.z, Y4.w};
  float dX[4], dY[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    dX[i] = X[(i + 1) & 3] - X[i];
    dY[i] = Y[(i + 1) & 3] - Y[i];
  }
  bool r1 = true, r2 = true;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float ay = py - Y[i], bx = px - X[i];
    if (!(ay * dX[i] - bx * dY[i] > 0.0f)) r1 = false;                   // edge i -> i+1
    if (!(ay * dX[(i + 3) & 3] - bx * dY[(i + 3) & 3] < 0.0f)) r2 = false; // edge i -> i-1
  }
  return r1 || r2;
}

// Which samples can pass upoly_covers at all.  When every corner coordinate is
// at least 32 and the corners span less than 16 px per axis, each difference
// the test takes (sample minus corner, corner minus corner) is exact
// (Sterbenz), so a positive rounded edge value means a positive exact one;
// a sample inside all four edges of either winding has a non-zero winding
// number and lies strictly inside the corners' bounding box.  There the
// coverage pass tests only the cells (pixel quadrants, or pixel centres with
// one sample) whose sample range meets the open box; elsewhere it tests all.
__device__ __forceinline__ bool exact_box(float mnx, float mxx, float mny, float mxy)
{
  return mnx >= 32.0f && mny >= 32.0f && mxx - mnx < 16.0f && mxy - mny < 16.0f && mxx < 4194304.0f &&
         mxy < 4194304.0f;
}

// The depth resolve.  The CPU shades micropolygons in its processing order with
//   while (remote > z) remote = atomicMin(bits, z);  pass iff zbuf == z
// so, per pixel, the surviving depth is the minimum m (the cleared 1.0
// included), its bits come from the FIRST fragment with depth m and the colour
// from the LAST one.  Every fragment carries its micropolygon's order key;
//   pass 1 (dice, reyes_big)  zmin <- min zorder(z); fragments with z <= 1
//                             are appended to a fragment list
//   pass 2 (reyes_keys)       klast <- max key of the fragments at m; where
//                             m is +-0, kfirst <- their min key (64-bit
//                             atomics): only there can the bits differ
//   pass 3 (reyes_resolve)    the fragment whose key is klast writes the
//                             colour and, unless m is +-0, the depth; at +-0
//                             the one whose key is kfirst writes the depth.
// A pixel nothing reaches keeps the cleared colour and depth; a fragment at
// exactly 1.0 takes the colour but leaves the (identical) cleared depth bits.
struct __align__(16) FragRec {
  unsigned long long key;
  uint32_t pix;
  float z;
  uint32_t color;
  uint32_t pad[3];
};
static_assert(sizeof(FragRec) == 32, "FragRec layout");

__device__ __forceinline__ void add_covered(const ReyesArgs& a, unsigned covered)
{
  covered = __reduce_add_sync(kFullR, covered);
  if ((threadIdx.x & 31) == 0 && covered) atomicAdd(&a.ctr->fc.covered, (unsigned long long)covered);
}

__device__ __forceinline__ void emit_fragment(const ReyesArgs& a, uint32_t slot, const UpolyRec& u, int x, int y,
                                              int smp)
{
  const uint32_t pix = ((uint32_t)y * (uint32_t)a.W + (uint32_t)x) * (uint32_t)a.spp + (uint32_t)smp;
  atomicMin(&a.zmin[pix], zorder(u.z));
  if (slot < a.frag_cap) {
    FragRec f;
    f.key = u.key;
    f.pix = pix;
    f.z = u.z;
    f.color = u.color;
    f.pad[0] = f.pad[1] = f.pad[2] = 0;
    const uint4* src = reinterpret_cast<const uint4*>(&f);
    uint4* dst = reinterpret_cast<uint4*>(&a.frags[slot]);
    dst[0] = src[0];
    dst[1] = src[1];
  } else {
    atomicOr(&a.ctr->fc.status, kStatusListOverflow);
  }
}

// Block-wide exclusive scan of n (all 256 threads call it) and one atomic on
// the fragment counter; returns this thread's first slot.
__device__ __forceinline__ uint32_t block_append(const ReyesArgs& a, uint32_t n, uint32_t* s_warp, uint32_t* s_base)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = n;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFullR, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t tot = 0;
    for (int w = 0; w < 8; ++w) { const uint32_t v = s_warp[w]; s_warp[w] = tot; tot += v; }
    *s_base = tot ? atomicAdd(&a.ctr->frag_count, tot) : 0u;
  }
  __syncthreads();
  const uint32_t r = *s_base + s_warp[warp] + inc - n;
  __syncthreads();
  return r;
}

// ------------------------------------------------------------------ dice
// A dice grid point: screen position and depth, and the per-channel "Phong"
// term of its normal (the reference's corner lighting) or, in the Phong
// variant, the normal itself.
struct GridPt {
  float sx, sy, sz, ph[3];
};

__device__ __forceinline__ void grid_point_row(const DiceRow& R, const ReyesArgs& a, float v, GridPt& g)
{
  float nx, ny, nz;
  dice_corner(R, a, v, g.sx, g.sy, g.sz, nx, ny, nz);
  if (a.phong) {
    g.ph[0] = nx; g.ph[1] = ny; g.ph[2] = nz;
  } else {
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) g.ph[ch] = phong_channel(nx, ny, nz, ch);
  }
}

__device__ __forceinline__ void grid_point(const float4* P, const ReyesArgs& a, float u, float v, GridPt& g)
{
  DiceRow R;
  dice_row(P, u, R);
  grid_point_row(R, a, v, g);
}

// The order key's leaf part: Dice bin of the leaf's id (dice.pikostage:18-43,
// ids (i0 + L(L+1)/2) / 128 mod the bin count), split level, position in the level.
__device__ __forceinline__ unsigned long long leaf_key(const ReyesArgs& a, uint32_t i0, uint32_t L,
                                                       unsigned long long s)
{
  const uint32_t id = i0 + L * (L + 1) / 2;
  const unsigned long long d = (unsigned long long)((id / 128u) % (uint32_t)a.nDice);
  return (d << 52) | ((unsigned long long)L << 47) | (s << 12);
}

// Micropolygon `local` of a leaf from its corners (k, j), (k+1, j), (k+1, j+1),
// (k, j+1): mean depth, averaged colour, order key (leaf part keyhi), and the
// pixel rectangle of its Shade bins (dice.pikostage:18-43,159-312;
// shade.pikostage:51-56,129-140).
__device__ __forceinline__ void make_upoly(const ReyesArgs& a, unsigned long long keyhi, uint32_t local,
                                           const GridPt& c0, const GridPt& c1, const GridPt& c2, const GridPt& c3,
                                           UpolyRec& o)
{
  o.sx[0] = c0.sx; o.sx[1] = c1.sx; o.sx[2] = c2.sx; o.sx[3] = c3.sx;
  o.sy[0] = c0.sy; o.sy[1] = c1.sy; o.sy[2] = c2.sy; o.sy[3] = c3.sy;
  o.z = ((c0.sz + c1.sz + c2.sz + c3.sz)) * 0.25f;
  float col[3];
  if (a.phong) {
    // Phong variant: the corner normals summed in corner order, renormalised,
    // and lit once (the reference lights the corners and averages)
    float nx = c0.ph[0] + c1.ph[0], ny = c0.ph[1] + c1.ph[1], nz = c0.ph[2] + c1.ph[2];
    nx = nx + c2.ph[0]; ny = ny + c2.ph[1]; nz = nz + c2.ph[2];
    nx = nx + c3.ph[0]; ny = ny + c3.ph[1]; nz = nz + c3.ph[2];
    const float mag = sqrtf(nx * nx + ny * ny + nz * nz);
    nx = nx / mag; ny = ny / mag; nz = nz / mag;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) col[ch] = phong_channel(nx, ny, nz, ch);
  } else {
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      float c = c0.ph[ch] + c1.ph[ch];
      c = c + c2.ph[ch];
      c = c + c3.ph[ch];
      col[ch] = std_minf(c, 4.0f) * 0.25f;
    }
  }
  o.color = (255u << 24) | (cvt_u32_x86(col[2] * 255.0f) << 16) | (cvt_u32_x86(col[1] * 255.0f) << 8) |
            cvt_u32_x86(col[0] * 255.0f);
  o.key = (keyhi | (unsigned long long)local) + 1ull;
  // Shade bins of corners 0..2 (computeBoundingBox + assignToBB)
  // (the reference takes these in double; widening a float is exact and the
  // comparisons are the same, so float std::min / std::max give the same values)
  const float lox = floorf(std_minf(o.sx[0], std_minf(o.sx[1], o.sx[2])));
  const float loy = floorf(std_minf(o.sy[0], std_minf(o.sy[1], o.sy[2])));
  const float hix = ceilf(std_maxf(o.sx[0], std_maxf(o.sx[1], o.sx[2])));
  const float hiy = ceilf(std_maxf(o.sy[0], std_maxf(o.sy[1], o.sy[2])));
  int bx1 = cvt_i32_x86(floorf(lox / 64.0f)), bx2 = cvt_i32_x86(floorf(hix / 64.0f));
  int by1 = cvt_i32_x86(floorf(loy / 64.0f)), by2 = cvt_i32_x86(floorf(hiy / 64.0f));
  if (bx1 < 0) bx1 = 0;
  if (by1 < 0) by1 = 0;
  if (bx2 >= a.nBx) bx2 = a.nBx - 1;
  if (by2 >= a.nBy) by2 = a.nBy - 1;
  // 4-corner bounds intersected with each Shade bin; the bins are adjacent,
  // so the union is one rectangle
  const float bminx = floorf(std_minf(std_minf(o.sx[0], o.sx[1]), std_minf(o.sx[2], o.sx[3])));
  const float bminy = floorf(std_minf(std_minf(o.sy[0], o.sy[1]), std_minf(o.sy[2], o.sy[3])));
  const float bmaxx = ceilf(std_maxf(std_maxf(o.sx[0], o.sx[1]), std_maxf(o.sx[2], o.sx[3])));
  const float bmaxy = ceilf(std_maxf(std_maxf(o.sy[0], o.sy[1]), std_maxf(o.sy[2], o.sy[3])));
  o.x0 = o.x1 = o.y0 = o.y1 = 0;
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
}

// Dice (R12, R13), then fragment pass 1 for micropolygons with at most
// kSmallPx candidate pixels (larger ones are queued for a warp each).
//
// The dice rows of all leaves (row k of a leaf: its micropolygons (k, 0..nv))
// are numbered in leaf-slot order and every CTA takes an equal range of them.
// It works through its range in groups of consecutive rows, possibly spanning
// leaves, of at most kUpBudget micropolygons whose grid points fit in shared
// memory.  For power-of-two grids (every extent-derived grid) k*du + du equals
// (k+1)*du exactly, so the grid points of a group's rows are evaluated once and
// shared by the four micropolygons around each (and the control rows at each
// u once per point row); other fixed grids evaluate the four corners of every
// micropolygon, as the CPU does.  Points and micropolygons of a group are
// spread over all threads whatever the leaves' sizes.
//
// Coverage is sample-parallel: each thread's micropolygon contributes a
// rectangle of cells (one per sample: a pixel quadrant with four samples, the
// pixel with one), cut to the cells exact_box allows; the CTA's cells go to a
// shared list and every thread tests one cell at a time, so lanes stay busy
// whatever the micropolygons' sizes.  A covered cell sets bit (its index in
// the rectangle) of its micropolygon's mask; the owner then emits.
constexpr int kMaxGridPts = 34 * 34;
constexpr int kLeafBatch = 32;     // leaf segments per group
constexpr int kDiceThreads = 256;
constexpr int kUpBudget = 1024;    // micropolygons per group
constexpr int kMaxPtRows = 64;     // grid point rows per group
constexpr int kCellCap = 4096;     // cells per pass of the shared list

struct DiceSmem {
  float4 cp[kLeafBatch][16];
  GridPt gp[kMaxGridPts];
  DiceRow rowdat[kMaxPtRows];                  // control rows at each point row's u
  float4 ux[kDiceThreads], uy[kDiceThreads];   // corners of each thread's micropolygon
  int2 org[kDiceThreads];                      // first cell of its cell rectangle
  uint32_t cwm[kDiceThreads];                  // rectangle width | (2^16 / width + 1) << 7
  unsigned long long mask[kDiceThreads];       // covered cells
  uint16_t cell[kCellCap];                     // (thread << 6) | cell index
  // the group's segments: rows k0 .. of leaf[i]; gpre / upre / rpre = first
  // grid point / micropolygon / point row of each segment in the group
  uint32_t leaf[kLeafBatch], k0[kLeafBatch], nu[kLeafBatch], nv[kLeafBatch];
  unsigned long long keyhi[kLeafBatch];
  uint32_t gpre[kLeafBatch + 1], upre[kLeafBatch + 1], rpre[kLeafBatch + 1];
  uint32_t wnu[32], wnv[32], wrb[32];         // grid and first row of the next 32 leaves
  uint32_t scan[8], append[8];
  uint32_t total, base;
  uint32_t nseg, next_leaf, next_row, found;
};
constexpr size_t kDiceSmem = sizeof(DiceSmem);

// q = n / d and r = n % d for the dice grid's row widths (d = nv + 1 or
// nv + 2 <= 34): a multiply by 0xffffffff / d and one correction
// (fast_divmod); wider rows divide.
struct DivMagic {
  uint32_t m[35];
  constexpr DivMagic() : m() { for (uint32_t d = 1; d < 35; ++d) m[d] = 0xffffffffu / d; }
};
__constant__ DivMagic kRowMagic = DivMagic();
__device__ __forceinline__ uint32_t row_divmod(uint32_t n, uint32_t d, uint32_t& r)
{
  if (d < 35u) return fast_divmod(n, d, kRowMagic.m[d], r);
  r = n % d;
  return n / d;
}

__device__ __forceinline__ int batch_find(const uint32_t* pre, int n, uint32_t f)
{
  int lo = 0, hi = n - 1;   // last i with pre[i] <= f
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= f) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Exclusive block-wide scan of n; *total gets the sum (all threads call it).
__device__ __forceinline__ uint32_t block_scan(uint32_t n, uint32_t* s_warp, uint32_t* total)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = n;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFullR, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t tot = 0;
    for (int w = 0; w < kDiceThreads / 32; ++w) { const uint32_t v = s_warp[w]; s_warp[w] = tot; tot += v; }
    *total = tot;
  }
  __syncthreads();
  return s_warp[warp] + inc - n;
}

// Cell index li of a rectangle cw cells wide: dy = li / cw by multiply-shift
// (exact for li < 64, cw <= 64).
__device__ __forceinline__ void cell_xy(uint32_t cwm, int2 org, int li, int& cx, int& cy)
{
  const int cw = (int)(cwm & 127u);
  const int dy = (int)(((uint32_t)li * (cwm >> 7)) >> 16);
  cx = org.x + li - dy * cw;
  cy = org.y + dy;
}

__device__ __forceinline__ void dice_cell(const ReyesArgs& a, DiceSmem& S, uint32_t q)
{
  const uint32_t e = S.cell[q];
  const int u = (int)(e >> 6), li = (int)(e & 63u);
  int cx, cy;
  cell_xy(S.cwm[u], S.org[u], li, cx, cy);
  float px, py;
  if (a.spp == 1) sample_pos(1, a.seed, cx, cy, 0, px, py);
  else sample_pos(a.spp, a.seed, cx >> 1, cy >> 1, (cx & 1) | ((cy & 1) << 1), px, py);
  if (upoly_covers(S.ux[u], S.uy[u], px, py)) atomicOr(&S.mask[u], 1ull << li);
}

// Three CTAs per SM (at most 80 registers): the extra warps hide more of the
// fixed-latency stalls than the few spilled values cost.
__global__ void __launch_bounds__(kDiceThreads, 3) reyes_dice(ReyesArgs a)
{
  pdl_wait();
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char dice_smem[];
  DiceSmem& S = *reinterpret_cast<DiceSmem*>(dice_smem);
  const unsigned long long meta = a.ctr->leaf_meta;
  const uint32_t nleaf = (uint32_t)(meta >> 40);
  // after a leaf overflow the frame runs again: nothing to dice now
  const unsigned long long R = nleaf <= a.leaf_cap ? (meta & ((1ull << 40) - 1)) : 0ull;
  const uint32_t r_begin = (uint32_t)(R * blockIdx.x / gridDim.x);
  const uint32_t r_end = (uint32_t)(R * (blockIdx.x + 1) / gridDim.x);
  const int r = a.spp == 1 ? 1 : 2;   // cells per pixel edge
  unsigned covered = 0;
  {
    // the last leaf whose first row <= r_begin: kDiceThreads-way search rounds
    // (two for up to 65,536 leaves); leaf lo always qualifies
    uint32_t lo = 0, span = R ? nleaf : 0u;
    while (span > 1) {
      const uint32_t step = (span + kDiceThreads - 1) / kDiceThreads;
      if (threadIdx.x == 0) S.found = 0;
      __syncthreads();
      const uint32_t idx = lo + threadIdx.x * step;
      if (threadIdx.x > 0 && threadIdx.x * step < span && a.leaves[idx].rowbase <= r_begin)
        atomicMax(&S.found, (uint32_t)threadIdx.x);
      __syncthreads();
      const uint32_t t = S.found;
      lo += t * step;
      span = min(step, span - t * step);
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      S.next_leaf = lo;
      S.next_row = r_begin;
    }
  }
  for (;;) {
    __syncthreads();
    const uint32_t row0 = S.next_row, leaf0 = S.next_leaf;
    if (row0 >= r_end) break;   // uniform
    __syncthreads();
    if (threadIdx.x < 32) {
      const uint32_t L = leaf0 + threadIdx.x;
      if (L < nleaf) {
        S.wnu[threadIdx.x] = a.leaves[L].nu;
        S.wnv[threadIdx.x] = a.leaves[L].nv;
        S.wrb[threadIdx.x] = a.leaves[L].rowbase;
      }
      __syncwarp();
      if (threadIdx.x == 0) {
        // rows while the micropolygon budget and the shared grid points allow
        uint32_t g = 0, u = 0, pr = 0, nseg = 0, leaf = leaf0, row = row0;
        while (row < r_end && nseg < (uint32_t)kLeafBatch && leaf < nleaf && leaf - leaf0 < 32u) {
          const uint32_t w = leaf - leaf0, nu = S.wnu[w], nv = S.wnv[w];
          const uint32_t k0 = row - S.wrb[w];
          const bool pow2 = ((nu & (nu - 1)) == 0) && ((nv & (nv - 1)) == 0);
          uint32_t n = min(nu + 1 - k0, r_end - row);
          n = min(n, ((uint32_t)kUpBudget - u) / (nv + 1));
          if (pow2) {   // point rows that still fit
            const uint32_t fit = min(((uint32_t)kMaxGridPts - g) / (nv + 2), (uint32_t)kMaxPtRows - pr);
            n = min(n, fit > 0 ? fit - 1 : 0u);
          }
          if (n == 0) break;
          S.leaf[nseg] = leaf;
          S.k0[nseg] = k0;
          S.nu[nseg] = nu;
          S.nv[nseg] = nv;
          S.gpre[nseg] = g;
          S.upre[nseg] = u;
          S.rpre[nseg] = pr;
          g += pow2 ? (n + 1) * (nv + 2) : 0u;
          pr += pow2 ? n + 1 : 0u;
          u += n * (nv + 1);
          ++nseg;
          row += n;
          if (k0 + n == nu + 1) ++leaf; else break;
        }
        if (nseg == 0) row = r_end;   // rows and leaves disagree (cannot happen): stop, never spin
        S.gpre[nseg] = g;
        S.upre[nseg] = u;
        S.rpre[nseg] = pr;
        S.nseg = nseg;
        S.next_row = row;
        S.next_leaf = leaf;
      }
    }
    __syncthreads();
    const int m = (int)S.nseg;
    for (int q = threadIdx.x; q < m * 16; q += blockDim.x) S.cp[q >> 4][q & 15] = a.leaves[S.leaf[q >> 4]].cp[q & 15];
    if (threadIdx.x < m) {
      const PatchRec& p = a.leaves[S.leaf[threadIdx.x]];
      S.keyhi[threadIdx.x] = leaf_key(a, p.i0, p.level, p.s);
    }
    __syncthreads();
    const uint32_t gtot = S.gpre[m], utot = S.upre[m], rtot = S.rpre[m];
    for (uint32_t t = threadIdx.x; t < rtot; t += blockDim.x) {
      const int i = batch_find(S.rpre, m, t);
      const uint32_t k = S.k0[i] + (t - S.rpre[i]);
      dice_row(S.cp[i], (float)k * (1.0f / ((float)S.nu[i])), S.rowdat[t]);
    }
    __syncthreads();
    for (uint32_t f = threadIdx.x; f < gtot; f += blockDim.x) {
      const int i = batch_find(S.gpre, m, f);
      const uint32_t nv = S.nv[i], g = f - S.gpre[i];
      uint32_t j;
      const uint32_t kk = row_divmod(g, nv + 2, j);
      grid_point_row(S.rowdat[S.rpre[i] + kk], a, (float)j * (1.0f / ((float)nv)), S.gp[f]);
    }
    __syncthreads();
    for (uint32_t f0 = 0; f0 < utot; f0 += blockDim.x) {
      const uint32_t f = f0 + threadIdx.x;
      UpolyRec o;
      int cnt = 0;          // cells to test
      uint32_t cwm = 0;
      int2 org = make_int2(0, 0);
      if (f < utot) {
        const int i = batch_find(S.upre, m, f);
        const uint32_t nu = S.nu[i], nv = S.nv[i], tl = f - S.upre[i];
        const uint32_t nv1 = nv + 1;
        uint32_t j;
        const uint32_t kk = row_divmod(tl, nv1, j);                  // row kk of the segment
        const uint32_t k = S.k0[i] + kk, t = k * nv1 + j;             // micropolygon t of the leaf
        const bool pow2 = ((nu & (nu - 1)) == 0) && ((nv & (nv - 1)) == 0);
        if (pow2) {
          const GridPt* gp = S.gp + S.gpre[i];
          const uint32_t gw = nv + 2;
          make_upoly(a, S.keyhi[i], t, gp[kk * gw + j], gp[(kk + 1) * gw + j], gp[(kk + 1) * gw + j + 1],
                     gp[kk * gw + j + 1], o);
        } else {
          const float du = 1.0f / ((float)nu), dv = 1.0f / ((float)nv);
          const float myU = (float)k * du, myV = (float)j * dv;
          GridPt c0, c1, c2, c3;
          grid_point(S.cp[i], a, myU, myV, c0);
          grid_point(S.cp[i], a, myU + du, myV, c1);
          grid_point(S.cp[i], a, myU + du, myV + dv, c2);
          grid_point(S.cp[i], a, myU, myV + dv, c3);
          make_upoly(a, S.keyhi[i], t, c0, c1, c2, c3, o);
        }
        if (o.z < 0.0f) atomicAdd(&a.ctr->negative_depth, 1u);
        const int n = (o.x1 - o.x0) * (o.y1 - o.y0);
        if (n > kSmallPx) {
          const uint32_t b = atomicAdd(&a.ctr->big_count, 1u);
          if (b < a.up_cap) {
            const uint4* src = reinterpret_cast<const uint4*>(&o);
            uint4* dst = reinterpret_cast<uint4*>(&a.up[b]);
#pragma unroll
            for (int q = 0; q < 4; ++q) dst[q] = src[q];
          } else {
            atomicOr(&a.ctr->fc.status, kStatusUpolyOverflow);
          }
        } else if (n > 0) {
          int cx0 = o.x0 * r, cx1 = o.x1 * r - 1, cy0 = o.y0 * r, cy1 = o.y1 * r - 1;
          const float mnx = std_minf(std_minf(o.sx[0], o.sx[1]), std_minf(o.sx[2], o.sx[3]));
          const float mxx = std_maxf(std_maxf(o.sx[0], o.sx[1]), std_maxf(o.sx[2], o.sx[3]));
          const float mny = std_minf(std_minf(o.sy[0], o.sy[1]), std_minf(o.sy[2], o.sy[3]));
          const float mxy = std_maxf(std_maxf(o.sy[0], o.sy[1]), std_maxf(o.sy[2], o.sy[3]));
          if (exact_box(mnx, mxx, mny, mxy)) {
            if (r == 1) {   // centre x + 0.5 strictly inside (mnx, mxx)
              cx0 = max(cx0, (int)floorf(mnx - 0.5f) + 1); cx1 = min(cx1, (int)ceilf(mxx - 0.5f) - 1);
              cy0 = max(cy0, (int)floorf(mny - 0.5f) + 1); cy1 = min(cy1, (int)ceilf(mxy - 0.5f) - 1);
            } else {        // quadrant q spans [q / 2, q / 2 + 1/2]
              cx0 = max(cx0, (int)floorf(2.0f * mnx)); cx1 = min(cx1, (int)ceilf(2.0f * mxx) - 1);
              cy0 = max(cy0, (int)floorf(2.0f * mny)); cy1 = min(cy1, (int)ceilf(2.0f * mxy) - 1);
            }
          }
          const int cw = cx1 - cx0 + 1, ch = cy1 - cy0 + 1;
          if (cw > 0 && ch > 0) {
            cnt = cw * ch;
            cwm = (uint32_t)cw | ((0x10000u / (uint32_t)cw + 1u) << 7);
            org = make_int2(cx0, cy0);
            S.ux[threadIdx.x] = make_float4(o.sx[0], o.sx[1], o.sx[2], o.sx[3]);
            S.uy[threadIdx.x] = make_float4(o.sy[0], o.sy[1], o.sy[2], o.sy[3]);
            S.org[threadIdx.x] = org;
            S.cwm[threadIdx.x] = cwm;
            S.mask[threadIdx.x] = 0ull;
          }
        }
      }
      const uint32_t pre = block_scan((uint32_t)cnt, S.scan, &S.total);
      const uint32_t total = S.total;
      for (uint32_t w0 = 0; w0 < total; w0 += kCellCap) {
        const int lo = max(0, (int)w0 - (int)pre), hi = min(cnt, (int)(w0 + kCellCap) - (int)pre);
        for (int c = lo; c < hi; ++c) S.cell[pre + (uint32_t)c - w0] = (uint16_t)((threadIdx.x << 6) | (uint32_t)c);
        __syncthreads();
        const uint32_t nw = min((uint32_t)kCellCap, total - w0);
        for (uint32_t q = threadIdx.x; q < nw; q += blockDim.x) dice_cell(a, S, q);
        __syncthreads();
      }
      unsigned long long mask = cnt > 0 ? S.mask[threadIdx.x] : 0ull;
      covered += __popcll(mask);
      if (cnt > 0 && !(o.z <= 1.0f)) mask = 0;  // behind the cleared depth (or NaN): never survives
      uint32_t slot = block_append(a, __popcll(mask), S.append, &S.base);
      while (mask) {
        const int c = __ffsll(mask) - 1;
        mask &= mask - 1;
        int cx, cy;
        cell_xy(cwm, org, c, cx, cy);
        if (r == 1) emit_fragment(a, slot++, o, cx, cy, 0);
        else emit_fragment(a, slot++, o, cx >> 1, cy >> 1, (cx & 1) | ((cy & 1) << 1));
      }
    }
  }
  add_covered(a, covered);
}

// Fragment pass 1 for the queued micropolygons: a warp each, a lane per pixel.
__global__ void __launch_bounds__(256) reyes_big(ReyesArgs a)
{
  pdl_wait();
  pdl_trigger();
  const uint32_t nbig = min(a.ctr->big_count, a.up_cap);
  const int lane = threadIdx.x & 31;
  const uint32_t nwarps = gridDim.x * (blockDim.x / 32);
  unsigned covered = 0;
  for (uint32_t wi = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; wi < nbig; wi += nwarps) {
    UpolyRec u;
    const uint4* src = reinterpret_cast<const uint4*>(&a.up[wi]);
    uint4* dst = reinterpret_cast<uint4*>(&u);
#pragma unroll
    for (int q = 0; q < 4; ++q) dst[q] = src[q];
    const int bw = u.x1 - u.x0;
    const int n = bw * (u.y1 - u.y0) * a.spp;   // candidate samples
    for (int k0 = 0; k0 < n; k0 += 32) {
      const int k = k0 + lane;
      const int pk = k / a.spp, smp = k - pk * a.spp;
      const int x = u.x0 + (bw ? pk % bw : 0), y = u.y0 + (bw ? pk / bw : 0);
      float px = 0.0f, py = 0.0f;
      if (k < n) sample_pos(a.spp, a.seed, x, y, smp, px, py);
      const bool cov = k < n && upoly_covers(make_float4(u.sx[0], u.sx[1], u.sx[2], u.sx[3]),
                                              make_float4(u.sy[0], u.sy[1], u.sy[2], u.sy[3]), px, py);
      const unsigned m = __ballot_sync(kFullR, cov);
      covered += cov ? 1u : 0u;
      const unsigned keep = (u.z <= 1.0f) ? m : 0u;
      uint32_t base = 0;
      if (lane == 0 && keep) base = atomicAdd(&a.ctr->frag_count, (uint32_t)__popc(keep));
      base = __shfl_sync(kFullR, base, 0);
      if (keep & (1u << lane)) emit_fragment(a, base + __popc(keep & ((1u << lane) - 1u)), u, x, y, smp);
    }
  }
  add_covered(a, covered);
}

// Passes 2 and 3 are bound by the latency of dependent loads (fragment, then
// its sample's minimum, then its keys): a thread takes kFragBatch fragments of
// its grid-stride range at a time and issues each level of loads for all of
// them before the next.  The fragments are independent, so the order changes
// nothing.
constexpr int kFragBatch = 4;

// Key, sample index and depth of a fragment: its first 16 bytes in one load.
struct FragHead {
  unsigned long long key;
  uint32_t pix;
  float z;
};

__device__ __forceinline__ FragHead frag_head(const FragRec* f, uint32_t i)
{
  const uint4 q = __ldg(reinterpret_cast<const uint4*>(&f[i]));
  FragHead h;
  h.key = (unsigned long long)q.x | ((unsigned long long)q.y << 32);
  h.pix = q.z;
  h.z = __uint_as_float(q.w);
  return h;
}

// Fragment pass 2: greatest key among the fragments at the minimum (the
// colour), and the least one where the minimum is +-0 (the only depth whose
// fragments can differ in their bits: elsewhere every fragment at the minimum
// carries the same bits, and the colour's fragment writes them).
__global__ void __launch_bounds__(256) reyes_keys(ReyesArgs a)
{
  pdl_wait();
  pdl_trigger();
  const uint32_t n = min(a.ctr->frag_count, a.frag_cap);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += kFragBatch * stride) {
    FragHead h[kFragBatch];
    bool ok[kFragBatch];
    uint32_t zm[kFragBatch];
#pragma unroll
    for (int u = 0; u < kFragBatch; ++u) {
      ok[u] = (uint32_t)u * stride < n - i0;
      if (ok[u]) h[u] = frag_head(a.frags, i0 + (uint32_t)u * stride);
    }
#pragma unroll
    for (int u = 0; u < kFragBatch; ++u) zm[u] = ok[u] ? a.zmin[h[u].pix] : 0u;
#pragma unroll
    for (int u = 0; u < kFragBatch; ++u) {
      if (!ok[u] || !(h[u].z == zorder_inv(zm[u]))) continue;
      atomicMax(&a.klast[h[u].pix], h[u].key);
      if (h[u].z == 0.0f) atomicMin(&a.kfirst[h[u].pix], h[u].key);
    }
  }
}

// Fragment pass 3: the last fragment at the minimum writes the colour and the
// depth; at a minimum of +-0 the first one writes the depth bits.
__global__ void __launch_bounds__(256) reyes_resolve(ReyesArgs a)
{
  pdl_wait();
  pdl_trigger();
  const uint32_t n = min(a.ctr->frag_count, a.frag_cap);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += kFragBatch * stride) {
    FragHead h[kFragBatch];
    uint32_t col[kFragBatch], zm[kFragBatch];
    bool at[kFragBatch];
    unsigned long long kl[kFragBatch], kf[kFragBatch];
#pragma unroll
    for (int u = 0; u < kFragBatch; ++u) {
      at[u] = (uint32_t)u * stride < n - i0;
      if (at[u]) {
        const uint32_t i = i0 + (uint32_t)u * stride;
        h[u] = frag_head(a.frags, i);
        col[u] = __ldg(&a.frags[i].color);
      }
    }
#pragma unroll
    for (int u = 0; u < kFragBatch; ++u) zm[u] = at[u] ? a.zmin[h[u].pix] : 0u;
#pragma unroll
    for (int u = 0; u < kFragBatch; ++u) {
      at[u] = at[u] && h[u].z == zorder_inv(zm[u]);
      kl[u] = at[u] ? a.klast[h[u].pix] : 0ull;
      kf[u] = (at[u] && h[u].z == 0.0f) ? a.kfirst[h[u].pix] : 0ull;
    }
#pragma unroll
    for (int u = 0; u < kFragBatch; ++u) {
      if (!at[u]) continue;
      const bool last = kl[u] == h[u].key;
      const bool dep = h[u].z == 0.0f ? kf[u] == h[u].key : last;
      const uint32_t p = h[u].pix;
      if (a.spp == 1) {
        if (last) a.fb[p] = col[u];
        if (dep) a.depth[p] = h[u].z;
      } else {
        if (last) a.scol[p] = col[u];
        if (dep) a.sdep[p] = h[u].z;
      }
    }
  }
}

// The last pass, over every pixel.  One sample per pixel: a pixel no fragment
// reached gets the clear colour and depth 1 (the resolve wrote the others).
// More samples: a pixel takes the rounded mean of its samples' colours per
// channel (the clear colour where no fragment reached a sample) and the depth
// of its nearest sample (the first such sample on ties).  Either way every
// reached sample's depth minimum and key bounds are set back to empty, so the
// next frame finds the per-sample state cleared.
__global__ void __launch_bounds__(256) reyes_pixels(ReyesArgs a, uint32_t npx)
{
  pdl_wait();
  const uint32_t spp = (uint32_t)a.spp;
  if (spp == 4) {
    // a pixel's four samples are 16 (u32) or 32 (u64) contiguous, aligned
    // bytes: one vector access per array; a pixel with any reached sample has
    // all four set back (a sample not reached already holds the empty state)
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npx; i += gridDim.x * blockDim.x) {
      const size_t s0 = 4 * (size_t)i;
      const uint4 zm = *reinterpret_cast<const uint4*>(&a.zmin[s0]);
      const bool r[4] = {zm.x != kZminEmpty, zm.y != kZminEmpty, zm.z != kZminEmpty, zm.w != kZminEmpty};
      uint32_t c[4] = {kClearColor, kClearColor, kClearColor, kClearColor};
      float z[4] = {1.0f, 1.0f, 1.0f, 1.0f};
      if (r[0] || r[1] || r[2] || r[3]) {
        const uint4 sc = *reinterpret_cast<const uint4*>(&a.scol[s0]);
        const float4 sd = *reinterpret_cast<const float4*>(&a.sdep[s0]);
        *reinterpret_cast<uint4*>(&a.zmin[s0]) = make_uint4(kZminEmpty, kZminEmpty, kZminEmpty, kZminEmpty);
        ulonglong2* kl = reinterpret_cast<ulonglong2*>(&a.klast[s0]);
        ulonglong2* kf = reinterpret_cast<ulonglong2*>(&a.kfirst[s0]);
        kl[0] = make_ulonglong2(0ull, 0ull);
        kl[1] = make_ulonglong2(0ull, 0ull);
        kf[0] = make_ulonglong2(~0ull, ~0ull);
        kf[1] = make_ulonglong2(~0ull, ~0ull);
        const uint32_t scv[4] = {sc.x, sc.y, sc.z, sc.w};
        const float sdv[4] = {sd.x, sd.y, sd.z, sd.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          if (r[k]) { c[k] = scv[k]; z[k] = sdv[k]; }
        }
      }
      uint32_t sum[3] = {0u, 0u, 0u};
      float best = 1.0f;
      uint32_t best_o = 0xffffffffu;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        sum[0] += c[k] & 255u;
        sum[1] += (c[k] >> 8) & 255u;
        sum[2] += (c[k] >> 16) & 255u;
        const uint32_t o = zorder(z[k]);
        if (k == 0 || o < best_o) { best_o = o; best = z[k]; }
      }
      a.fb[i] = 0xff000000u | (((sum[2] + 2u) / 4u) << 16) | (((sum[1] + 2u) / 4u) << 8) | ((sum[0] + 2u) / 4u);
      a.depth[i] = best;
    }
    return;
  }
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npx; i += gridDim.x * blockDim.x) {
    uint32_t sum[3] = {0u, 0u, 0u};
    float best = 1.0f;
    uint32_t best_o = 0xffffffffu;
    bool any = false;
    for (uint32_t k = 0; k < spp; ++k) {
      const uint32_t si = i * spp + k;
      const bool reached = a.zmin[si] != kZminEmpty;
      if (reached) {
        a.zmin[si] = kZminEmpty;
        a.klast[si] = 0ull;
        a.kfirst[si] = ~0ull;
        any = true;
      }
      if (spp == 1) continue;
      const uint32_t c = reached ? a.scol[si] : kClearColor;
      const float z = reached ? a.sdep[si] : 1.0f;
      sum[0] += c & 255u;
      sum[1] += (c >> 8) & 255u;
      sum[2] += (c >> 16) & 255u;
      const uint32_t o = zorder(z);
      if (k == 0 || o < best_o) { best_o = o; best = z; }
    }
    if (spp == 1) {
      if (!any) {
        a.fb[i] = kClearColor;
        a.depth[i] = 1.0f;
      }
      continue;
    }
    a.fb[i] = 0xff000000u | (((sum[2] + spp / 2u) / spp) << 16) | (((sum[1] + spp / 2u) / spp) << 8) |
              ((sum[0] + spp / 2u) / spp);
    a.depth[i] = best;
  }
}

// A launch that may begin while the previous kernel of the stream finishes
// (the kernel's pdl_wait() holds it until that kernel's writes are visible).
template <typename... KArgs, typename... Args>
static cudaError_t launch_chained(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t st,
                                  Args... args)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

cudaError_t launch_reyes_frame(const ReyesArgs& a, uint32_t npx, int sms, cudaStream_t st, cudaEvent_t* ev)
{
  // occupancies, found once per process (host threads may launch frames
  // concurrently; call_once makes the others wait for the first)
  static std::once_flag once;
  static int dice_per_sm = 1;
  static cudaError_t setup_err = cudaSuccess;
  std::call_once(once, [] {
    int sp = 0, dp = 1;
    cudaError_t e = cudaFuncSetAttribute(reyes_split, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSplitSmem);
    if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sp, reyes_split, kSplitThreads, kSplitSmem);
    // the split's grid barriers need every CTA resident: one per SM
    if (!e && sp < 1) e = cudaErrorCooperativeLaunchTooLarge;
    if (!e) e = cudaFuncSetAttribute(reyes_dice, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDiceSmem);
    if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&dp, reyes_dice, kDiceThreads, kDiceSmem);
    setup_err = e;
    dice_per_sm = std::max(1, dp);
  });
  if (setup_err) return setup_err;
  if (ev) cudaEventRecord(ev[0], st);
  ReyesArgs args = a;
  void* params[] = {(void*)&args};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)reyes_split, dim3(sms), dim3(kSplitThreads), params,
                                              kSplitSmem, st);
  if (e != cudaSuccess) return e;
  if (ev) cudaEventRecord(ev[1], st);
  // the launches after the split may start while their predecessor drains
  // (programmatic dependent launch); each waits for it before touching memory
  const int grid = sms * 8;
  e = launch_chained(reyes_dice, sms * dice_per_sm, kDiceThreads, kDiceSmem, st, a);
  if (!e) e = launch_chained(reyes_big, grid, 256, 0, st, a);
  if (ev) cudaEventRecord(ev[2], st);
  if (!e) e = launch_chained(reyes_keys, grid, 256, 0, st, a);
  if (ev) cudaEventRecord(ev[3], st);
  if (!e) e = launch_chained(reyes_resolve, grid, 256, 0, st, a);
  if (!e) e = launch_chained(reyes_pixels, grid, 256, 0, st, a, npx);
  if (ev) cudaEventRecord(ev[4], st);
  if (e) return e;
  return cudaGetLastError();
}

}  // namespace piko

using namespace piko;

// ------------------------------------------------------------------ host state
// Work buffers and counters of a Reyes scene.  A scene may borrow the work
// buffers of another state (`buffers`): frames run in stream order on one
// stream can share them (the served form gives each stream lane one set),
// while every scene keeps its own counters for its overflow checks.
struct ReyesState {
  ReyesState* buffers = nullptr;  // borrowed work buffers (not owned), or null
  PatchRec* lvl[2] = {nullptr, nullptr};
  PatchRec* leaves = nullptr;
  UpolyRec* up = nullptr;
  FragRec* frags = nullptr;
  uint32_t lvl_cap = 0, leaf_cap = 0, up_cap = 0, frag_cap = 0;
  uint32_t* zmin = nullptr;
  unsigned long long* kfirst = nullptr;
  unsigned long long* klast = nullptr;
  uint32_t* scol = nullptr;
  float* sdep = nullptr;
  size_t npx_cap = 0;   // samples
  bool clean = false;   // per-sample state all empty (set when allocated; every frame leaves it so)
  ReyesCounters* ctr = nullptr;
  ReyesCounters* h_ctr = nullptr;
  cudaEvent_t ev[5] = {};
  bool ev_made = false;
};

static void reyes_state_free(ReyesState* r)
{
  dfree(r->lvl[0]); dfree(r->lvl[1]); dfree(r->leaves); dfree(r->up); dfree(r->frags);
  dfree(r->zmin); dfree(r->kfirst); dfree(r->klast); dfree(r->scol); dfree(r->sdep); dfree(r->ctr);
  if (r->h_ctr) cudaFreeHost(r->h_ctr);
  if (r->ev_made) for (auto& e : r->ev) cudaEventDestroy(e);
  delete r;
}

void piko_reyes_release(piko_scene* s)
{
  if (!s->reyes) return;
  reyes_state_free(s->reyes);
  s->reyes = nullptr;
}

ReyesState* reyes_buffers_new() { return new ReyesState(); }
void reyes_buffers_free(ReyesState* b)
{
  if (b) reyes_state_free(b);
}
void reyes_borrow_buffers(piko_scene* s, ReyesState* b)
{
  if (!s->reyes) s->reyes = new ReyesState();
  s->reyes->buffers = b;
}

static cudaError_t reyes_alloc(ReyesState* r, uint32_t lvl_cap, uint32_t leaf_cap, uint32_t up_cap, uint32_t frag_cap,
                               size_t npx)
{
  cudaError_t e = cudaSuccess;
  if (r->buffers) {
    if ((e = reyes_alloc(r->buffers, lvl_cap, leaf_cap, up_cap, frag_cap, npx))) return e;
    lvl_cap = leaf_cap = up_cap = frag_cap = 0;
    npx = 0;
  }
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
  if (frag_cap > r->frag_cap) {
    dfree(r->frags);
    if ((e = dalloc(&r->frags, frag_cap))) return e;
    r->frag_cap = frag_cap;
  }
  if (npx > r->npx_cap) {
    dfree(r->zmin); dfree(r->kfirst); dfree(r->klast); dfree(r->scol); dfree(r->sdep);
    r->npx_cap = 0;
    r->clean = false;
    if ((e = dalloc(&r->zmin, npx)) || (e = dalloc(&r->kfirst, npx)) || (e = dalloc(&r->klast, npx)) ||
        (e = dalloc(&r->scol, npx)) || (e = dalloc(&r->sdep, npx)))
      return e;
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
  ReyesState* b = r->buffers ? r->buffers : r;
  const uint32_t P = (uint32_t)s->N;
  const size_t npx = (size_t)s->W * (size_t)s->H;
  const size_t nsamp = npx * (size_t)p->samples_per_pixel;
  CU(ctx, reyes_alloc(r, std::max<uint32_t>(1u << 16, 64u * P), std::max<uint32_t>(1u << 16, 64u * P),
                      b->up_cap ? b->up_cap : (1u << 16),
                      b->frag_cap ? b->frag_cap : (uint32_t)std::max<size_t>(1u << 20, nsamp), nsamp));
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
  a.lvl[0] = b->lvl[0]; a.lvl[1] = b->lvl[1]; a.lvl_cap = b->lvl_cap;
  a.leaves = b->leaves; a.leaf_cap = b->leaf_cap;
  a.up = b->up; a.up_cap = b->up_cap;
  a.frags = b->frags; a.frag_cap = b->frag_cap;
  a.ctr = r->ctr;
  a.fb = s->fb; a.depth = s->depth;
  a.zmin = b->zmin; a.kfirst = b->kfirst; a.klast = b->klast;
  a.spp = p->samples_per_pixel;
  a.seed = p->sample_seed;
  a.phong = p->phong;
  a.scol = b->scol; a.sdep = b->sdep;
  if (!b->clean) {
    // fresh sample buffers, or a frame whose launches failed part way
    CU(ctx, cudaMemsetAsync(b->zmin, 0xff, sizeof(uint32_t) * b->npx_cap, st));
    CU(ctx, cudaMemsetAsync(b->kfirst, 0xff, sizeof(unsigned long long) * b->npx_cap, st));
    CU(ctx, cudaMemsetAsync(b->klast, 0, sizeof(unsigned long long) * b->npx_cap, st));
    b->clean = true;
  }
  const cudaError_t le = launch_reyes_frame(a, (uint32_t)npx, ctx->sms, st, timed ? r->ev : nullptr);
  if (le != cudaSuccess) b->clean = false;
  CU(ctx, le);
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
    if (st & kStatusBarrierTimeout) return set_err(ctx, PIKO_ERR_TIMEOUT, "%s", "split level barrier timed out");
    if (!(st & (kStatusPatchOverflow | kStatusUpolyOverflow | kStatusListOverflow))) {
      s->pending = false;
      return PIKO_OK;
    }
    uint32_t maxlvl = 0;
    for (int i = 0; i < 40; ++i) maxlvl = std::max(maxlvl, c.level_count[i]);
    const uint32_t leaves = (uint32_t)(c.leaf_meta >> 40);
    const ReyesState* b = r->buffers ? r->buffers : r;
    uint32_t lvl = b->lvl_cap, lf = b->leaf_cap, up = b->up_cap, fr = b->frag_cap;
    if (st & kStatusPatchOverflow) { lvl = std::max(lvl, maxlvl + maxlvl / 2 + 1024); lf = std::max(lf, 2 * leaves + 1024); }
    if (st & kStatusUpolyOverflow) up = (uint32_t)std::min<unsigned long long>(c.big_count + c.big_count / 4ull + 4096, 0xffffffffull);
    if (st & kStatusListOverflow) fr = (uint32_t)std::min<unsigned long long>(c.frag_count + c.frag_count / 4ull + 4096, 0xffffffffull);
    CU(ctx, reyes_alloc(r, lvl, lf, up, fr, b->npx_cap));
    piko_status rr = piko_reyes_run(s, s->last_stream, s->timed);
    if (rr != PIKO_OK) return rr;
  }
  return set_err(ctx, PIKO_ERR_QUEUE_OVERFLOW, "%s", "Reyes queues kept overflowing");
}

namespace piko {
// One CTA waiting at level barrier 0 with no CTA to release it: the bounded
// wait must give up and record kStatusBarrierTimeout.
__global__ void __launch_bounds__(32) reyes_wait_selftest(ReyesCounters* c)
{
  __shared__ uint32_t s_count;
  barrier_wait(c, 0u, &s_count);
}
}  // namespace piko

extern "C" piko_status piko_selftest_wait_timeout(piko_ctx* ctx)
{
  if (!ctx) return PIKO_ERR_INVALID;
  cudaSetDevice(ctx->device);
  ReyesCounters* d = nullptr;
  CU(ctx, dalloc(&d, 1));
  ReyesCounters h;
  cudaError_t e = cudaMemset(d, 0, sizeof(ReyesCounters));
  if (!e) {
    reyes_wait_selftest<<<1, 32>>>(d);
    e = cudaGetLastError();
  }
  if (!e) e = cudaMemcpy(&h, d, sizeof(ReyesCounters), cudaMemcpyDeviceToHost);
  cudaFree(d);
  CU(ctx, e);
  if (h.fc.status & kStatusBarrierTimeout)
    return set_err(ctx, PIKO_ERR_TIMEOUT, "%s", "self-test: the bounded barrier wait gave up as designed");
  return PIKO_OK;
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
  o->upolys = c.upolys;
  o->bin_entries = c.big_count;   // micropolygons shaded a warp each
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
