/* TEST INFRASTRUCTURE — the oracle's CPU restatement of the Reyes path.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * as the checker; the product path never links or calls it.
 *
 * It restates what the reference's ReyesPipe computes when its CPU backend runs
 * with one thread (the Split self-loop runs level by level:
 * pikoc/src/Backend/CPUBackend.cpp:460-516, pikoc/src/pikoc.cpp:294-308):
 *   R11 SplitStage::process   pikoc/samples/reyesPipe/split.pikostage:240-343
 *       (getUVPixelExtents :47-94, splitU/V :95-224, pow2roundup :34-45)
 *   R12 DiceStage             dice.pikostage:149-312 (patchEval :111-121,
 *       normEval :123-146, Bernstein terms :85-93)
 *   R13 ShadeStage            shade.pikostage:51-258 (phongShadeReyes :64-85,
 *       computeLighting :22-30 with its arguments as the call site passes them)
 * Three parameters generalise constants the reference hard-codes: the split
 * threshold (THRESHOLD_PIXELS = 4.0f), the split limit (20) and an optional
 * fixed dice grid (the reference derives nu, nv from the extents).  With
 * threshold 4, limit 20 and grid 0 this is the reference's pipeline.
 */
#include <stdlib.h>
#include <stdio.h>
#include "oracle_common.h"

typedef struct { float x, y, z, w; } f4;
typedef struct {
  f4 cp[16];
  int numSplits, nu, nv, id;
} patch;

static f4 add4(f4 a, f4 b) { f4 r = {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; return r; }
static f4 mul4(f4 a, float k) { f4 r = {a.x * k, a.y * k, a.z * k, a.w * k}; return r; }

static f4 matmul4(const float* m, f4 v)
{
  /* piko::matmultfloat4 (cvec4f), piko/math.h:395-403 */
  f4 o;
  o.x = m[0] * v.x + m[4] * v.y + m[8] * v.z + m[12] * v.w;
  o.y = m[1] * v.x + m[5] * v.y + m[9] * v.z + m[13] * v.w;
  o.z = m[2] * v.x + m[6] * v.y + m[10] * v.z + m[14] * v.w;
  o.w = m[3] * v.x + m[7] * v.y + m[11] * v.z + m[15] * v.w;
  return o;
}

static float dist2(float ax, float ay, float bx, float by)
{
  float cx = ax - bx, cy = ay - by;
  return sqrtf(cx * cx + cy * cy);
}

static int pow2roundup(int x)
{
  if (x < 0) return 0;
  --x;
  x |= x >> 1; x |= x >> 2; x |= x >> 4; x |= x >> 8; x |= x >> 16;
  return x + 1;
}

static int cvt_i32_d(double d)
{
  if (!(d >= -2147483648.0 && d < 2147483648.0)) return INT32_MIN;
  return (int)d;
}

static void split_uv(const f4* cp, f4* a, f4* b, int along_u)
{
  for (int i = 0; i < 4; ++i) {
    int c0, c1, c2, c3;
    if (along_u) { c0 = i * 4; c1 = c0 + 1; c2 = c0 + 2; c3 = c0 + 3; }
    else { c0 = i; c1 = i + 4; c2 = i + 8; c3 = i + 12; }
    a[c0] = cp[c0];
    b[c3] = cp[c3];
    a[c1] = mul4(add4(cp[c0], cp[c1]), 0.5f);
    b[c2] = mul4(add4(cp[c2], cp[c3]), 0.5f);
    f4 t = mul4(add4(cp[c1], cp[c2]), 0.5f);
    a[c2] = mul4(add4(a[c1], t), 0.5f);
    b[c1] = mul4(add4(b[c2], t), 0.5f);
    a[c3] = mul4(add4(a[c2], b[c1]), 0.5f);
    b[c0] = a[c3];
  }
}

/* returns 1 = split into *c1,*c2; 0 = leaf (nu, nv filled) */
static int split_process(patch* p, const float* vp, int W, int H, float thr, int max_splits,
                         int grid, patch* c1, patch* c2)
{
  float cl[64];
  for (int i = 0; i < 16; ++i) {
    f4 c = matmul4(vp, p->cp[i]);
    if (c.w == 0.0f) c.w = 1.0f;
    c.x /= c.w; c.y /= c.w; c.z /= c.w;
    c.x = (float)(((double)c.x + 1.0) * 0.5 * (double)W);
    c.y = (float)(((double)c.y + 1.0) * 0.5 * (double)H);
    cl[i * 4 + 0] = c.x; cl[i * 4 + 1] = c.y; cl[i * 4 + 2] = c.z; cl[i * 4 + 3] = c.w;
  }
  float ue = 0.0f, ve = 0.0f;
  for (int i = 0; i < 4; ++i) {
    const float* r = cl + i * 16;
    float s = dist2(r[0], r[1], r[4], r[5]) + dist2(r[4], r[5], r[8], r[9]) + dist2(r[8], r[9], r[12], r[13]);
    ue = std_maxf(ue, s);
  }
  for (int i = 0; i < 4; ++i) {
    const float* c = cl + i * 4;
    float s = dist2(c[0], c[1], c[16], c[17]) + dist2(c[16], c[17], c[32], c[33]) + dist2(c[32], c[33], c[48], c[49]);
    ve = std_maxf(ve, s);
  }
  int split = (ue >= thr) || (ve >= thr);
  if (p->numSplits >= max_splits) split = 0;
  if (split) {
    split_uv(p->cp, c1->cp, c2->cp, ue >= thr);
    c1->numSplits = c2->numSplits = p->numSplits + 1;
    c1->id = c2->id = p->id + c1->numSplits;
    c1->nu = c1->nv = c2->nu = c2->nv = 0;
    return 1;
  }
  int nu = pow2roundup(cvt_i32_d(ceil((double)(ue / thr))) + 1);
  int nv = pow2roundup(cvt_i32_d(ceil((double)(ve / thr))) + 1);
  if (nu < 2) nu = 2;
  if (nv < 2) nv = 2;
  if (nu > 32) nu = 32;
  if (nv > 32) nv = 32;
  if (grid > 0) { nu = grid; nv = grid; }
  p->nu = nu; p->nv = nv;
  return 0;
}

/* ---------------------------------------------------------------- dice */
static float B0(float u) { return ((1.0f - u) * (1.0f - u) * (1.0f - u)); }
static float B1(float u) { return ((3.0f * u) * (1.0f - u) * (1.0f - u)); }
static float B2(float u) { return ((3.0f * u) * (u - u * u)); }
static float B3(float u) { return ((u) * (u * u)); }
static float dB0(float u) { return (-3.0f * (1.0f - u) * (1.0f - u)); }
static float dB1(float u) { return (3.0f * (1.0f - u) * (1.0f - 3.0f * u)); }
static float dB2(float u) { return (3.0f * u * (2.0f - 3.0f * u)); }
static float dB3(float u) { return (3.0f * u * u); }

static f4 bez(float t, f4 a, f4 b, f4 c, f4 d)
{
  f4 o;
  o.x = B0(t) * a.x + B1(t) * b.x + B2(t) * c.x + B3(t) * d.x;
  o.y = B0(t) * a.y + B1(t) * b.y + B2(t) * c.y + B3(t) * d.y;
  o.z = B0(t) * a.z + B1(t) * b.z + B2(t) * c.z + B3(t) * d.z;
  o.w = B0(t) * a.w + B1(t) * b.w + B2(t) * c.w + B3(t) * d.w;
  return o;
}
static f4 dbez(float t, f4 a, f4 b, f4 c, f4 d)
{
  f4 o;
  o.x = dB0(t) * a.x + dB1(t) * b.x + dB2(t) * c.x + dB3(t) * d.x;
  o.y = dB0(t) * a.y + dB1(t) * b.y + dB2(t) * c.y + dB3(t) * d.y;
  o.z = dB0(t) * a.z + dB1(t) * b.z + dB2(t) * c.z + dB3(t) * d.z;
  o.w = dB0(t) * a.w + dB1(t) * b.w + dB2(t) * c.w + dB3(t) * d.w;
  return o;
}
static f4 patch_eval(const f4* P, float u, float v)
{
  f4 r0 = bez(u, P[0], P[1], P[2], P[3]), r1 = bez(u, P[4], P[5], P[6], P[7]);
  f4 r2 = bez(u, P[8], P[9], P[10], P[11]), r3 = bez(u, P[12], P[13], P[14], P[15]);
  return bez(v, r0, r1, r2, r3);
}
static f4 norm_eval(const f4* P, float u, float v)
{
  f4 r0 = dbez(u, P[0], P[1], P[2], P[3]), r1 = dbez(u, P[4], P[5], P[6], P[7]);
  f4 r2 = dbez(u, P[8], P[9], P[10], P[11]), r3 = dbez(u, P[12], P[13], P[14], P[15]);
  f4 v1 = bez(v, r0, r1, r2, r3);
  r0 = bez(u, P[0], P[1], P[2], P[3]); r1 = bez(u, P[4], P[5], P[6], P[7]);
  r2 = bez(u, P[8], P[9], P[10], P[11]); r3 = bez(u, P[12], P[13], P[14], P[15]);
  f4 v2 = dbez(v, r0, r1, r2, r3);
  f4 c;
  c.x = v1.y * v2.z - v1.z * v2.y;
  c.y = v1.z * v2.x - v1.x * v2.z;
  c.z = v1.x * v2.y - v1.y * v2.x;
  float mag = sqrtf(c.x * c.x + c.y * c.y + c.z * c.z);
  c.x /= mag; c.y /= mag; c.z /= mag;
  c.w = 1.0f;
  return c;
}

/* a micropolygon as Shade consumes it: screen x, y, z and normal of 4 corners */
typedef struct { float sx[4], sy[4], sz[4], nx[4], ny[4], nz[4]; } upoly;

static void dice_corner(const patch* p, const float* vp, int W, int H, float u, float v, upoly* q, int c)
{
  f4 pt = patch_eval(p->cp, u, v);
  f4 ss = matmul4(vp, pt);
  f4 n = norm_eval(p->cp, u, v);
  float onebyw = 1.0f / ss.w;
  q->sx[c] = (ss.x * onebyw + 1.0f) * (float)W * 0.5f;
  q->sy[c] = (ss.y * onebyw + 1.0f) * (float)H * 0.5f;
  q->sz[c] = (ss.z * onebyw);
  q->nx[c] = n.x; q->ny[c] = n.y; q->nz[c] = n.z;
}

/* ---------------------------------------------------------------- shade */
static double std_min_d(double a, double b) { return (b < a) ? b : a; }
static double std_max_d(double a, double b) { return (a < b) ? b : a; }

static void shade_bins(const upoly* q, int W, int H, int* bx1, int* bx2, int* by1, int* by2)
{
  /* computeBoundingBox (dice.pikostage:18-22, corners 0..2, double fmin/fmax)
   * then assignToBB (:24-43) with 64-pixel bins */
  float lox = floorf((float)std_min_d(q->sx[0], std_min_d(q->sx[1], q->sx[2])));
  float loy = floorf((float)std_min_d(q->sy[0], std_min_d(q->sy[1], q->sy[2])));
  float hix = ceilf((float)std_max_d(q->sx[0], std_max_d(q->sx[1], q->sx[2])));
  float hiy = ceilf((float)std_max_d(q->sy[0], std_max_d(q->sy[1], q->sy[2])));
  int nBx = W / 64, nBy = H / 64;
  int a = cvt_i32(floorf(lox / 64.0f)), b = cvt_i32(floorf(hix / 64.0f));
  int c = cvt_i32(floorf(loy / 64.0f)), d = cvt_i32(floorf(hiy / 64.0f));
  if (a < 0) a = 0;
  if (c < 0) c = 0;
  if (b >= nBx) b = nBx - 1;
  if (d >= nBy) d = nBy - 1;
  *bx1 = a; *bx2 = b; *by1 = c; *by2 = d;
}

static float phong_channel(float nx, float ny, float nz, int ch)
{
  /* phongShadeReyes: negated normal; computeLighting(normal, matcol, lightvec)
   * so the "light" operand of the dot product is matcol and the scale is lightvec */
  const float mat[3] = {0.10f, 0.35f, 0.85f};
  const float lv[3] = {0.1773f, 0.5773f, 0.973f};
  nx = -nx; ny = -ny; nz = -nz;
  float d = nx * mat[0] + ny * mat[1] + nz * mat[2];
  d = d < 0.0f ? 0.0f : d;
  float o = 0.2f + d * lv[ch];
  return o > 1.0f ? 1.0f : (o < 0.0f ? 0.0f : o);
}

typedef struct {
  int W, H;
  int spp;           /* samples per pixel: 1 (the reference) or 4 */
  uint32_t seed;     /* jitter seed (spp 4) */
  int phong;         /* 0: the reference's corner-lit colour, 1: Phong (interpolated normal) */
  uint32_t* fb;      /* per sample colour, W*H*spp */
  int32_t* zb;       /* per sample depth bits, W*H*spp */
  long long covered, passed, hangs;
} shade_ctx;

/* Phong variant (no reference counterpart): the corner normals are
 * interpolated to the micropolygon's centre (summed in corner order and
 * renormalised) and lit once with the reference's lighting, instead of lighting
 * the corners and averaging the colours. */
static void phong_colour(const upoly* q, float* col)
{
  float nx = q->nx[0] + q->nx[1], ny = q->ny[0] + q->ny[1], nz = q->nz[0] + q->nz[1];
  nx = nx + q->nx[2]; ny = ny + q->ny[2]; nz = nz + q->nz[2];
  nx = nx + q->nx[3]; ny = ny + q->ny[3]; nz = nz + q->nz[3];
  const float mag = sqrtf(nx * nx + ny * ny + nz * nz);
  nx = nx / mag; ny = ny / mag; nz = nz / mag;
  for (int ch = 0; ch < 3; ++ch) col[ch] = phong_channel(nx, ny, nz, ch);
}

static void shade_upoly(shade_ctx* sc, const upoly* q, int bin)
{
  int nBx = sc->W / 64;
  float z = ((q->sz[0] + q->sz[1] + q->sz[2] + q->sz[3])) * 0.25f;
  float col[3];
  if (sc->phong) {
    phong_colour(q, col);
  } else {
    for (int ch = 0; ch < 3; ++ch) {
      float c = phong_channel(q->nx[0], q->ny[0], q->nz[0], ch) + phong_channel(q->nx[1], q->ny[1], q->nz[1], ch);
      c = c + phong_channel(q->nx[2], q->ny[2], q->nz[2], ch);
      c = c + phong_channel(q->nx[3], q->ny[3], q->nz[3], ch);
      c = std_minf(c, 4.0f);
      col[ch] = c * 0.25f;
    }
  }
  float bminx = std_minf(std_minf(q->sx[0], q->sx[1]), std_minf(q->sx[2], q->sx[3]));
  float bminy = std_minf(std_minf(q->sy[0], q->sy[1]), std_minf(q->sy[2], q->sy[3]));
  float bmaxx = std_maxf(std_maxf(q->sx[0], q->sx[1]), std_maxf(q->sx[2], q->sx[3]));
  float bmaxy = std_maxf(std_maxf(q->sy[0], q->sy[1]), std_maxf(q->sy[2], q->sy[3]));
  bminx = floorf(bminx); bminy = floorf(bminy); bmaxx = ceilf(bmaxx); bmaxy = ceilf(bmaxy);
  int bbx = (int)((unsigned)bin % (unsigned)nBx) * 64, bby = (int)((unsigned)bin / (unsigned)nBx) * 64;
  int bex = bbx + 64, bey = bby + 64;
  /* intersectBBi macro: float/int ternaries, result truncated to int */
  int pbx = cvt_i32((bminx > (float)bbx) ? bminx : (float)bbx);
  int pby = cvt_i32((bminy > (float)bby) ? bminy : (float)bby);
  int pex = cvt_i32((bmaxx < (float)bex) ? bmaxx : (float)bex);
  int pey = cvt_i32((bmaxy < (float)bey) ? bmaxy : (float)bey);
  const float *X = q->sx, *Y = q->sy;
  for (int my = pby; my < pey; ++my) {
    for (int mx = pbx; mx < pex; ++mx) {
     for (int smp = 0; smp < sc->spp; ++smp) {
      float px, py;
      sample_pos(sc->spp, sc->seed, mx, my, smp, &px, &py);
      int r1 = 1, r2 = 1;
      if (((py - Y[0]) * (X[1] - X[0]) - (px - X[0]) * (Y[1] - Y[0])) <= 0.0f) r1 = 0;
      if (((py - Y[1]) * (X[2] - X[1]) - (px - X[1]) * (Y[2] - Y[1])) <= 0.0f) r1 = 0;
      if (((py - Y[2]) * (X[3] - X[2]) - (px - X[2]) * (Y[3] - Y[2])) <= 0.0f) r1 = 0;
      if (((py - Y[3]) * (X[0] - X[3]) - (px - X[3]) * (Y[0] - Y[3])) <= 0.0f) r1 = 0;
      if (((py - Y[0]) * (X[3] - X[0]) - (px - X[0]) * (Y[3] - Y[0])) <= 0.0f) r2 = 0;
      if (((py - Y[3]) * (X[2] - X[3]) - (px - X[3]) * (Y[2] - Y[3])) <= 0.0f) r2 = 0;
      if (((py - Y[2]) * (X[1] - X[2]) - (px - X[2]) * (Y[1] - Y[2])) <= 0.0f) r2 = 0;
      if (((py - Y[1]) * (X[0] - X[1]) - (px - X[1]) * (Y[0] - Y[1])) <= 0.0f) r2 = 0;
      if (!(r1 + r2)) continue;
      int pix = (my * sc->W + mx) * sc->spp + smp;
      sc->covered++;
      /* while (remoteZ > z) remoteZ = atomicMin(bits, zbits); bounded here: a
       * third round can only repeat the second (negative depths never settle) */
      float remote = bits2f(sc->zb[pix]);
      int32_t zi = f2bits(z);
      int rounds = 0;
      while (remote > z) {
        int32_t old = sc->zb[pix];
        sc->zb[pix] = old < zi ? old : zi;
        remote = bits2f(old);
        if (++rounds > 2) { sc->hangs++; break; }
      }
      if (bits2f(sc->zb[pix]) == z) {
        sc->fb[pix] = (255u << 24) | (cvt_u32(col[2] * 255.0f) << 16) | (cvt_u32(col[1] * 255.0f) << 8) |
                      cvt_u32(col[0] * 255.0f);
        sc->passed++;
      }
     }
    }
  }
}

/* cps: P*16 float4 control points; stats: [0] leaves, [1] micropolygons,
 * [2] (micropolygon, bin) pairs, [3] covered samples, [4] passed samples,
 * [5] depth loops that would never end in the reference (negative depths),
 * [6] split levels run.  leaf_out (optional, 4 ints per leaf, cap leaves):
 * id, numSplits, nu, nv in Dice processing order. */
static int reyes_frame(int W, int H, int P, const float* cps, const float* vp,
                       float thr, int max_splits, int grid, int spp, uint32_t seed, int phong,
                       uint32_t* fb, float* depth, long long* stats,
                       int* leaf_out, long long leaf_cap);

int oracle_reyes_frame(int W, int H, int P, const float* cps, const float* vp,
                       float thr, int max_splits, int grid,
                       uint32_t* fb, float* depth, long long* stats,
                       int* leaf_out, long long leaf_cap)
{
  return reyes_frame(W, H, P, cps, vp, thr, max_splits, grid, 1, 0u, 0, fb, depth, stats, leaf_out, leaf_cap);
}

/* The multi-sample / Phong variant (no reference counterpart): spp samples per
 * pixel (1 or 4) at sample_pos(), each with the reference's coverage test and
 * depth loop; phong = 1 lights the interpolated normal (phong_colour).  The
 * pixel takes the rounded mean of its samples' colours per channel and the
 * depth of its nearest sample (the first such sample on ties).  stats[3] and
 * stats[4] count samples. */
int oracle_reyes_frame_ms(int W, int H, int P, const float* cps, const float* vp,
                          float thr, int max_splits, int grid, int spp, uint32_t seed, int phong,
                          uint32_t* fb, float* depth, long long* stats)
{
  if (spp != 1 && spp != 4) return -1;
  return reyes_frame(W, H, P, cps, vp, thr, max_splits, grid, spp, seed, phong, fb, depth, stats, NULL, 0);
}

static int reyes_frame(int W, int H, int P, const float* cps, const float* vp,
                       float thr, int max_splits, int grid, int spp, uint32_t seed, int phong,
                       uint32_t* fb, float* depth, long long* stats,
                       int* leaf_out, long long leaf_cap)
{
  size_t cap = (size_t)(P > 0 ? P : 1), n = 0;
  patch* level = (patch*)malloc(sizeof(patch) * cap);
  for (int i = 0; i < P; ++i) {
    memcpy(level[i].cp, cps + (size_t)i * 64, 64 * sizeof(float));
    level[i].numSplits = 0; level[i].id = i; level[i].nu = level[i].nv = 0;
  }
  n = (size_t)P;
  size_t lcap = 1024, nleaf = 0;
  patch* leaves = (patch*)malloc(sizeof(patch) * lcap);
  long long levels = 0;
  while (n > 0) {
    levels++;
    size_t ncap = 2 * n, nn = 0;
    patch* next = (patch*)malloc(sizeof(patch) * ncap);
    for (size_t i = 0; i < n; ++i) {
      patch c1, c2;
      if (split_process(&level[i], vp, W, H, thr, max_splits, grid, &c1, &c2)) {
        next[nn++] = c1;
        next[nn++] = c2;
      } else {
        if (nleaf == lcap) { lcap *= 2; leaves = (patch*)realloc(leaves, sizeof(patch) * lcap); }
        leaves[nleaf++] = level[i];
      }
    }
    free(level);
    level = next;
    n = nn;
  }
  free(level);

  /* Dice bins: (id / 128) % nDice, processed in bin order, FIFO inside a bin */
  int nDice = (W / 64) * (H / 64);
  if (nDice < 1) nDice = 1;
  size_t* order = (size_t*)malloc(sizeof(size_t) * (nleaf ? nleaf : 1));
  size_t k = 0;
  for (int b = 0; b < nDice; ++b)
    for (size_t i = 0; i < nleaf; ++i)
      if ((leaves[i].id / 128) % nDice == b) order[k++] = i;

  /* generate micropolygons in Dice order and their Shade bins */
  int nBx = W / 64, nBy = H / 64, nShade = nBx * nBy;
  size_t ucap = 1024, nu_ = 0;
  upoly* ups = (upoly*)malloc(sizeof(upoly) * ucap);
  size_t pcap = 1024, np = 0;
  int* pbin = (int*)malloc(sizeof(int) * pcap);
  size_t* pup = (size_t*)malloc(sizeof(size_t) * pcap);
  for (size_t o = 0; o < k; ++o) {
    const patch* p = &leaves[order[o]];
    if (leaf_out && (long long)o < leaf_cap) {
      leaf_out[4 * o + 0] = p->id; leaf_out[4 * o + 1] = p->numSplits;
      leaf_out[4 * o + 2] = p->nu; leaf_out[4 * o + 3] = p->nv;
    }
    float du = 1.0f / ((float)p->nu), dv = 1.0f / ((float)p->nv);
    for (int kk = 0; kk <= p->nu; ++kk)
      for (int j = 0; j <= p->nv; ++j) {
        float u = (float)kk * du, v = (float)j * dv;
        upoly q;
        dice_corner(p, vp, W, H, u, v, &q, 0);
        dice_corner(p, vp, W, H, u + du, v, &q, 1);
        dice_corner(p, vp, W, H, u + du, v + dv, &q, 2);
        dice_corner(p, vp, W, H, u, v + dv, &q, 3);
        if (nu_ == ucap) { ucap *= 2; ups = (upoly*)realloc(ups, sizeof(upoly) * ucap); }
        ups[nu_] = q;
        int a, b, c, d;
        shade_bins(&q, W, H, &a, &b, &c, &d);
        for (int by = c; by <= d; ++by)
          for (int bx = a; bx <= b; ++bx) {
            if (np == pcap) {
              pcap *= 2;
              pbin = (int*)realloc(pbin, sizeof(int) * pcap);
              pup = (size_t*)realloc(pup, sizeof(size_t) * pcap);
            }
            pbin[np] = by * nBx + bx; pup[np] = nu_; np++;
          }
        nu_++;
      }
  }
  /* stable counting sort by shade bin (FIFO inside each bin) */
  size_t* start = (size_t*)calloc((size_t)nShade + 1, sizeof(size_t));
  for (size_t i = 0; i < np; ++i) start[pbin[i] + 1]++;
  for (int b = 0; b < nShade; ++b) start[b + 1] += start[b];
  size_t* cur = (size_t*)malloc(sizeof(size_t) * (nShade ? nShade : 1));
  for (int b = 0; b < nShade; ++b) cur[b] = start[b];
  size_t* lst = (size_t*)malloc(sizeof(size_t) * (np ? np : 1));
  for (size_t i = 0; i < np; ++i) lst[cur[pbin[i]]++] = pup[i];

  shade_ctx sc;
  memset(&sc, 0, sizeof(sc));
  sc.W = W; sc.H = H; sc.spp = spp; sc.seed = seed; sc.phong = phong;
  const size_t nsamp = (size_t)W * H * (size_t)spp;
  sc.fb = spp == 1 ? fb : (uint32_t*)malloc(sizeof(uint32_t) * nsamp);
  sc.zb = (int32_t*)malloc(sizeof(int32_t) * nsamp);
  for (size_t i = 0; i < nsamp; ++i) { sc.fb[i] = 0xff663313u; sc.zb[i] = f2bits(1.0f); }
  for (int b = 0; b < nShade; ++b)
    for (size_t i = start[b]; i < start[b + 1]; ++i) shade_upoly(&sc, &ups[lst[i]], b);
  if (spp == 1) {
    memcpy(depth, sc.zb, sizeof(float) * (size_t)W * H);
  } else {
    for (size_t pix = 0; pix < (size_t)W * H; ++pix) {
      const uint32_t* c = sc.fb + pix * spp;
      const int32_t* z = sc.zb + pix * spp;
      uint32_t out = 0xff000000u;
      for (int ch = 0; ch < 3; ++ch) {
        uint32_t sum = 0;
        for (int k = 0; k < spp; ++k) sum += (c[k] >> (8 * ch)) & 255u;
        out |= ((sum + (uint32_t)spp / 2u) / (uint32_t)spp) << (8 * ch);
      }
      int best = 0;
      for (int k = 1; k < spp; ++k)
        if (zorder_u(bits2f(z[k])) < zorder_u(bits2f(z[best]))) best = k;
      fb[pix] = out;
      memcpy(&depth[pix], &z[best], 4);
    }
    free(sc.fb);
  }
  if (stats) {
    stats[0] = (long long)nleaf; stats[1] = (long long)nu_; stats[2] = (long long)np;
    stats[3] = sc.covered; stats[4] = sc.passed; stats[5] = sc.hangs; stats[6] = levels;
  }
  free(leaves); free(order); free(ups); free(pbin); free(pup); free(start); free(cur); free(lst); free(sc.zb);
  return 0;
}
