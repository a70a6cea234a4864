/* TEST INFRASTRUCTURE — the oracle's CPU restatement of the binned raster path.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * as the checker; the product path never links or calls it.
 *
 * It restates, in plain sequential C, what the reference's RasterPipe computes
 * when its CPU backend runs with one thread:
 *   R1 host pre-transform + Gouraud lighting
 *        pikoc/samples/rasterPipelineFixPt/main.cpp:299-400
 *   R2 VertexShaderStage::assignBin  vertexShader.pikostage:25-29
 *   R3 VertexShaderStage::process    vertexShader.pikostage:36-109, rasterMacros.h:23-75
 *   R4 RasterStage::assignBin        raster.pikostage:40-117, rasterMacros.h:152-170
 *   R5 bin order (1 CPU thread)      piko/stage.h:339-343, internal/datatypes.h:88-93,156-172,
 *                                    pikoc/src/Backend/CPUBackend.cpp:428-520
 *   R6 coverage mask                 raster.pikostage:124-242
 *   R7 fragments, depth, colour      raster.pikostage:244-320, piko/math.h:279-289,323-330
 *   R8 PikoScreen::assignBin         piko/stage.h:57-61 (clear colour :83-85)
 * plus one extension with no reference counterpart (the textured variant: the
 * Gouraud colour times a nearest, wrapped texel at the screen-space
 * interpolated UV), which is pinned by this restatement alone.
 */
#include <stdlib.h>
#include "oracle_common.h"

#define VS_BIN 32
#define RB_LG2 3
#define RB (1 << RB_LG2)
#define GUARD (225 << 4)
#define CLEAR_COLOR 0xff663313u

typedef struct { float x, y, z; } f3;

/* ---------------------------------------------------------------- R1 */
static f3 vtransform3(const float* m, f3 v, float* w)
{
  /* basicTypes/../piko/matrices.h:112-117, left-to-right sums */
  f3 o;
  o.x = v.x * m[0] + v.y * m[4] + v.z * m[8] + m[12];
  o.y = v.x * m[1] + v.y * m[5] + v.z * m[9] + m[13];
  o.z = v.x * m[2] + v.y * m[6] + v.z * m[10] + m[14];
  *w  = v.x * m[3] + v.y * m[7] + v.z * m[11] + m[15];
  return o;
}

static f3 host_normalize(f3 v)
{
  /* HOST::normalize, util/host_math.h:51-59: divide by the magnitude */
  float mag = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
  v.x /= mag; v.y /= mag; v.z /= mag;
  return v;
}

static f3 normalize_inplace(f3 v)
{
  /* normalizeInplace, piko/cvec.h:139-142: multiply by the reciprocal */
  float m = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
  if (m != 0.0f) { float r = 1.0f / m; v.x = v.x * r; v.y = v.y * r; v.z = v.z * r; }
  return v;
}

static float sat1(float v) { return v > 1.0f ? 1.0f : (v < 0.0f ? 0.0f : v); }

static uint32_t light_abgr(f3 n, f3 l, f3 mat)
{
  /* computeLightingHost + toABGRHost, main.cpp:317-334 */
  float d = n.x * l.x + n.y * l.y + n.z * l.z;
  d = d < 0.0f ? 0.0f : d;
  float r = sat1(d * mat.x + 0.15f);
  float g = sat1(d * mat.y + 0.15f);
  float b = sat1(d * mat.z + 0.30f);
  return 0xff000000u | (cvt_u32(b * 255.0f) << 16) | (cvt_u32(g * 255.0f) << 8) | cvt_u32(r * 255.0f);
}

/* pos/nrm/col: float4 [3][N] (col NULL: the fixed material colour (0.9, 0.9,
 * 0.6) of main.cpp:380 for every vertex); light_mode 0: light3 is the light
 * vector for all vertices; 1: light vector = normalize(eye - position)
 * (main.cpp:372-378).
 * Writes the pre-transformed raster_wtri payload: xyz[9N], icol[3N]. */
int oracle_r1_setup(int N, int W, int H, const float* pos, const float* nrm, const float* col,
                    const float* vp, int light_mode, const float* light3, const float* eye3,
                    float* xyz, uint32_t* icol)
{
  float halfW = 0.5f * (float)W, halfH = 0.5f * (float)H;
  for (int t = 0; t < N; ++t) {
    for (int k = 0; k < 3; ++k) {
      const float* p4 = pos + ((size_t)k * N + t) * 4;
      const float* n4 = nrm + ((size_t)k * N + t) * 4;
      static const float matcol[4] = {0.9000f, 0.9000f, 0.6000f, 1.0f};
      const float* c4 = col ? col + ((size_t)k * N + t) * 4 : matcol;
      f3 wp = {p4[0], p4[1], p4[2]};
      f3 n = host_normalize((f3){n4[0], n4[1], n4[2]});
      f3 l;
      if (light_mode == 1) {
        l.x = eye3[0] - wp.x; l.y = eye3[1] - wp.y; l.z = eye3[2] - wp.z;
        l = normalize_inplace(l);
      } else {
        l.x = light3[0]; l.y = light3[1]; l.z = light3[2];
      }
      /* inPlaceTransform, main.cpp:299-308 */
      float w;
      f3 tv = vtransform3(vp, wp, &w);
      float onebyw = 1.0f / w;
      xyz[9 * t + 3 * k + 0] = (tv.x * onebyw + 1.0f) * halfW;
      xyz[9 * t + 3 * k + 1] = (tv.y * onebyw + 1.0f) * halfH;
      xyz[9 * t + 3 * k + 2] = (tv.z * onebyw);
      icol[3 * t + k] = light_abgr(n, l, (f3){c4[0], c4[1], c4[2]});
    }
  }
  return 0;
}

/* The vertex stage's own transform when the pipe is built without
 * VTX_PRETRANSFORM (vertexShader.pikostage:56-80): vtxTransform
 * (rasterMacros.h:14-21) = matmultfloat4 of the world position
 * (piko/math.h:375-383, the same left-to-right sums as vtransform3), one over w
 * by rcp_approx (1.0f / w on the CPU, piko/math.h:279), then the viewport with
 * halfW = (float)W * 0.5f.  xyz_world: [N][9] world positions; out: the
 * screen x, y and depth of the 3 vertices, as the pre-transformed payload. */
int oracle_vs_world(int N, int W, int H, const float* xyz_world, const float* vp, float* xyz)
{
  const float halfW = (float)W * 0.5f, halfH = (float)H * 0.5f;
  for (int t = 0; t < N; ++t) {
    for (int k = 0; k < 3; ++k) {
      const float* q = xyz_world + 9 * (size_t)t + 3 * k;
      f3 wp = {q[0], q[1], q[2]};
      float w;
      f3 tv = vtransform3(vp, wp, &w);
      float onebyw = 1.0f / w;
      xyz[9 * t + 3 * k + 0] = (tv.x * onebyw + 1.0f) * halfW;
      xyz[9 * t + 3 * k + 1] = (tv.y * onebyw + 1.0f) * halfH;
      xyz[9 * t + 3 * k + 2] = (tv.z * onebyw);
    }
  }
  return 0;
}

/* ---------------------------------------------------------------- R3 / R4 */
typedef struct {
  int32_t x[3], y[3];
  float z[3];
  uint32_t c[3];
} stri;

/* quantise + cull (vertexShader.pikostage:46-67, rasterMacros.h:23-75);
 * returns 1 when the triangle is emitted to the raster stage */
static int vs_process(const float* xyz, const uint32_t* icol, int t, int W, int H, stri* s)
{
  for (int k = 0; k < 3; ++k) {
    s->x[k] = cvt_i32(xyz[9 * t + 3 * k + 0] * 16.0f);
    s->y[k] = cvt_i32(xyz[9 * t + 3 * k + 1] * 16.0f);
    s->z[k] = xyz[9 * t + 3 * k + 2];
    s->c[k] = icol[3 * t + k];
  }
  /* isFrontFacingFixPt */
  int32_t cr = wsub(wmul(wsub(s->y[2], s->y[0]), wsub(s->x[1], s->x[0])),
                    wmul(wsub(s->x[2], s->x[0]), wsub(s->y[1], s->y[0])));
  if (!(cr > 0)) return 0;
  /* isInsideFrustumFixPt with W*16, H*16 passed as float -> int */
  int32_t Wf = cvt_i32((float)W * 16.0f), Hf = cvt_i32((float)H * 16.0f);
  for (int k = 0; k < 3; ++k) {
    if (s->x[k] < -GUARD || s->x[k] >= wadd(Wf, GUARD)) return 0;
    if (s->y[k] < -GUARD || s->y[k] >= wadd(Hf, GUARD)) return 0;
  }
  /* isBBBetweenSamples: only the Y axis is tested (`bCullYaxis || bCullYaxis`) */
  int32_t loy = imin_(imin_(s->y[0], s->y[1]), s->y[2]);
  int32_t hiy = imax_(imax_(s->y[0], s->y[1]), s->y[2]);
  if ((wsub(loy, 8) >> 4) == (wsub(hiy, 8) >> 4)) return 0;
  return 1;
}

static void pixel_bbox(const stri* s, int32_t* lox, int32_t* loy, int32_t* hix, int32_t* hiy)
{
  /* computePixelBoundingBoxFixPt: round to 256 (16 pixels) in 28.4 */
  *lox = imin_(imin_(s->x[0], s->x[1]), s->x[2]) & (int32_t)0xffffff00;
  *loy = imin_(imin_(s->y[0], s->y[1]), s->y[2]) & (int32_t)0xffffff00;
  *hix = wadd(imax_(imax_(s->x[0], s->x[1]), s->x[2]), 0xff) & (int32_t)0xffffff00;
  *hiy = wadd(imax_(imax_(s->y[0], s->y[1]), s->y[2]), 0xff) & (int32_t)0xffffff00;
}

/* Calls emit(bin) for every bin RasterStage::assignBin assigns the triangle to. */
typedef void (*bin_cb)(void* ctx, int bin);
static void raster_assign(const stri* s, int nBx, int nBy, bin_cb cb, void* ctx)
{
  int32_t lox, loy, hix, hiy;
  pixel_bbox(s, &lox, &loy, &hix, &hiy);
  const int bits = 4 + RB_LG2;
  int bx1 = imax_(0, lox >> bits), bx2 = imin_(hix >> bits, nBx - 1);
  int by1 = imax_(0, loy >> bits), by2 = imin_(hiy >> bits, nBy - 1);
  int32_t dx[3], dy[3], stx[3], sty[3], rs[3];
  for (int i = 0; i < 3; ++i) {
    int j = (i + 1) % 3;
    dx[i] = wsub(s->x[j], s->x[i]);
    dy[i] = wsub(s->y[j], s->y[i]);
    stx[i] = -wshl(dy[i], bits);
    sty[i] = wshl(dx[i], bits);
  }
  int32_t startx = wshl(bx1, bits), starty = wshl(by1, bits);
  for (int i = 0; i < 3; ++i) {
    int32_t off = (dy[i] < 0 ? stx[i] : 0);
    off = wadd(off, dx[i] >= 0 ? sty[i] : 0);
    rs[i] = wsub(wadd(off, wmul(wsub(starty, s->y[i]), dx[i])), wmul(wsub(startx, s->x[i]), dy[i]));
  }
  for (int by = by1; by <= by2; ++by) {
    int32_t t0 = rs[0], t1 = rs[1], t2 = rs[2];
    for (int bx = bx1; bx <= bx2; ++bx) {
      if ((t0 | t1 | t2) >= 0) cb(ctx, by * nBx + bx);
      t0 = wadd(t0, stx[0]); t1 = wadd(t1, stx[1]); t2 = wadd(t2, stx[2]);
    }
    rs[0] = wadd(rs[0], sty[0]); rs[1] = wadd(rs[1], sty[1]); rs[2] = wadd(rs[2], sty[2]);
  }
}

/* ---------------------------------------------------------------- R6 */
static uint64_t coverage_mask(const stri* s, int bin, int nBx)
{
  int32_t lox, loy, hix, hiy;
  pixel_bbox(s, &lox, &loy, &hix, &hiy);
  int32_t bbx = (bin % nBx) * (RB << 4), bby = (bin / nBx) * (RB << 4);
  int32_t bex = bbx + (RB << 4), bey = bby + (RB << 4);
  int32_t pbx = imax_(lox, bbx), pby = imax_(loy, bby);
  int32_t pex = imin_(hix, bex), pey = imin_(hiy, bey);
  int32_t dx[3], dy[3], stx[3], sty[3], rs[3];
  for (int i = 0; i < 3; ++i) {
    int j = (i + 1) % 3;
    dx[i] = wsub(s->x[j], s->x[i]);
    dy[i] = wsub(s->y[j], s->y[i]);
    stx[i] = -wshl(dy[i], 4);
    sty[i] = wshl(dx[i], 4);
    rs[i] = wsub(wmul(wsub(wadd(pby, 8), s->y[i]), dx[i]), wmul(wsub(wadd(pbx, 8), s->x[i]), dy[i]));
  }
  int32_t ta = 0;
  for (int i = 0; i < 3; ++i) {
    int32_t off = (dy[i] >= 0 ? stx[i] : 0);
    off = wadd(off, dx[i] < 0 ? sty[i] : 0);
    ta |= wadd(rs[i], wshl(off, RB_LG2));
  }
  if ((ta & (int32_t)0x80000000) == 0) return ~0ull;
  uint64_t mask = 0;
  for (int32_t y = pby; y < pey; y += 16) {
    int32_t e0 = rs[0], e1 = rs[1], e2 = rs[2];
    for (int32_t x = pbx; x < pex; x += 16) {
      if ((e0 | e1 | e2) >= 0) {
        int bit = ((x - bbx) + ((y - bby) << 3)) >> 4;
        mask |= 1ull << bit;
      }
      e0 = wadd(e0, stx[0]); e1 = wadd(e1, stx[1]); e2 = wadd(e2, stx[2]);
    }
    rs[0] = wadd(rs[0], sty[0]); rs[1] = wadd(rs[1], sty[1]); rs[2] = wadd(rs[2], sty[2]);
  }
  return mask;
}

/* ---------------------------------------------------------------- R7 / R8 */
typedef struct {
  int W, H, nBx;
  uint32_t* fb;
  int32_t* zb;
  const float* uv;        /* NULL, or 6 floats per triangle (u0,v0,u1,v1,u2,v2) */
  const uint8_t* tex;     /* RGBA8 [TH][TW] */
  int TW, TH;
  long long covered, passed;
} frag_ctx;

static float interp(float f0mf2, float f1mf2, float f2, float a, float b)
{
  /* interpolate_alphabeta, raster.pikostage:28-32: f2 + a*f0mf2 + b*f1mf2 */
  return f2 + a * f0mf2 + b * f1mf2;
}

static void shade_bin(frag_ctx* fc, const stri* s, int tri, int bin, uint64_t mask)
{
  if (!mask) return;
  int32_t bbx = (bin % fc->nBx) * (RB << 4), bby = (bin / fc->nBx) * (RB << 4);
  int32_t dx1 = wsub(s->x[2], s->x[1]), dy1 = wsub(s->y[2], s->y[1]);
  int32_t dx2 = wsub(s->x[0], s->x[2]), dy2 = wsub(s->y[0], s->y[2]);
  int32_t x1mx0 = wsub(s->x[1], s->x[0]), y1my0 = wsub(s->y[1], s->y[0]);
  int32_t barydenom = wadd(wmul(-dy2, x1mx0), wmul(dx2, y1my0));
  float onebybary = 1.0f / (float)barydenom;
  int32_t rs1 = wsub(wmul(wsub(wadd(bby, 8), s->y[1]), dx1), wmul(wsub(wadd(bbx, 8), s->x[1]), dy1));
  int32_t rs2 = wsub(wmul(wsub(wadd(bby, 8), s->y[2]), dx2), wmul(wsub(wadd(bbx, 8), s->x[2]), dy2));
  int32_t st1x = -wshl(dy1, 4), st1y = wshl(dx1, 4), st2x = -wshl(dy2, 4), st2y = wshl(dx2, 4);
  float z0mz2 = s->z[0] - s->z[2], z1mz2 = s->z[1] - s->z[2];
  float vc[3][3];
  for (int k = 0; k < 3; ++k) {
    vc[k][0] = (float)((s->c[k] >> 0) & 255) / 255.0f;
    vc[k][1] = (float)((s->c[k] >> 8) & 255) / 255.0f;
    vc[k][2] = (float)((s->c[k] >> 16) & 255) / 255.0f;
  }
  float d0[3], d1[3];
  for (int c = 0; c < 3; ++c) { d0[c] = vc[0][c] - vc[2][c]; d1[c] = vc[1][c] - vc[2][c]; }
  float u0mu2 = 0, u1mu2 = 0, v0mv2 = 0, v1mv2 = 0, u2 = 0, v2 = 0;
  if (fc->uv) {
    const float* q = fc->uv + 6 * (size_t)tri;
    u0mu2 = q[0] - q[4]; u1mu2 = q[2] - q[4]; u2 = q[4];
    v0mv2 = q[1] - q[5]; v1mv2 = q[3] - q[5]; v2 = q[5];
  }
  uint64_t m = mask;
  while (m) {
    int low = __builtin_ctzll(m);
    int x = low & 7, y = low >> 3;
    int32_t e1 = wadd(wadd(rs1, wmul(x, st1x)), wmul(y, st1y));
    int32_t e2 = wadd(wadd(rs2, wmul(x, st2x)), wmul(y, st2y));
    int32_t X = wadd(x << 4, bbx), Y = wadd(y << 4, bby);
    float alpha = (float)e1 * onebybary;
    float beta = (float)e2 * onebybary;
    float z = interp(z0mz2, z1mz2, s->z[2], alpha, beta);
    int32_t zi = f2bits(z);
    int32_t pix = wadd(wmul(Y, fc->W), X) >> 4;
    fc->covered++;
    /* do { remote = atomicMin(zbuf, zi) } while (remote > zi); pass iff remote >= zi */
    int32_t remote = fc->zb[pix];
    if (remote > zi) { fc->zb[pix] = zi; remote = zi; }
    if (remote >= zi) {
      float cr = interp(d0[0], d1[0], vc[2][0], alpha, beta);
      float cg = interp(d0[1], d1[1], vc[2][1], alpha, beta);
      float cb = interp(d0[2], d1[2], vc[2][2], alpha, beta);
      if (fc->uv) {
        float u = interp(u0mu2, u1mu2, u2, alpha, beta);
        float v = interp(v0mv2, v1mv2, v2, alpha, beta);
        int tx = cvt_i32(floorf(u * (float)fc->TW)) & (fc->TW - 1);
        int ty = cvt_i32(floorf(v * (float)fc->TH)) & (fc->TH - 1);
        const uint8_t* tp = fc->tex + ((size_t)ty * fc->TW + tx) * 4;
        cr = cr * ((float)tp[0] / 255.0f);
        cg = cg * ((float)tp[1] / 255.0f);
        cb = cb * ((float)tp[2] / 255.0f);
      }
      uint32_t color = 0xff000000u | (cvt_u32(cb * 255.0f) << 16) | (cvt_u32(cg * 255.0f) << 8) | cvt_u32(cr * 255.0f);
      uint32_t px = (uint32_t)(X >> 4), py = (uint32_t)(Y >> 4);
      fc->fb[(int32_t)(py * (uint32_t)fc->W + px)] = color;
      fc->passed++;
    }
    m &= m - 1;
  }
}

/* ---------------------------------------------------------------- frame */
typedef struct { int* bins; int* tris; size_t n, cap; } pairs;
static void pairs_push(void* ctx, int bin)
{
  pairs* p = (pairs*)ctx;
  if (p->n == p->cap) {
    p->cap = p->cap ? 2 * p->cap : 1024;
    p->bins = (int*)realloc(p->bins, p->cap * sizeof(int));
    p->tris = (int*)realloc(p->tris, p->cap * sizeof(int));
  }
  p->bins[p->n] = bin;
  p->tris[p->n] = -1;
  p->n++;
}

/* The submission order of the one-thread CPU backend: VS bins in index order,
 * and inside VS bin b the ids with (id/512) % nVS == b ascending (R5).
 * Fills order[N]; returns nothing. */
void oracle_submission_order(int N, int W, int H, int* order)
{
  int nVS = (W / VS_BIN) * (H / VS_BIN);
  if (nVS < 1) nVS = 1;
  int k = 0;
  for (int b = 0; b < nVS; ++b)
    for (int c = b; (long long)c * 512 < N; c += nVS)
      for (int id = c * 512; id < N && id < (c + 1) * 512; ++id) order[k++] = id;
}

/* stats: [0] triangles kept by the vertex stage, [1] (triangle, bin) pairs,
 * [2] covered samples, [3] samples that passed the depth test (emits). */
int oracle_raster_frame(int W, int H, int N, const float* xyz, const uint32_t* icol,
                        const float* uv, const uint8_t* tex, int TW, int TH,
                        uint32_t* fb, float* depth, long long* stats)
{
  int nBx = W / RB, nBy = H / RB;
  int* order = (int*)malloc(sizeof(int) * (N > 0 ? N : 1));
  oracle_submission_order(N, W, H, order);
  stri* st = (stri*)malloc(sizeof(stri) * (N > 0 ? N : 1));
  pairs pr = {0};
  long long kept = 0;
  for (int k = 0; k < N; ++k) {
    int t = order[k];
    if (!vs_process(xyz, icol, t, W, H, &st[t])) continue;
    kept++;
    size_t before = pr.n;
    raster_assign(&st[t], nBx, nBy, pairs_push, &pr);
    for (size_t i = before; i < pr.n; ++i) pr.tris[i] = t;
  }
  /* stable counting sort of the (bin, tri) pairs by bin: each bin's list keeps
   * insertion order, as the single-threaded ring buffers do */
  int nb = nBx * nBy;
  size_t* start = (size_t*)calloc((size_t)nb + 1, sizeof(size_t));
  for (size_t i = 0; i < pr.n; ++i) start[pr.bins[i] + 1]++;
  for (int b = 0; b < nb; ++b) start[b + 1] += start[b];
  int* lst = (int*)malloc(sizeof(int) * (pr.n ? pr.n : 1));
  size_t* cur = (size_t*)malloc(sizeof(size_t) * (nb ? nb : 1));
  for (int b = 0; b < nb; ++b) cur[b] = start[b];
  for (size_t i = 0; i < pr.n; ++i) lst[cur[pr.bins[i]]++] = pr.tris[i];

  frag_ctx fc;
  memset(&fc, 0, sizeof(fc));
  fc.W = W; fc.H = H; fc.nBx = nBx; fc.fb = fb;
  fc.zb = (int32_t*)malloc(sizeof(int32_t) * (size_t)W * H);
  fc.uv = uv; fc.tex = tex; fc.TW = TW; fc.TH = TH;
  for (size_t i = 0; i < (size_t)W * H; ++i) { fb[i] = CLEAR_COLOR; fc.zb[i] = f2bits(1.0f); }
  for (int b = 0; b < nb; ++b)
    for (size_t i = start[b]; i < start[b + 1]; ++i) {
      const stri* s = &st[lst[i]];
      shade_bin(&fc, s, lst[i], b, coverage_mask(s, b, nBx));
    }
  memcpy(depth, fc.zb, sizeof(float) * (size_t)W * H);
  if (stats) { stats[0] = kept; stats[1] = (long long)pr.n; stats[2] = fc.covered; stats[3] = fc.passed; }
  free(order); free(st); free(pr.bins); free(pr.tris); free(start); free(lst); free(cur); free(fc.zb);
  return 0;
}

/* Coverage masks of every (triangle, 8x8 bin) pair with a non-empty mask.
 * Writes up to cap records (tri, bin, mask); returns the total count. */
long long oracle_raster_coverage(int W, int H, int N, const float* xyz, const uint32_t* icol,
                                 int* out_tri, int* out_bin, uint64_t* out_mask, long long cap)
{
  int nBx = W / RB, nBy = H / RB;
  long long n = 0;
  stri s;
  for (int t = 0; t < N; ++t) {
    if (!vs_process(xyz, icol, t, W, H, &s)) continue;
    pairs pr = {0};
    raster_assign(&s, nBx, nBy, pairs_push, &pr);
    for (size_t i = 0; i < pr.n; ++i) {
      uint64_t m = coverage_mask(&s, pr.bins[i], nBx);
      if (!m) continue;
      if (n < cap) { out_tri[n] = t; out_bin[n] = pr.bins[i]; out_mask[n] = m; }
      n++;
    }
    free(pr.bins); free(pr.tris);
  }
  return n;
}
