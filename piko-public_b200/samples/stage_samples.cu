// Two pipelines written against the stage API of include/piko_stage.cuh (the
// reference's Stage / assignBin / schedule / process / emit interface), built
// into libpiko_stage_samples.so and driven by tests/test_stage_api.py:
//
//  * raster2: the reference's RasterPipe structure -- a vertex stage in
//    32x32-pixel bins taking (id / 512) % bins (vertexShader.pikostage:25-29)
//    that quantizes pre-transformed triangles to 28.4 and culls them
//    (:36-109), and a raster stage in 8x8 bins with the trivial reject of
//    raster.pikostage:77-105 whose process tests the pixel centres of its bin
//    with the 28.4 edge functions, resolves depth with the atomicMin loop on
//    the depth bits and emits Gouraud-coloured Pixels to the screen
//    (:124-320).  The runtime resolves the screen in the reference's
//    one-thread order, so depth, the covered-sample count and the colour all
//    equal the sequential CPU result.  The covered-sample counter is a side
//    effect of process, so it counts in pass 0 only (the screen resolve runs
//    process twice more).
//  * subdivide: a stage connected to itself (like the reference's Split
//    stage) halves segments longer than a threshold, up to a depth limit, and
//    sends the rest to a stamp stage in 16x16 bins that marks each segment's
//    midpoint on the screen.
#include <climits>
#include <cstdio>

#include "../../include/piko_stage.cuh"

namespace {

__device__ __forceinline__ int32_t trunc_i32(float f)
{
  return (f >= -2147483648.0f && f < 2147483648.0f) ? __float2int_rz(f) : INT32_MIN;
}
__device__ __forceinline__ int32_t wsub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
__device__ __forceinline__ int32_t wmul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }
__device__ __forceinline__ int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
__device__ __forceinline__ int32_t wshl(int32_t a, int s) { return (int32_t)((uint32_t)a << s); }

// ----------------------------------------------------------------- raster2
struct WTri {            // pre-transformed triangle: screen x, y (pixels), depth, ABGR colours
  int id;
  float x[3], y[3], z[3];
  unsigned icol[3];
};
struct STri {            // 28.4 screen triangle
  int id;
  int32_t x[3], y[3];
  float z[3];
  unsigned icol[3];
};

struct VertexStage : piko::Stage<32, 32, 512, WTri, STri> {
  __device__ void assignBin(WTri p) { assignToBin(p, (p.id / 512) % getNumBins()); }
  __device__ void schedule(int) { specifySchedule(piko::LOAD_BALANCE); }
  __device__ void process(WTri p)
  {
    STri s;
    s.id = p.id;
    for (int k = 0; k < 3; ++k) {
      s.x[k] = trunc_i32(p.x[k] * 16.0f);
      s.y[k] = trunc_i32(p.y[k] * 16.0f);
      s.z[k] = p.z[k];
      s.icol[k] = p.icol[k];
    }
    const int W = constState.screenSizeX * 16, H = constState.screenSizeY * 16, guard = 225 << 4;
    // front facing, inside the guard band, not between sample rows
    if (wsub(wmul(wsub(s.y[2], s.y[0]), wsub(s.x[1], s.x[0])), wmul(wsub(s.x[2], s.x[0]), wsub(s.y[1], s.y[0]))) <= 0)
      return;
    for (int k = 0; k < 3; ++k)
      if (s.x[k] < -guard || s.x[k] >= W + guard || s.y[k] < -guard || s.y[k] >= H + guard) return;
    const int32_t lo = min(min(s.y[0], s.y[1]), s.y[2]), hi = max(max(s.y[0], s.y[1]), s.y[2]);
    if ((wsub(lo, 8) >> 4) == (wsub(hi, 8) >> 4)) return;
    emit(s, 0);
  }
};

struct RasterStage : piko::Stage<8, 8, 32, STri, piko::Pixel> {
  unsigned long long* covered;   // covered samples (counted by the sample)

  __device__ void assignBin(STri p)
  {
    const int32_t lox = min(min(p.x[0], p.x[1]), p.x[2]) & (int32_t)0xffffff00;
    const int32_t loy = min(min(p.y[0], p.y[1]), p.y[2]) & (int32_t)0xffffff00;
    const int32_t hix = wadd(max(max(p.x[0], p.x[1]), p.x[2]), 0xff) & (int32_t)0xffffff00;
    const int32_t hiy = wadd(max(max(p.y[0], p.y[1]), p.y[2]), 0xff) & (int32_t)0xffffff00;
    const int bx1 = max(0, lox >> 7), bx2 = min(hix >> 7, getNumBinsX() - 1);
    const int by1 = max(0, loy >> 7), by2 = min(hiy >> 7, getNumBinsY() - 1);
    for (int by = by1; by <= by2; ++by)
      for (int bx = bx1; bx <= bx2; ++bx) {
        int32_t tr = 0;
        for (int i = 0; i < 3; ++i) {
          const int j = i == 2 ? 0 : i + 1;
          const int32_t dx = wsub(p.x[j], p.x[i]), dy = wsub(p.y[j], p.y[i]);
          int32_t off = dy < 0 ? -wshl(dy, 7) : 0;
          off = wadd(off, dx >= 0 ? wshl(dx, 7) : 0);
          tr |= wadd(off, wsub(wmul(wsub(by * 128, p.y[i]), dx), wmul(wsub(bx * 128, p.x[i]), dy)));
        }
        if (tr >= 0) assignToBin(p, by * getNumBinsX() + bx);
      }
  }
  __device__ void schedule(int) { specifySchedule(piko::LOAD_BALANCE); }
  __device__ void process(STri p)
  {
    const int bin = getBinID();
    const int bx = (bin % getNumBinsX()) * 8, by = (bin / getNumBinsX()) * 8;
    const int32_t hix = wadd(max(max(p.x[0], p.x[1]), p.x[2]), 0xff) & (int32_t)0xffffff00;
    const int32_t hiy = wadd(max(max(p.y[0], p.y[1]), p.y[2]), 0xff) & (int32_t)0xffffff00;
    const int32_t x1mx0 = wsub(p.x[1], p.x[0]), y1my0 = wsub(p.y[1], p.y[0]);
    const int32_t x2mx1 = wsub(p.x[2], p.x[1]), y2my1 = wsub(p.y[2], p.y[1]);
    const int32_t x0mx2 = wsub(p.x[0], p.x[2]), y0my2 = wsub(p.y[0], p.y[2]);
    const float inv = piko::rcp_approx((float)wadd(wmul(-y0my2, x1mx0), wmul(x0mx2, y1my0)));
    // trivial accept of the whole bin at its first pixel centre
    int32_t ta = 0;
    const int32_t dxs[3] = {x1mx0, x2mx1, x0mx2}, dys[3] = {y1my0, y2my1, y0my2};
    for (int i = 0; i < 3; ++i) {
      int32_t offa = dys[i] >= 0 ? -wshl(dys[i], 4) : 0;
      offa = wadd(offa, dxs[i] < 0 ? wshl(dxs[i], 4) : 0);
      ta |= wadd(wsub(wmul(wsub(by * 16 + 8, p.y[i]), dxs[i]), wmul(wsub(bx * 16 + 8, p.x[i]), dys[i])), wshl(offa, 3));
    }
    const bool accept = (ta & (int32_t)0x80000000) == 0;
    unsigned long long n = 0;
    for (int q = 0; q < 64; ++q) {
      const int px = bx + (q & 7), py = by + (q >> 3);
      const int32_t X = px * 16 + 8, Y = py * 16 + 8;
      const int32_t e0 = wsub(wmul(wsub(Y, p.y[0]), x1mx0), wmul(wsub(X, p.x[0]), y1my0));
      const int32_t e1 = wsub(wmul(wsub(Y, p.y[1]), x2mx1), wmul(wsub(X, p.x[1]), y2my1));
      const int32_t e2 = wsub(wmul(wsub(Y, p.y[2]), x0mx2), wmul(wsub(X, p.x[2]), y0my2));
      const bool cov = accept || (px < (hix >> 4) && py < (hiy >> 4) && (e0 | e1 | e2) >= 0);
      if (!cov) continue;
      ++n;
      const float alpha = (float)e1 * inv, beta = (float)e2 * inv;
      const float z = p.z[2] + alpha * (p.z[0] - p.z[2]) + beta * (p.z[1] - p.z[2]);
      // the reference's depth loop on the bits as signed ints (ties pass); the
      // stored value only decreases, so the second atomicMin returns at most
      // `mine` and the loop ends
      int* zb = reinterpret_cast<int*>(mutableState->zBuffer) + (size_t)py * constState.screenSizeX + px;
      const int mine = __float_as_int(z);
      int remote;
      do { remote = atomicMin(zb, mine); } while (remote > mine);
      if (remote < mine) continue;
      // Gouraud colour with the reference's helpers (raster.pikostage:183-185,
      // 251-252, 289-309): fromABGR, vertex differences, interpolation in the
      // reference's order, toABGR by truncation
      const piko::cvec3f v0 = piko::fromABGR(p.icol[0]), v1 = piko::fromABGR(p.icol[1]),
                         v2 = piko::fromABGR(p.icol[2]);
      const piko::cvec3f d0 = v0 - v2, d1 = v1 - v2;
      piko::cvec3f c;
      c.x = v2.x + alpha * d0.x + beta * d1.x;
      c.y = v2.y + alpha * d0.y + beta * d1.y;
      c.z = v2.z + alpha * d0.z + beta * d1.z;
      piko::Pixel pix;
      pix.pos.x = px;
      pix.pos.y = py;
      pix.color = piko::toABGR(c);
      emit(pix, 0);
    }
    if (n && passIndex() == 0) atomicAdd(covered, n);
  }
};

// --------------------------------------------------------------- subdivide
struct Seg {
  int binID;
  float x0, y0, x1, y1;
  int depth;
};

struct SplitSeg : piko::Stage<0, 0, 64, Seg, Seg> {
  float threshold;
  int max_depth;
  __device__ void assignBin(Seg s) { assignToBin(s, 0); }
  __device__ void schedule(int) { specifySchedule(piko::LOAD_BALANCE); }
  __device__ void process(Seg s)
  {
    const float dx = s.x1 - s.x0, dy = s.y1 - s.y0;
    if (sqrtf(dx * dx + dy * dy) >= threshold && s.depth < max_depth) {
      const float mx = (s.x0 + s.x1) * 0.5f, my = (s.y0 + s.y1) * 0.5f;
      emit(Seg{0, s.x0, s.y0, mx, my, s.depth + 1}, 1);
      emit(Seg{0, mx, my, s.x1, s.y1, s.depth + 1}, 1);
    } else {
      emit(s, 0);
    }
  }
};

struct Stamp : piko::Stage<16, 16, 64, Seg, piko::Pixel> {
  unsigned long long* leaves;
  __device__ void assignBin(Seg s)
  {
    const int x = __float2int_rd((s.x0 + s.x1) * 0.5f), y = __float2int_rd((s.y0 + s.y1) * 0.5f);
    if (x < 0 || y < 0 || x >= constState.screenSizeX || y >= constState.screenSizeY) return;
    // the bin grid covers whole bins only: the border strip joins the last bin
    assignToBin(s, min(y / 16, getNumBinsY() - 1) * getNumBinsX() + min(x / 16, getNumBinsX() - 1));
  }
  __device__ void schedule(int) { specifySchedule(piko::ROUND_ROBIN); }
  __device__ void process(Seg s)
  {
    if (passIndex() == 0) atomicAdd(leaves, 1ull);
    piko::Pixel p;
    p.pos.x = __float2int_rd((s.x0 + s.x1) * 0.5f);
    p.pos.y = __float2int_rd((s.y0 + s.y1) * 0.5f);
    p.color = 0xffffffffu;
    emit(p, 0);
  }
};

}  // namespace

extern "C" {

// raster2 on count pre-transformed triangles (xyz [count][9]: x, y, z of each
// vertex in pixels / depth; icol [count][3]); fb and depth receive W*H words.
// Returns 0, or -1 with the message on stderr.
int piko_sample_raster(int W, int H, const float* xyz, const unsigned* icol, int count, unsigned* fb, float* depth,
                       unsigned long long* covered)
{
  try {
    std::vector<WTri> in((size_t)count);
    for (int i = 0; i < count; ++i) {
      in[i].id = i;
      for (int k = 0; k < 3; ++k) {
        in[i].x[k] = xyz[9 * i + 3 * k];
        in[i].y[k] = xyz[9 * i + 3 * k + 1];
        in[i].z[k] = xyz[9 * i + 3 * k + 2];
        in[i].icol[k] = icol[3 * i + k];
      }
    }
    piko::Pipe<VertexStage, RasterStage> pipe;
    pipe.connect(0, 0, 1);
    pipe.connect(1, 0, piko::kScreen);
    piko::ConstantState cs;
    memset(&cs, 0, sizeof(cs));
    cs.screenSizeX = W; cs.screenSizeY = H;
    cs.halfW = 0.5f * (float)W; cs.halfH = 0.5f * (float)H;
    float* d_z = nullptr;
    unsigned long long* d_cov = nullptr;
    if (cudaMalloc(&d_z, sizeof(float) * (size_t)W * H) != cudaSuccess) return -1;
    if (cudaMalloc(&d_cov, sizeof(unsigned long long)) != cudaSuccess) { cudaFree(d_z); return -1; }
    std::vector<float> ones((size_t)W * H, 1.0f);
    cudaMemcpy(d_z, ones.data(), sizeof(float) * ones.size(), cudaMemcpyHostToDevice);
    cudaMemset(d_cov, 0, sizeof(unsigned long long));
    piko::MutableState ms{d_z};
    std::get<1>(pipe.stages).covered = d_cov;
    pipe.allocate(cs, ms, in.data(), count);
    pipe.prepare();
    pipe.run_single();
    pipe.getData(fb);
    cudaMemcpy(depth, d_z, sizeof(float) * (size_t)W * H, cudaMemcpyDeviceToHost);
    cudaMemcpy(covered, d_cov, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d_z);
    cudaFree(d_cov);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  } catch (const std::exception& e) {
    fprintf(stderr, "piko_sample_raster: %s\n", e.what());
    return -1;
  }
}

// subdivide on count segments (segs [count][4]: x0, y0, x1, y1 in pixels).
int piko_sample_subdivide(int W, int H, const float* segs, int count, float threshold, int max_depth, unsigned* fb,
                          unsigned long long* leaves, int* rounds, unsigned long long* split_processed)
{
  try {
    std::vector<Seg> in((size_t)count);
    for (int i = 0; i < count; ++i) in[i] = Seg{0, segs[4 * i], segs[4 * i + 1], segs[4 * i + 2], segs[4 * i + 3], 0};
    piko::Pipe<SplitSeg, Stamp> pipe;
    pipe.connect(0, 1, 0);             // the self loop
    pipe.connect(0, 0, 1);
    pipe.connect(1, 0, piko::kScreen);
    std::get<0>(pipe.stages).threshold = threshold;
    std::get<0>(pipe.stages).max_depth = max_depth;
    unsigned long long* d_leaves = nullptr;
    if (cudaMalloc(&d_leaves, sizeof(unsigned long long)) != cudaSuccess) return -1;
    cudaMemset(d_leaves, 0, sizeof(unsigned long long));
    std::get<1>(pipe.stages).leaves = d_leaves;
    piko::ConstantState cs;
    memset(&cs, 0, sizeof(cs));
    cs.screenSizeX = W; cs.screenSizeY = H;
    piko::MutableState ms{nullptr};
    pipe.allocate(cs, ms, in.data(), count);
    pipe.clearScreen(0xff000000u);
    pipe.prepare();
    pipe.run_single();
    pipe.getData(fb);
    cudaMemcpy(leaves, d_leaves, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d_leaves);
    *rounds = pipe.rounds(0);
    *split_processed = pipe.processed()[0];
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  } catch (const std::exception& e) {
    fprintf(stderr, "piko_sample_subdivide: %s\n", e.what());
    return -1;
  }
}

}  // extern "C"
