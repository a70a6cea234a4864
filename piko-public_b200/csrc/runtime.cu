// Host runtime of libpiko_b200.so: contexts, pipeline descriptors, scenes,
// per-frame scratch, the frame launch sequence and the batched form.  It
// replaces the host code pikoc generates (allocate / prepare / run_single /
// destroy, pikoc/src/Backend/PTXBackend.cpp:741-1026) with a C ABI whose calls
// return status codes instead of exiting.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

#include "runtime_internal.h"

namespace piko {
cudaError_t launch_raster_frame(const RasterFrameArgs& a, int raster_ctas, cudaStream_t st, cudaEvent_t* ev);
cudaError_t raster_tiles_occupancy(int tile, int* blocks_per_sm);
}  // namespace piko

using namespace piko;

#define PIKO_VERSION "piko-b200 0.1"

namespace {

void fill_scene_dev(const RasterDraw& dr, int T, uint32_t tile_base, uint32_t tri_base, RasterSceneDev& d)
{
  const piko_scene* s = dr.mesh;
  const piko_const_state& stt = *dr.state;
  scene_dev_geometry(d, s->W, s->H, s->N, T);
  d.input_kind = s->kind == PIKO_SCENE_WTRI ? kInputWtri : s->kind == PIKO_SCENE_WTRI_WORLD ? kInputWtriWorld : kInputSoA;
  d.light_mode = stt.light_mode;
  d.tile_base = tile_base;
  d.tri_base = tri_base;
  memcpy(d.vp, stt.view_proj, sizeof(d.vp));
  memcpy(d.light, stt.light, sizeof(d.light));
  memcpy(d.eye, stt.eye, sizeof(d.eye));
  d.pos = s->pos; d.nrm = s->nrm; d.col = s->col; d.uv = s->uv;
  d.pos3 = s->pos3; d.nrm3 = s->nrm3;
  d.wtri_xyz = s->wtri_xyz; d.wtri_icol = s->wtri_icol;
  d.tex = s->tex; d.tex_w = s->tex_w; d.tex_h = s->tex_h;
  d.fb = dr.fb; d.depth = dr.depth;
}

}  // namespace

int raster_ctas(piko_ctx* ctx, int tile, int ctas_per_sm)
{
  int per_sm = ctas_per_sm;
  if (per_sm <= 0) {
    per_sm = 1;
    raster_tiles_occupancy(tile, &per_sm);
    if (per_sm < 1) per_sm = 1;
  }
  return ctx->sms * per_sm;
}

uint32_t heavy_threshold(int tile)
{
  // list entries above which a tile is served from the heavy queue first
  return tile == 8 ? 32u : 64u;
}

// Enqueues one frame of draws [0, n) sharing one scratch.
piko_status enqueue_raster_draws(piko_ctx* ctx, const RasterDraw* draws, int n, RasterScratch& scr, int T, int ctas,
                                 cudaStream_t st, bool timed, bool coverage, uint32_t chunk)
{
  if (chunk == 0) chunk = kDefaultChunk;
  uint32_t tris = 0, tiles = 0;
  for (int i = 0; i < n; ++i) {
    int tx, ty;
    tris += (uint32_t)draws[i].mesh->N;
    tiles += (uint32_t)tiles_for(draws[i].mesh->W, draws[i].mesh->H, T, &tx, &ty);
  }
  uint32_t list_need = std::max<uint32_t>(scr.list_cap, 4u * tris + tiles + 1024u);
  CU(ctx, scr.ensure(tris, tiles, list_need, n));
  static_assert(kQueueMin <= kQueueMax, "a group of short lists must fit one warp");
  const uint32_t queue_min = std::min(kQueueMin, chunk);
  CU(ctx, scr.ensure_heavy(tiles, T, chunk, queue_min));
  uint32_t tb = 0, rb = 0;
  for (int i = 0; i < n; ++i) {
    int tx, ty;
    fill_scene_dev(draws[i], T, tb, rb, scr.h_scenes[i]);
    tb += (uint32_t)tiles_for(draws[i].mesh->W, draws[i].mesh->H, T, &tx, &ty);
    rb += (uint32_t)draws[i].mesh->N;
  }
  CU(ctx, cudaMemcpyAsync(scr.d_scenes, scr.h_scenes, sizeof(RasterSceneDev) * n, cudaMemcpyHostToDevice, st));
  CU(ctx, cudaMemsetAsync(scr.ctr, 0, sizeof(FrameCounters), st));
  CU(ctx, cudaMemsetAsync(scr.tile_cnt, 0, sizeof(uint32_t) * tiles, st));
  CU(ctx, cudaMemsetAsync(scr.scan_flags, 0, sizeof(unsigned long long) * raster_scan_blocks(tiles), st));
  RasterFrameArgs a;
  memset(&a, 0, sizeof(a));
  a.scenes = scr.d_scenes;
  a.n_scenes = n;
  a.tile = T;
  a.n_tris_total = tris;
  a.n_tiles_total = tiles;
  a.setup = scr.setup;
  a.tile_cnt = scr.tile_cnt;
  a.tile_off = scr.tile_off;
  a.tile_list = scr.tile_list;
  a.pair_tl = scr.pair_tl;
  a.pair_g = scr.pair_g;
  a.list_cap = scr.list_cap;
  a.heavy = scr.heavy;
  a.heavy_threshold = heavy_threshold(T);
  a.heavy_cap = scr.heavy_cap;
  a.large_seg = scr.large_seg;
  a.seg_cap = scr.seg_cap;
  a.large_walk = scr.large_walk;
  a.big_cap = scr.seg_cap;
  a.chunk = chunk;
  a.queue_min = queue_min;
  a.chunk_base = scr.chunk_base;
  a.chunk_heavy = scr.chunk_heavy;
  a.hdone = scr.hdone;
  a.chunk_keys = scr.chunk_keys;
  a.chunk_cap = scr.chunk_cap;
  a.scan_flags = scr.scan_flags;
  a.epoch = 0;
  a.ctr = scr.ctr;
  if (coverage) {
    a.cov_tri = scr.cov_tri;
    a.cov_pix = scr.cov_pix;
    a.cov_cap = scr.cov_cap;
  }
  CU(ctx, launch_raster_frame(a, ctas, st, timed ? scr.ev : nullptr));
  return PIKO_OK;
}

piko_status enqueue_raster(piko_ctx* ctx, piko_scene* const* scenes, int n, RasterScratch& scr, const TuneCfg& cfg,
                           cudaStream_t st, bool timed, bool coverage)
{
  std::vector<RasterDraw> draws((size_t)n);
  for (int i = 0; i < n; ++i) draws[i] = RasterDraw{scenes[i], &scenes[i]->state, scenes[i]->fb, scenes[i]->depth};
  return enqueue_raster_draws(ctx, draws.data(), n, scr, cfg.tile, raster_ctas(ctx, cfg.tile, cfg.ctas_per_sm), st, timed,
                              coverage, cfg.chunk);
}

namespace {

// The status of a frame whose counters are already in scr.h_ctr; grows the
// bin-queue capacity when the device reported an overflow.  Returns
// PIKO_ERR_QUEUE_OVERFLOW when a re-run is needed.
piko_status check_counters(piko_ctx* ctx, RasterScratch& scr)
{
  const FrameCounters& c = *scr.h_ctr;
  if (c.status & kStatusScanTimeout) return set_err(ctx, PIKO_ERR_TIMEOUT, "%s", "tile scan look-back timed out");
  if (c.status & kStatusListOverflow) {
    CU(ctx, scr.regrow(c));
    return PIKO_ERR_QUEUE_OVERFLOW;
  }
  return PIKO_OK;
}

// Reads the counters of the last frame and checks them (check_counters).
piko_status check_frame(piko_ctx* ctx, RasterScratch& scr, cudaStream_t st)
{
  CU(ctx, cudaMemcpyAsync(scr.h_ctr, scr.ctr, sizeof(FrameCounters), cudaMemcpyDeviceToHost, st));
  CU(ctx, cudaStreamSynchronize(st));
  return check_counters(ctx, scr);
}

cudaStream_t pick_stream(piko_scene* s, void* stream)
{
  return stream ? (cudaStream_t)stream : s->own_stream;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

const char* piko_version(void) { return PIKO_VERSION; }

piko_status piko_ctx_create(const piko_ctx_opts* opts, piko_ctx** out)
{
  if (!out) return PIKO_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return PIKO_ERR_NO_DEVICE;
  }
  piko_ctx* c = new piko_ctx();
  c->device = opts ? opts->device : 0;
  c->time_kernels = opts ? opts->time_kernels != 0 : false;
  if (c->device < 0 || c->device >= ndev) { delete c; return PIKO_ERR_INVALID; }
  if (cudaSetDevice(c->device) != cudaSuccess) { delete c; return PIKO_ERR_CUDA; }
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return PIKO_ERR_CUDA; }
  *out = c;
  return PIKO_OK;
}

piko_status piko_ctx_destroy(piko_ctx* ctx)
{
  if (!ctx) return PIKO_ERR_INVALID;
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return PIKO_OK;
}

const char* piko_last_error(const piko_ctx* ctx) { return ctx ? ctx->err : "no context"; }

void piko_pipe_desc_raster(piko_pipe_desc* d)
{
  memset(d, 0, sizeof(*d));
  d->n_stages = 2;
  d->stages[0] = {32, 32, 512, PIKO_PRIM_RASTER_WTRI, PIKO_PRIM_RASTER_STRI};
  d->stages[1] = {8, 8, 32, PIKO_PRIM_RASTER_STRI, PIKO_PRIM_PIXEL};
  d->n_links = 1;
  d->links[0] = {0, 1, 0, 0};
}

void piko_pipe_desc_reyes(piko_pipe_desc* d)
{
  memset(d, 0, sizeof(*d));
  d->n_stages = 3;
  d->stages[0] = {0, 0, 256, PIKO_PRIM_PATCH, PIKO_PRIM_PATCH};
  d->stages[1] = {64, 64, 128, PIKO_PRIM_PATCH, PIKO_PRIM_UPOLY};
  d->stages[2] = {64, 64, 512, PIKO_PRIM_UPOLY, PIKO_PRIM_PIXEL};
  d->n_links = 3;
  d->links[0] = {0, 1, 0, 0};
  d->links[1] = {1, 2, 0, 0};
  d->links[2] = {0, 0, 1, 1};
}

static bool same_stage(const piko_stage_desc& a, const piko_stage_desc& b)
{
  return a.bin_size_x == b.bin_size_x && a.bin_size_y == b.bin_size_y && a.threads_per_tile == b.threads_per_tile &&
         a.in_prim == b.in_prim && a.out_prim == b.out_prim;
}

static bool same_shape(const piko_pipe_desc* d, const piko_pipe_desc& ref)
{
  if (d->n_stages != ref.n_stages || d->n_links != ref.n_links) return false;
  for (int i = 0; i < d->n_stages; ++i)
    if (!same_stage(d->stages[i], ref.stages[i])) return false;
  for (int i = 0; i < d->n_links; ++i) {
    bool found = false;
    for (int j = 0; j < ref.n_links; ++j)
      if (!memcmp(&d->links[i], &ref.links[j], sizeof(piko_link))) found = true;
    if (!found) return false;
  }
  return true;
}

piko_status piko_pipe_create(piko_ctx* ctx, const piko_pipe_desc* desc, piko_pipe** out)
{
  if (!ctx || !desc || !out) return PIKO_ERR_INVALID;
  *out = nullptr;
  if (desc->n_stages < 1 || desc->n_stages > PIKO_MAX_STAGES || desc->n_links < 0 || desc->n_links > PIKO_MAX_STAGES)
    return set_err(ctx, PIKO_ERR_INVALID, "%s", "stage or link count out of range");
  piko_pipe_desc r, y;
  piko_pipe_desc_raster(&r);
  piko_pipe_desc_reyes(&y);
  int kind = same_shape(desc, r) ? kPipeRaster : same_shape(desc, y) ? kPipeReyes : 0;
  if (!kind)
    return set_err(ctx, PIKO_ERR_UNSUPPORTED, "%s",
                   "pipeline shape not implemented (supported: RasterPipe, ReyesPipe)");
  if (desc->tile_px != 0 && desc->tile_px != 8 && desc->tile_px != 16 && desc->tile_px != 32)
    return set_err(ctx, PIKO_ERR_INVALID, "%s", "tile_px must be 8, 16 or 32");
  if (desc->samples_per_pixel != 0 && desc->samples_per_pixel != 1 && desc->samples_per_pixel != 4)
    return set_err(ctx, PIKO_ERR_INVALID, "%s", "samples_per_pixel must be 1 or 4");
  if (desc->phong != 0 && desc->phong != 1) return set_err(ctx, PIKO_ERR_INVALID, "%s", "phong must be 0 or 1");
  if (desc->chunk_entries < 0 || desc->chunk_entries > 4096)
    return set_err(ctx, PIKO_ERR_INVALID, "%s", "chunk_entries must be 0..4096");
  if (desc->split_threshold_px < 0.0f || desc->max_splits < 0 || desc->dice_grid < 0 || desc->dice_grid > 32)
    return set_err(ctx, PIKO_ERR_INVALID, "%s", "bad Reyes parameters");
  piko_pipe* p = new piko_pipe();
  p->ctx = ctx;
  p->kind = kind;
  p->tile = desc->tile_px ? desc->tile_px : 8;
  p->ctas_per_sm = desc->ctas_per_sm;
  p->chunk = desc->chunk_entries > 0 ? (uint32_t)desc->chunk_entries : 0u;
  p->split_threshold = desc->split_threshold_px > 0.0f ? desc->split_threshold_px : 4.0f;
  p->max_splits = desc->max_splits > 0 ? desc->max_splits : 20;
  p->dice_grid = desc->dice_grid;
  p->samples_per_pixel = desc->samples_per_pixel ? desc->samples_per_pixel : 1;
  p->sample_seed = desc->sample_seed;
  p->phong = desc->phong;
  *out = p;
  return PIKO_OK;
}

piko_status piko_pipe_destroy(piko_pipe* pipe)
{
  if (!pipe) return PIKO_ERR_INVALID;
  delete pipe;
  return PIKO_OK;
}

static void scene_free(piko_scene* s)
{
  dfree(s->pos); dfree(s->nrm); dfree(s->pos3); dfree(s->nrm3); dfree(s->col); dfree(s->uv); dfree(s->tex);
  dfree(s->wtri_xyz); dfree(s->wtri_icol); dfree(s->patches); dfree(s->fb); dfree(s->depth);
  s->scr.release();
  piko_reyes_release(s);
  if (s->own_stream) cudaStreamDestroy(s->own_stream);
  s->own_stream = nullptr;
}

static piko_status validate_desc(piko_ctx* ctx, piko_pipe* pipe, const piko_scene_desc* d)
{
  if (d->width < 32 || d->height < 32 || d->width > 16384 || d->height > 16384 || d->count < 0)
    return set_err(ctx, PIKO_ERR_INVALID, "%s", "framebuffer must be 32..16384 pixels per side; count >= 0");
  if (pipe->kind == kPipeRaster) {
    if (d->kind == PIKO_SCENE_TRIANGLES) {
      if (d->count && (!d->pos || !d->nrm))
        return set_err(ctx, PIKO_ERR_INVALID, "%s", "pos and nrm are required");
      if (d->uv) {
        if (!d->texture || d->tex_w <= 0 || d->tex_h <= 0 || (d->tex_w & (d->tex_w - 1)) || (d->tex_h & (d->tex_h - 1)))
          return set_err(ctx, PIKO_ERR_INVALID, "%s", "uv needs an RGBA8 texture with power-of-two sides");
      }
    } else if (d->kind == PIKO_SCENE_WTRI) {
      if (d->count && (!d->wtri_xyz || !d->wtri_icol))
        return set_err(ctx, PIKO_ERR_INVALID, "%s", "wtri_xyz and wtri_icol are required");
    } else if (d->kind == PIKO_SCENE_WTRI_WORLD) {
      if (d->count && !d->wtri_xyz) return set_err(ctx, PIKO_ERR_INVALID, "%s", "wtri_xyz is required");
    } else {
      return set_err(ctx, PIKO_ERR_INVALID, "%s",
                     "raster scenes are PIKO_SCENE_TRIANGLES, PIKO_SCENE_WTRI or PIKO_SCENE_WTRI_WORLD");
    }
  } else {
    if (d->kind != PIKO_SCENE_PATCHES || (d->count && !d->patches))
      return set_err(ctx, PIKO_ERR_INVALID, "%s", "Reyes scenes are PIKO_SCENE_PATCHES with patches");
  }
  return PIKO_OK;
}

static piko_status upload(piko_scene* s, const piko_scene_desc* d, cudaStream_t st)
{
  piko_ctx* ctx = s->pipe->ctx;
  const size_t n = (size_t)s->N;
  auto cp = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
    if (!bytes || !src) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
  };
  if (s->kind == PIKO_SCENE_TRIANGLES) {
    if (s->packed) {
      CU(ctx, cp(s->pos3, d->pos, 9 * n * sizeof(float)));
      CU(ctx, cp(s->nrm3, d->nrm, 9 * n * sizeof(float)));
    } else {
      CU(ctx, cp(s->pos, d->pos, 3 * n * sizeof(float4)));
      CU(ctx, cp(s->nrm, d->nrm, 3 * n * sizeof(float4)));
    }
    CU(ctx, cp(s->col, d->col, 3 * n * sizeof(float4)));
    if (s->uv) CU(ctx, cp(s->uv, d->uv, 3 * n * sizeof(float2)));
    if (s->tex) CU(ctx, cp(s->tex, d->texture, (size_t)s->tex_w * s->tex_h * 4));
  } else if (s->kind == PIKO_SCENE_WTRI || s->kind == PIKO_SCENE_WTRI_WORLD) {
    CU(ctx, cp(s->wtri_xyz, d->wtri_xyz, n * 9 * sizeof(float)));
    if (s->wtri_icol) CU(ctx, cp(s->wtri_icol, d->wtri_icol, n * 3 * sizeof(uint32_t)));
  } else {
    CU(ctx, cp(s->patches, d->patches, n * 16 * sizeof(float4)));
  }
  return PIKO_OK;
}

piko_status piko_scene_create(piko_pipe* pipe, const piko_scene_desc* d, piko_scene** out)
{
  if (!pipe || !d || !out) return PIKO_ERR_INVALID;
  *out = nullptr;
  piko_ctx* ctx = pipe->ctx;
  piko_status st = validate_desc(ctx, pipe, d);
  if (st != PIKO_OK) return st;
  cudaSetDevice(ctx->device);
  piko_scene* s = new piko_scene();
  s->pipe = pipe;
  s->kind = d->kind;
  s->W = d->width; s->H = d->height; s->N = d->count;
  const size_t n = (size_t)s->N;
  cudaError_t e = cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking);
  if (!e) e = dalloc(&s->fb, (size_t)s->W * s->H);
  if (!e) e = dalloc(&s->depth, (size_t)s->W * s->H);
  if (!e && s->kind == PIKO_SCENE_TRIANGLES) {
    s->packed = d->packed ? 1 : 0;
    if (s->packed) {
      e = dalloc(&s->pos3, 9 * n);
      if (!e) e = dalloc(&s->nrm3, 9 * n);
    } else {
      e = dalloc(&s->pos, 3 * n);
      if (!e) e = dalloc(&s->nrm, 3 * n);
    }
    if (!e && d->col) e = dalloc(&s->col, 3 * n);   // none: the fixed material colour
    if (!e && d->uv) {
      e = dalloc(&s->uv, 3 * n);
      s->tex_w = d->tex_w; s->tex_h = d->tex_h;
      if (!e) e = dalloc(&s->tex, (size_t)d->tex_w * d->tex_h);
    }
  } else if (!e && (s->kind == PIKO_SCENE_WTRI || s->kind == PIKO_SCENE_WTRI_WORLD)) {
    e = dalloc(&s->wtri_xyz, n * 9);
    if (!e && s->kind == PIKO_SCENE_WTRI) e = dalloc(&s->wtri_icol, n * 3);
  } else if (!e && s->kind == PIKO_SCENE_PATCHES) {
    e = dalloc(&s->patches, n * 16);
  }
  if (e) {
    scene_free(s);
    delete s;
    return set_err(ctx, e == cudaErrorMemoryAllocation ? PIKO_ERR_OOM : PIKO_ERR_CUDA, "%s", cudaGetErrorString(e));
  }
  // default state: identity camera, the reference's fixed light (main.cpp:384)
  for (int i = 0; i < 16; ++i) s->state.view_proj[i] = (i % 5 == 0) ? 1.0f : 0.0f;
  s->state.light_mode = 0;
  s->state.light[0] = s->state.light[1] = s->state.light[2] = 0.5773f;
  st = upload(s, d, s->own_stream);
  if (st == PIKO_OK && cudaStreamSynchronize(s->own_stream) != cudaSuccess) st = set_err(ctx, PIKO_ERR_CUDA, "%s", "upload failed");
  if (st != PIKO_OK) {
    scene_free(s);
    delete s;
    return st;
  }
  *out = s;
  return PIKO_OK;
}

piko_status piko_scene_upload(piko_scene* s, const piko_scene_desc* d, void* stream)
{
  if (!s || !d) return PIKO_ERR_INVALID;
  if (d->kind != s->kind || d->count != s->N || d->width != s->W || d->height != s->H)
    return set_err(s->pipe->ctx, PIKO_ERR_INVALID, "%s", "upload must keep kind, count and size");
  if ((d->uv != nullptr) != (s->uv != nullptr))
    return set_err(s->pipe->ctx, PIKO_ERR_INVALID, "%s", "upload must keep the textured variant");
  if (d->kind == PIKO_SCENE_TRIANGLES && (d->col != nullptr) != (s->col != nullptr))
    return set_err(s->pipe->ctx, PIKO_ERR_INVALID, "%s", "upload must keep the colour source");
  if (d->kind == PIKO_SCENE_TRIANGLES && (d->packed != 0) != (s->packed != 0))
    return set_err(s->pipe->ctx, PIKO_ERR_INVALID, "%s", "upload must keep the packed layout");
  return upload(s, d, pick_stream(s, stream));
}

piko_status piko_scene_destroy(piko_scene* s)
{
  if (!s) return PIKO_ERR_INVALID;
  if (s->last_stream) cudaStreamSynchronize(s->last_stream);
  scene_free(s);
  delete s;
  return PIKO_OK;
}

piko_status piko_frame_prepare(piko_scene* s, const piko_const_state* state)
{
  if (!s || !state) return PIKO_ERR_INVALID;
  if (state->light_mode != 0 && state->light_mode != 1)
    return set_err(s->pipe->ctx, PIKO_ERR_INVALID, "%s", "light_mode must be 0 or 1");
  s->state = *state;
  return PIKO_OK;
}

piko_status piko_frame_run(piko_scene* s, void* stream)
{
  if (!s) return PIKO_ERR_INVALID;
  piko_ctx* ctx = s->pipe->ctx;
  cudaStream_t st = pick_stream(s, stream);
  s->timed = ctx->time_kernels;
  piko_status r;
  if (s->pipe->kind == kPipeReyes) {
    r = piko_reyes_run(s, st, s->timed);
  } else {
    piko_scene* one[1] = {s};
    r = enqueue_raster(ctx, one, 1, s->scr, pipe_cfg(s->pipe), st, s->timed, false);
  }
  if (r == PIKO_OK) { s->last_stream = st; s->pending = true; }
  return r;
}

piko_status piko_frame_finish(piko_scene* s)
{
  if (!s) return PIKO_ERR_INVALID;
  if (!s->pending) return PIKO_OK;
  if (s->pipe->kind == kPipeReyes) return piko_reyes_finish(s);
  piko_ctx* ctx = s->pipe->ctx;
  for (int attempt = 0; attempt < 4; ++attempt) {
    piko_status r = check_frame(ctx, s->scr, s->last_stream);
    if (r == PIKO_OK) { s->pending = false; return PIKO_OK; }
    if (r != PIKO_ERR_QUEUE_OVERFLOW) return r;
    piko_scene* one[1] = {s};
    r = enqueue_raster(ctx, one, 1, s->scr, pipe_cfg(s->pipe), s->last_stream, s->timed, false);
    if (r != PIKO_OK) return r;
  }
  return set_err(ctx, PIKO_ERR_QUEUE_OVERFLOW, "%s", "bin queues kept overflowing");
}

piko_status piko_frame_read(piko_scene* s, uint32_t* rgba, float* depth)
{
  if (!s) return PIKO_ERR_INVALID;
  piko_ctx* ctx = s->pipe->ctx;
  const size_t n = (size_t)s->W * s->H;
  auto copy_image = [&](cudaStream_t st) -> cudaError_t {
    cudaError_t e = cudaSuccess;
    if (rgba) e = cudaMemcpyAsync(rgba, s->fb, n * 4, cudaMemcpyDeviceToHost, st);
    if (!e && depth) e = cudaMemcpyAsync(depth, s->depth, n * 4, cudaMemcpyDeviceToHost, st);
    return e;
  };
  if (s->pending && s->pipe->kind == kPipeRaster) {
    // one wait for the frame's counters and image together; a frame that
    // overflowed its queues is drawn again (finish) and copied again
    cudaStream_t st = s->last_stream;
    CU(ctx, cudaMemcpyAsync(s->scr.h_ctr, s->scr.ctr, sizeof(FrameCounters), cudaMemcpyDeviceToHost, st));
    CU(ctx, copy_image(st));
    CU(ctx, cudaStreamSynchronize(st));
    const piko_status r = check_counters(ctx, s->scr);
    if (r == PIKO_OK) {
      s->pending = false;
      return PIKO_OK;
    }
    if (r != PIKO_ERR_QUEUE_OVERFLOW) return r;
    piko_scene* one[1] = {s};
    const piko_status rr = enqueue_raster(ctx, one, 1, s->scr, pipe_cfg(s->pipe), st, s->timed, false);
    if (rr != PIKO_OK) return rr;
  }
  piko_status r = piko_frame_finish(s);
  if (r != PIKO_OK) return r;
  cudaStream_t st = s->last_stream ? s->last_stream : s->own_stream;
  CU(ctx, copy_image(st));
  CU(ctx, cudaStreamSynchronize(st));
  return PIKO_OK;
}

piko_status piko_frame_device_buffers(piko_scene* s, uint32_t** rgba, float** depth)
{
  if (!s) return PIKO_ERR_INVALID;
  if (rgba) *rgba = s->fb;
  if (depth) *depth = s->depth;
  return PIKO_OK;
}

// Adds one launch sequence's counters (and kernel times) to *o.
static void fill_stats(const RasterScratch& scr, bool timed, piko_frame_stats* o)
{
  const FrameCounters& c = *scr.h_ctr;
  o->prims_kept += c.kept;
  o->bin_entries += c.list_total;
  o->covered += c.covered;
  o->wrap_risk += c.risk;
  o->status |= c.status;
  if (timed && scr.ev_made) {
    o->n_kernels = 4;
    for (int i = 0; i < 4; ++i) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, scr.ev[i], scr.ev[i + 1]);
      o->kernel_ms[i] += ms;
    }
  }
}

piko_status piko_frame_stats_get(piko_scene* s, piko_frame_stats* out)
{
  if (!s || !out) return PIKO_ERR_INVALID;
  memset(out, 0, sizeof(*out));
  piko_status r = piko_frame_finish(s);
  if (r != PIKO_OK) return r;
  if (s->pipe->kind == kPipeReyes) return piko_reyes_stats(s, out);
  if (!s->scr.h_ctr) return PIKO_OK;
  piko_ctx* ctx = s->pipe->ctx;
  CU(ctx, cudaMemcpy(s->scr.h_ctr, s->scr.ctr, sizeof(FrameCounters), cudaMemcpyDeviceToHost));
  out->prims_in = (uint64_t)s->N;
  fill_stats(s->scr, s->timed, out);
  return PIKO_OK;
}

piko_status piko_frame_coverage(piko_scene* s, uint32_t* tri, uint32_t* pix, uint64_t cap, uint64_t* count)
{
  if (!s || !count) return PIKO_ERR_INVALID;
  if (s->pipe->kind != kPipeRaster) return PIKO_ERR_UNSUPPORTED;
  piko_ctx* ctx = s->pipe->ctx;
  piko_status r = piko_frame_finish(s);
  if (r != PIKO_OK) return r;
  cudaStream_t st = s->own_stream;
  uint32_t want = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(cap, 1), 1u << 30);
  for (int attempt = 0; attempt < 4; ++attempt) {
    if (want > s->scr.cov_cap) {
      dfree(s->scr.cov_tri); dfree(s->scr.cov_pix);
      CU(ctx, dalloc(&s->scr.cov_tri, want));
      CU(ctx, dalloc(&s->scr.cov_pix, want));
      s->scr.cov_cap = want;
    }
    piko_scene* one[1] = {s};
    r = enqueue_raster(ctx, one, 1, s->scr, pipe_cfg(s->pipe), st, false, true);
    if (r != PIKO_OK) return r;
    r = check_frame(ctx, s->scr, st);
    if (r == PIKO_OK) break;
    if (r != PIKO_ERR_QUEUE_OVERFLOW) return r;
  }
  uint64_t n = s->scr.h_ctr->cov_count;
  *count = n;
  uint64_t m = std::min<uint64_t>(std::min<uint64_t>(n, cap), s->scr.cov_cap);
  if (m && tri) CU(ctx, cudaMemcpy(tri, s->scr.cov_tri, m * 4, cudaMemcpyDeviceToHost));
  if (m && pix) CU(ctx, cudaMemcpy(pix, s->scr.cov_pix, m * 4, cudaMemcpyDeviceToHost));
  s->pending = false;
  return PIKO_OK;
}

// ------------------------------------------------------------------ batched form
}  // extern "C"

// Groups the scenes by launch configuration (cfgs[i] for scene i) and makes a
// batch with one launch sequence per group.
piko_status batch_make(piko_ctx* ctx, piko_scene* const* scenes, int n, const TuneCfg* cfgs, piko_batch** out)
{
  piko_batch* b = new piko_batch();
  b->ctx = ctx;
  b->scenes.assign(scenes, scenes + n);
  for (int i = 0; i < n; ++i) {
    BatchGroup* g = nullptr;
    for (auto* x : b->groups)
      if (x->cfg == cfgs[i]) g = x;
    if (!g) {
      g = new BatchGroup();
      g->cfg = cfgs[i];
      b->groups.push_back(g);
    }
    g->scenes.push_back(scenes[i]);
  }
  cudaError_t e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (size_t k = 0; k < b->groups.size() && e == cudaSuccess; ++k) {
    e = cudaEventCreateWithFlags(&b->groups[k]->done, cudaEventDisableTiming);
    if (k > 0 && e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->groups[k]->stream, cudaStreamNonBlocking);
  }
  if (e != cudaSuccess) {
    piko_batch_destroy(b);
    return set_err(ctx, PIKO_ERR_CUDA, "%s", cudaGetErrorString(e));
  }
  *out = b;
  return PIKO_OK;
}

// Enqueues every group: group 0 on st, the others on their own streams forked
// from st and joined back into it (parallel branches when captured).
static piko_status batch_enqueue(piko_batch* b, cudaStream_t st, bool timed)
{
  piko_ctx* ctx = b->ctx;
  const bool fork = b->groups.size() > 1;
  if (fork) CU(ctx, cudaEventRecord(b->fork, st));
  for (size_t k = 0; k < b->groups.size(); ++k) {
    BatchGroup* g = b->groups[k];
    cudaStream_t gs = k == 0 ? st : g->stream;
    if (k > 0) CU(ctx, cudaStreamWaitEvent(gs, b->fork, 0));
    piko_status r = enqueue_raster(ctx, g->scenes.data(), (int)g->scenes.size(), g->scr, g->cfg, gs, timed, false);
    if (r != PIKO_OK) return r;
    if (k > 0) CU(ctx, cudaEventRecord(g->done, gs));
  }
  for (size_t k = 1; k < b->groups.size(); ++k) CU(ctx, cudaStreamWaitEvent(st, b->groups[k]->done, 0));
  return PIKO_OK;
}

extern "C" {

piko_status piko_batch_create(piko_ctx* ctx, piko_scene* const* scenes, int n, piko_batch** out)
{
  if (!ctx || !scenes || n <= 0 || !out) return PIKO_ERR_INVALID;
  *out = nullptr;
  const TuneCfg c0 = pipe_cfg(scenes[0]->pipe);
  std::vector<TuneCfg> cfgs((size_t)n, c0);
  for (int i = 0; i < n; ++i) {
    if (!scenes[i] || scenes[i]->pipe->kind != kPipeRaster)
      return set_err(ctx, PIKO_ERR_UNSUPPORTED, "%s", "batches hold raster scenes");
    if (scenes[i]->pipe->tile != c0.tile)
      return set_err(ctx, PIKO_ERR_INVALID, "%s", "scenes of one batch share the tile size (use a tuner for mixed sizes)");
  }
  return batch_make(ctx, scenes, n, cfgs.data(), out);
}

static void drop_graph(piko_batch* b)
{
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->graph_exec = nullptr;
  b->graph = nullptr;
  b->graph_stream = nullptr;
}

piko_status piko_batch_run(piko_batch* b, void* stream, int use_graph)
{
  if (!b) return PIKO_ERR_INVALID;
  piko_ctx* ctx = b->ctx;
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  const bool timed = ctx->time_kernels;
  if (use_graph && !timed) {
    if (!b->graph_exec) {
      // size the scratch outside the capture (allocation is not capturable)
      piko_status r = batch_enqueue(b, st, false);
      if (r != PIKO_OK) return r;
      CU(ctx, cudaStreamSynchronize(st));
      CU(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      r = batch_enqueue(b, st, false);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(st, &g);
      if (r != PIKO_OK) { if (g) cudaGraphDestroy(g); return r; }
      CU(ctx, e);
      b->graph = g;
      CU(ctx, cudaGraphInstantiate(&b->graph_exec, g, 0));
    }
    CU(ctx, cudaGraphLaunch(b->graph_exec, st));
  } else {
    piko_status r = batch_enqueue(b, st, timed);
    if (r != PIKO_OK) return r;
  }
  b->last_stream = st;
  b->pending = true;
  return PIKO_OK;
}

piko_status piko_batch_finish(piko_batch* b, piko_frame_stats* out)
{
  if (!b) return PIKO_ERR_INVALID;
  piko_ctx* ctx = b->ctx;
  if (out) memset(out, 0, sizeof(*out));
  if (b->pending) {
    for (auto* g : b->groups) {
      for (int attempt = 0;; ++attempt) {
        piko_status r = check_frame(ctx, g->scr, b->last_stream);
        if (r == PIKO_OK) break;
        if (r != PIKO_ERR_QUEUE_OVERFLOW || attempt >= 3) return r;
        drop_graph(b);  // the queue buffers moved
        r = enqueue_raster(ctx, g->scenes.data(), (int)g->scenes.size(), g->scr, g->cfg, b->last_stream, false, false);
        if (r != PIKO_OK) return r;
      }
    }
    b->pending = false;
  }
  if (out) {
    for (auto* s : b->scenes) out->prims_in += (uint64_t)s->N;
    for (auto* g : b->groups)
      if (g->scr.h_ctr) fill_stats(g->scr, ctx->time_kernels, out);
  }
  return PIKO_OK;
}

piko_status piko_batch_destroy(piko_batch* b)
{
  if (!b) return PIKO_ERR_INVALID;
  if (b->last_stream) cudaStreamSynchronize(b->last_stream);
  drop_graph(b);
  for (auto* g : b->groups) {
    if (g->stream) cudaStreamSynchronize(g->stream);
    g->scr.release();
    if (g->done) cudaEventDestroy(g->done);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
  }
  if (b->fork) cudaEventDestroy(b->fork);
  delete b;
  return PIKO_OK;
}

}  // extern "C"

