// Launch-configuration tuner of the batched raster form (no reference
// counterpart: the reference fixes its bin sizes in the pipeline source and
// pikoc's planner picks no launch shapes at run time).
//
// Scenes fall into 16 buckets by resolution class (<= 256^2, <= 512^2,
// <= 1280x720, larger) and triangle class (< 4K, < 16K, < 64K, more).  For
// every bucket that holds scenes of a given mix, tune() renders those scenes as
// one batch with each candidate configuration -- tile edge 8 / 16 / 32 px,
// persistent CTAs per SM, list entries per chunk of the 8x8 tile queue -- and
// keeps the fastest (median device time of replayed CUDA graphs); the table is
// then checked on the whole mix against each candidate used for every scene:
// the mixed table stays only if it beats the fastest single configuration by
// more than 3%, else that configuration is used for every bucket.  A tuned batch groups its scenes by their
// bucket's configuration and runs one launch sequence per group on parallel
// branches of one graph.  Every
// configuration renders the same image (coverage and depth are tile-size
// invariant, the winner key is order independent), so tuning changes speed
// only.
#include <algorithm>
#include <vector>

#include "runtime_internal.h"

int tune_bucket(int W, int H, int N)
{
  const long long px = (long long)W * H;
  const int r = px <= 256LL * 256 ? 0 : px <= 512LL * 512 ? 1 : px <= 1280LL * 720 ? 2 : 3;
  const int t = N < 4096 ? 0 : N < 16384 ? 1 : N < 65536 ? 2 : 3;
  return r * 4 + t;
}

namespace {

const TuneCfg kCandidates[] = {
    {8, 0, 16}, {8, 0, 32}, {8, 0, 64}, {8, 2, 32}, {8, 3, 32},
    {16, 0, 0}, {16, 1, 0},
    {32, 0, 0}, {32, 2, 0},
};

// Median device time (ms) of `reps` graph replays of a batch of `scenes`,
// scene i drawn with cfgs[i]; <0 on failure.
float time_cfgs(piko_ctx* ctx, const std::vector<piko_scene*>& scenes, const std::vector<TuneCfg>& cfgs, int reps,
                cudaStream_t st)
{
  piko_batch* b = nullptr;
  if (batch_make(ctx, scenes.data(), (int)scenes.size(), cfgs.data(), &b) != PIKO_OK) return -1.0f;
  float result = -1.0f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::vector<float> ms;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) goto done;
  // the first frame sizes the queues (an overflow grows them and redraws)
  for (int w = 0; w < 2; ++w) {
    if (piko_batch_run(b, st, 1) != PIKO_OK || piko_batch_finish(b, nullptr) != PIKO_OK) goto done;
  }
  for (int i = 0; i < reps; ++i) {
    if (cudaEventRecord(e0, st) != cudaSuccess) goto done;
    if (piko_batch_run(b, st, 1) != PIKO_OK) goto done;
    if (cudaEventRecord(e1, st) != cudaSuccess) goto done;
    if (piko_batch_finish(b, nullptr) != PIKO_OK) goto done;
    float t = 0.0f;
    if (cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) goto done;
    ms.push_back(t);
  }
  std::sort(ms.begin(), ms.end());
  result = ms[ms.size() / 2];
done:
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  piko_batch_destroy(b);
  return result;
}

float time_cfg(piko_ctx* ctx, const std::vector<piko_scene*>& scenes, const TuneCfg& cfg, int reps, cudaStream_t st)
{
  return time_cfgs(ctx, scenes, std::vector<TuneCfg>(scenes.size(), cfg), reps, st);
}

}  // namespace

extern "C" {

int piko_tune_bucket(int width, int height, int triangles) { return tune_bucket(width, height, triangles); }

piko_status piko_tuner_create(piko_tuner** out)
{
  if (!out) return PIKO_ERR_INVALID;
  *out = new piko_tuner();
  return PIKO_OK;
}

piko_status piko_tuner_destroy(piko_tuner* t)
{
  if (!t) return PIKO_ERR_INVALID;
  delete t;
  return PIKO_OK;
}

piko_status piko_tuner_get(const piko_tuner* t, int bucket, piko_tune_cfg* out)
{
  if (!t || !out || bucket < 0 || bucket >= kTuneBuckets) return PIKO_ERR_INVALID;
  const TuneCfg& c = t->cfg[bucket];
  out->tile_px = c.tile;
  out->ctas_per_sm = c.ctas_per_sm;
  out->chunk_entries = (int)c.chunk;
  out->ms = t->ms[bucket];
  out->tuned = t->tuned[bucket] ? 1 : 0;
  return PIKO_OK;
}

piko_status piko_tuner_set(piko_tuner* t, int bucket, const piko_tune_cfg* in)
{
  if (!t || !in || bucket < 0 || bucket >= kTuneBuckets) return PIKO_ERR_INVALID;
  if (in->tile_px != 8 && in->tile_px != 16 && in->tile_px != 32) return PIKO_ERR_INVALID;
  if (in->ctas_per_sm < 0 || in->ctas_per_sm > 32 || in->chunk_entries < 0 || in->chunk_entries > 4096)
    return PIKO_ERR_INVALID;
  t->cfg[bucket] = TuneCfg{in->tile_px, in->ctas_per_sm, (uint32_t)in->chunk_entries};
  t->ms[bucket] = in->ms;
  t->tuned[bucket] = in->tuned != 0;
  return PIKO_OK;
}

piko_status piko_tuner_tune(piko_tuner* t, piko_ctx* ctx, piko_scene* const* scenes, int n, int reps)
{
  if (!t || !ctx || !scenes || n <= 0) return PIKO_ERR_INVALID;
  if (reps <= 0) reps = 5;
  std::vector<piko_scene*> by[kTuneBuckets];
  for (int i = 0; i < n; ++i) {
    if (!scenes[i] || scenes[i]->pipe->kind != kPipeRaster)
      return set_err(ctx, PIKO_ERR_UNSUPPORTED, "%s", "the tuner takes raster scenes");
    by[tune_bucket(scenes[i]->W, scenes[i]->H, scenes[i]->N)].push_back(scenes[i]);
  }
  cudaStream_t st = ctx->stream;
  constexpr int kNC = (int)(sizeof(kCandidates) / sizeof(kCandidates[0]));
  float bucket_ms[kTuneBuckets][kNC] = {};
  for (int k = 0; k < kTuneBuckets; ++k) {
    if (by[k].empty()) continue;
    float best = -1.0f;
    TuneCfg best_cfg = t->cfg[k];
    for (int c = 0; c < kNC; ++c) {
      const float ms = time_cfg(ctx, by[k], kCandidates[c], reps, st);
      if (ms < 0.0f) return set_err(ctx, PIKO_ERR_CUDA, "%s", "tuner: a candidate configuration failed");
      bucket_ms[k][c] = ms;
      if (best < 0.0f || ms < best) { best = ms; best_cfg = kCandidates[c]; }
    }
    t->cfg[k] = best_cfg;
    t->ms[k] = best;
    t->tuned[k] = true;
  }
  // The buckets' groups run side by side in the tuned batch and compete for
  // the GPU, so the per-bucket choice is checked on the whole mix against
  // every candidate used for all of it.  A mixed table is kept only if it
  // beats the fastest single configuration by more than kMixedMargin (the
  // timings carry a few percent of noise, and one group -- one launch
  // sequence over one global tile queue -- is the simpler batch).
  std::vector<piko_scene*> all(scenes, scenes + n);
  auto table_cfgs = [&](const TuneCfg* tab) {
    std::vector<TuneCfg> c((size_t)n);
    for (int i = 0; i < n; ++i) c[i] = tab[tune_bucket(scenes[i]->W, scenes[i]->H, scenes[i]->N)];
    return c;
  };
  const float table_ms = time_cfgs(ctx, all, table_cfgs(t->cfg), reps, st);
  if (table_ms < 0.0f) return set_err(ctx, PIKO_ERR_CUDA, "%s", "tuner: the tuned table failed");
  int best_single = -1;
  float single_ms = 0.0f;
  for (int c = 0; c < kNC; ++c) {
    const float ms = time_cfg(ctx, all, kCandidates[c], reps, st);
    if (ms < 0.0f) return set_err(ctx, PIKO_ERR_CUDA, "%s", "tuner: a candidate configuration failed");
    if (best_single < 0 || ms < single_ms) { single_ms = ms; best_single = c; }
  }
  constexpr float kMixedMargin = 0.03f;
  if (table_ms < single_ms * (1.0f - kMixedMargin)) best_single = -1;   // the mixed table wins clearly
  if (best_single >= 0) {
    for (int k = 0; k < kTuneBuckets; ++k) {
      if (by[k].empty()) continue;
      t->cfg[k] = kCandidates[best_single];
      t->ms[k] = bucket_ms[k][best_single];
    }
  }
  return PIKO_OK;
}

piko_status piko_batch_create_tuned(piko_ctx* ctx, piko_scene* const* scenes, int n, const piko_tuner* t,
                                    piko_batch** out)
{
  if (!ctx || !scenes || n <= 0 || !t || !out) return PIKO_ERR_INVALID;
  *out = nullptr;
  std::vector<TuneCfg> cfgs((size_t)n);
  for (int i = 0; i < n; ++i) {
    if (!scenes[i] || scenes[i]->pipe->kind != kPipeRaster)
      return set_err(ctx, PIKO_ERR_UNSUPPORTED, "%s", "batches hold raster scenes");
    cfgs[i] = t->cfg[tune_bucket(scenes[i]->W, scenes[i]->H, scenes[i]->N)];
  }
  return batch_make(ctx, scenes, n, cfgs.data(), out);
}

}  // extern "C"
