// Served form: a render-request loop with continuous batching (no counterpart in
// the reference, which renders one scene per run_single call).
//
// Requests name a resident mesh (a piko_scene: triangles or patches already in
// HBM), a camera state and whether the caller wants the image back.  A worker
// thread
//   * admits queued requests in arrival order into output slots (framebuffer +
//     depth buffer), allocating a new slot only while the HBM budget allows;
//   * packs whatever is admitted into one launch sequence per free "lane" (a
//     CUDA stream with its own bin-queue scratch): every raster request of the
//     batch becomes one draw of a single multi-scene raster launch, every
//     Reyes request gets its own split/dice/shade sequence on the same stream;
//   * keeps up to `lanes` batches in flight, so requests that arrive while
//     others are on the GPU are launched as soon as a lane is free and overlap
//     with them on the device;
//   * retires a lane when its event completes, recording each request's latency
//     (submit to completion, host clock).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "runtime_internal.h"

namespace {

double now_s()
{
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct SrvRequest {
  uint64_t id = 0;
  piko_scene* mesh = nullptr;
  piko_const_state state{};
  bool keep = false;
  double t_submit = 0, t_done = 0;
  int slot = -1;
  int phase = 0;  // 0 queued, 1 running, 2 done, 3 failed
  piko_status status = PIKO_OK;
};

struct SrvSlot {
  uint32_t* fb = nullptr;
  float* depth = nullptr;
  size_t pixels = 0;
  bool busy = false;
  piko_scene* shadow = nullptr;  // Reyes requests: a scene view sharing the mesh's patches
};

struct SrvLane {
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;
  bool busy = false;
  std::vector<uint64_t> reqs;
  std::map<int, RasterScratch> scr;          // per raster tile size
  std::map<int, std::vector<RasterDraw>> draws;
  std::vector<piko_const_state> states;      // stable storage for the draws' states
  std::vector<int> reyes_slots;
  ReyesState* reyes_buf = nullptr;           // Reyes work buffers of this lane's requests
};

}  // namespace

struct piko_server {
  piko_ctx* ctx = nullptr;
  piko_server_opts opts{};
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::atomic<bool> stop{false};
  std::deque<uint64_t> queue;
  std::unordered_map<uint64_t, SrvRequest> reqs;
  std::vector<SrvSlot> slots;
  std::vector<SrvLane> lanes;
  uint64_t next_id = 1;
  size_t hbm_used = 0;
  std::unordered_map<const piko_scene*, size_t> meshes;
  // statistics since the last reset
  std::vector<double> latencies_ms;
  uint64_t submitted = 0, completed = 0, failed = 0, batches = 0, batched_reqs = 0;
  double first_submit = 0, last_done = 0;
  cudaStream_t io = nullptr;
};

namespace {

size_t mesh_bytes(const piko_scene* s)
{
  const size_t n = (size_t)s->N;
  if (s->kind == PIKO_SCENE_TRIANGLES)
    return n * 3 * ((s->packed ? 12 : 16) * 2 + (s->col ? 16 : 0) + (s->uv ? 8 : 0)) + (size_t)s->tex_w * s->tex_h * 4;
  if (s->kind == PIKO_SCENE_WTRI) return n * 48;
  if (s->kind == PIKO_SCENE_WTRI_WORLD) return n * 36;
  return n * 256;
}

size_t scratch_bytes(const RasterScratch& r)
{
  // setup records, per-tile counters and offsets, tile lists and the count
  // passes' pair records (12 bytes per list entry)
  return (size_t)r.tris_cap * sizeof(TriSetup) + (size_t)r.tiles_cap * 8 + (size_t)r.list_cap * 16;
}

// slot with room for `pixels`, allocating one within the budget; -1 if none
int acquire_slot(piko_server* sv, size_t pixels)
{
  int best = -1;
  for (int i = 0; i < (int)sv->slots.size(); ++i)
    if (!sv->slots[i].busy && sv->slots[i].pixels >= pixels && (best < 0 || sv->slots[i].pixels < sv->slots[best].pixels))
      best = i;
  if (best >= 0) {
    sv->slots[best].busy = true;
    return best;
  }
  if ((int)sv->slots.size() >= sv->opts.max_slots) return -1;
  const size_t alloc_px = std::max(pixels, (size_t)sv->opts.max_pixels);
  const size_t bytes = alloc_px * 8;
  if (sv->hbm_used + bytes > sv->opts.hbm_budget_bytes) return -1;
  SrvSlot s;
  if (dalloc(&s.fb, alloc_px) != cudaSuccess || dalloc(&s.depth, alloc_px) != cudaSuccess) {
    dfree(s.fb);
    dfree(s.depth);
    return -1;
  }
  s.pixels = alloc_px;
  s.busy = true;
  sv->hbm_used += bytes;
  sv->slots.push_back(s);
  return (int)sv->slots.size() - 1;
}

piko_scene* reyes_view(SrvSlot& slot, piko_scene* mesh, const piko_const_state& st)
{
  if (!slot.shadow) slot.shadow = new piko_scene();
  piko_scene* v = slot.shadow;
  v->pipe = mesh->pipe;
  v->kind = mesh->kind;
  v->W = mesh->W; v->H = mesh->H; v->N = mesh->N;
  v->patches = mesh->patches;
  v->fb = slot.fb;
  v->depth = slot.depth;
  v->state = st;
  return v;
}

void release_view(SrvSlot& slot)
{
  if (!slot.shadow) return;
  piko_reyes_release(slot.shadow);
  slot.shadow->patches = nullptr;  // borrowed from the mesh
  delete slot.shadow;
  slot.shadow = nullptr;
}

// Takes queued requests into a lane and enqueues them.  Called with the lock
// held; releases it around the CUDA calls.
bool dispatch(piko_server* sv, SrvLane& lane, std::unique_lock<std::mutex>& lk)
{
  lane.reqs.clear();
  lane.draws.clear();
  lane.states.clear();
  lane.reyes_slots.clear();
  std::vector<uint64_t> taken;
  while (!sv->queue.empty() && (int)taken.size() < sv->opts.max_batch) {
    SrvRequest& r = sv->reqs[sv->queue.front()];
    const int slot = acquire_slot(sv, (size_t)r.mesh->W * r.mesh->H);
    if (slot < 0) break;  // admission: wait for a slot or budget to free up
    r.slot = slot;
    r.phase = 1;
    taken.push_back(r.id);
    sv->queue.pop_front();
  }
  if (taken.empty()) return false;
  lane.reqs = taken;
  lane.states.reserve(taken.size());
  for (uint64_t id : taken) {
    SrvRequest& r = sv->reqs[id];
    SrvSlot& sl = sv->slots[r.slot];
    lane.states.push_back(r.state);
    if (r.mesh->pipe->kind == kPipeRaster) {
      lane.draws[r.mesh->pipe->tile].push_back(RasterDraw{r.mesh, &lane.states.back(), sl.fb, sl.depth});
    } else {
      reyes_view(sl, r.mesh, r.state);
      if (!lane.reyes_buf) lane.reyes_buf = reyes_buffers_new();
      reyes_borrow_buffers(sl.shadow, lane.reyes_buf);
      lane.reyes_slots.push_back(r.slot);
    }
  }
  lane.busy = true;
  sv->batches++;
  sv->batched_reqs += taken.size();
  lk.unlock();
  piko_status st = PIKO_OK;
  for (auto& kv : lane.draws) {
    const int T = kv.first;
    const int cps = kv.second.front().mesh->pipe->ctas_per_sm;
    piko_status r = enqueue_raster_draws(sv->ctx, kv.second.data(), (int)kv.second.size(), lane.scr[T], T,
                                         raster_ctas(sv->ctx, T, cps), lane.st, false, false,
                                         kv.second.front().mesh->pipe->chunk);
    if (r != PIKO_OK) st = r;
  }
  for (int si : lane.reyes_slots) {
    piko_status r = piko_reyes_run(sv->slots[si].shadow, lane.st, false);
    sv->slots[si].shadow->last_stream = lane.st;
    sv->slots[si].shadow->pending = true;
    if (r != PIKO_OK) st = r;
  }
  cudaEventRecord(lane.ev, lane.st);
  lk.lock();
  if (st != PIKO_OK)
    for (uint64_t id : taken) sv->reqs[id].status = st;
  return true;
}

// Checks a completed lane's frames, re-rendering after a queue overflow (and
// waiting for the re-render), and returns the lane's status: a CUDA error, a
// scan timeout, queues that kept overflowing, or a Reyes frame's error.
// Called without the lock.
piko_status finish_lane(piko_server* sv, SrvLane& lane)
{
  piko_status result = PIKO_OK;
  for (auto& kv : lane.draws) {
    RasterScratch& scr = lane.scr[kv.first];
    piko_status st = PIKO_ERR_QUEUE_OVERFLOW;
    for (int attempt = 0; attempt < 5; ++attempt) {
      cudaError_t e = cudaMemcpyAsync(scr.h_ctr, scr.ctr, sizeof(FrameCounters), cudaMemcpyDeviceToHost, lane.st);
      if (!e) e = cudaStreamSynchronize(lane.st);
      if (e) { st = PIKO_ERR_CUDA; break; }
      const uint32_t status = scr.h_ctr->status;
      if (status & kStatusScanTimeout) { st = PIKO_ERR_TIMEOUT; break; }
      if (!(status & kStatusListOverflow)) { st = PIKO_OK; break; }
      if (attempt == 4) break;   // still overflowing: reported
      if (scr.regrow(*scr.h_ctr) != cudaSuccess) { st = PIKO_ERR_OOM; break; }
      const int cps = kv.second.front().mesh->pipe->ctas_per_sm;
      const piko_status r = enqueue_raster_draws(sv->ctx, kv.second.data(), (int)kv.second.size(), scr, kv.first,
                                                 raster_ctas(sv->ctx, kv.first, cps), lane.st, false, false,
                                                 kv.second.front().mesh->pipe->chunk);
      if (r != PIKO_OK) { st = r; break; }
    }
    if (st != PIKO_OK && result == PIKO_OK) result = st;
  }
  for (int si : lane.reyes_slots) {
    const piko_status r = piko_reyes_finish(sv->slots[si].shadow);
    if (r != PIKO_OK && result == PIKO_OK) result = r;
  }
  return result;
}

void worker_loop(piko_server* sv)
{
  cudaSetDevice(sv->ctx->device);
  std::unique_lock<std::mutex> lk(sv->mu);
  while (!sv->stop.load()) {
    bool progress = false;
    for (auto& lane : sv->lanes) {
      if (!lane.busy) continue;
      lk.unlock();
      const cudaError_t q = cudaEventQuery(lane.ev);
      const piko_status fin = q == cudaSuccess ? finish_lane(sv, lane) : PIKO_OK;
      const double t = now_s();
      lk.lock();
      if (q == cudaErrorNotReady) continue;
      for (uint64_t id : lane.reqs) {
        SrvRequest& r = sv->reqs[id];
        r.t_done = t;
        if (q != cudaSuccess && r.status == PIKO_OK) r.status = PIKO_ERR_CUDA;
        if (fin != PIKO_OK && r.status == PIKO_OK) r.status = fin;
        r.phase = r.status == PIKO_OK ? 2 : 3;
        if (r.phase == 2) {
          sv->completed++;
          sv->latencies_ms.push_back((r.t_done - r.t_submit) * 1e3);
          sv->last_done = std::max(sv->last_done, t);
        } else {
          sv->failed++;
        }
        if (!r.keep) {
          sv->slots[r.slot].busy = false;
          sv->reqs.erase(id);
        }
      }
      lane.busy = false;
      lane.reqs.clear();
      progress = true;
      sv->cv_done.notify_all();
    }
    for (auto& lane : sv->lanes) {
      if (lane.busy || sv->queue.empty()) continue;
      if (dispatch(sv, lane, lk)) progress = true;
    }
    if (!progress) sv->cv_work.wait_for(lk, std::chrono::microseconds(sv->opts.poll_us));
  }
}

}  // namespace

extern "C" {

piko_status piko_server_create(piko_ctx* ctx, const piko_server_opts* opts, piko_server** out)
{
  if (!ctx || !out) return PIKO_ERR_INVALID;
  *out = nullptr;
  piko_server* sv = new piko_server();
  sv->ctx = ctx;
  piko_server_opts o{};
  if (opts) o = *opts;
  if (!o.hbm_budget_bytes) o.hbm_budget_bytes = (size_t)120 << 30;
  if (o.max_slots <= 0) o.max_slots = 256;
  if (o.max_batch <= 0) o.max_batch = 64;
  if (o.lanes <= 0) o.lanes = 3;
  if (o.max_pixels <= 0) o.max_pixels = 1920 * 1080;
  if (o.poll_us <= 0) o.poll_us = 20;
  sv->opts = o;
  cudaSetDevice(ctx->device);
  sv->lanes.resize((size_t)o.lanes);
  for (auto& l : sv->lanes) {
    if (cudaStreamCreateWithFlags(&l.st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&l.ev, cudaEventDisableTiming) != cudaSuccess) {
      delete sv;
      return set_err(ctx, PIKO_ERR_CUDA, "%s", "server stream creation failed");
    }
  }
  cudaStreamCreateWithFlags(&sv->io, cudaStreamNonBlocking);
  sv->worker = std::thread(worker_loop, sv);
  *out = sv;
  return PIKO_OK;
}

piko_status piko_server_submit(piko_server* sv, piko_scene* mesh, const piko_const_state* state, int keep_result,
                               uint64_t* request_id)
{
  if (!sv || !mesh || !state) return PIKO_ERR_INVALID;
  if (state->light_mode != 0 && state->light_mode != 1) return PIKO_ERR_INVALID;
  const double t = now_s();
  std::lock_guard<std::mutex> lk(sv->mu);
  SrvRequest r;
  r.id = sv->next_id++;
  r.mesh = mesh;
  r.state = *state;
  r.keep = keep_result != 0;
  r.t_submit = t;
  if (sv->submitted == 0 || t < sv->first_submit) sv->first_submit = t;
  sv->submitted++;
  if (!sv->meshes.count(mesh)) {
    const size_t b = mesh_bytes(mesh);
    sv->meshes[mesh] = b;
    sv->hbm_used += b;
  }
  sv->reqs[r.id] = r;
  sv->queue.push_back(r.id);
  if (request_id) *request_id = r.id;
  sv->cv_work.notify_one();
  return PIKO_OK;
}

piko_status piko_server_wait(piko_server* sv, uint64_t id, int timeout_ms)
{
  if (!sv) return PIKO_ERR_INVALID;
  std::unique_lock<std::mutex> lk(sv->mu);
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
  for (;;) {
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return PIKO_OK;  // done and not kept
    if (it->second.phase >= 2) return it->second.status;
    if (sv->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
      it = sv->reqs.find(id);
      if (it == sv->reqs.end()) return PIKO_OK;
      if (it->second.phase >= 2) return it->second.status;
      return PIKO_ERR_TIMEOUT;
    }
  }
}

piko_status piko_server_drain(piko_server* sv, int timeout_ms)
{
  if (!sv) return PIKO_ERR_INVALID;
  std::unique_lock<std::mutex> lk(sv->mu);
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
  for (;;) {
    bool busy = !sv->queue.empty();
    for (auto& l : sv->lanes) busy = busy || l.busy;
    if (!busy) return PIKO_OK;
    if (sv->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) return PIKO_ERR_TIMEOUT;
  }
}

piko_status piko_server_read(piko_server* sv, uint64_t id, uint32_t* rgba, float* depth)
{
  if (!sv) return PIKO_ERR_INVALID;
  piko_status st = piko_server_wait(sv, id, 60000);
  if (st != PIKO_OK) return st;
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(id);
  if (it == sv->reqs.end()) return set_err(sv->ctx, PIKO_ERR_INVALID, "%s", "request was not kept or already read");
  SrvRequest r = it->second;
  SrvSlot& sl = sv->slots[r.slot];
  const size_t n = (size_t)r.mesh->W * r.mesh->H;
  lk.unlock();
  cudaError_t e = cudaSuccess;
  if (rgba) e = cudaMemcpyAsync(rgba, sl.fb, n * 4, cudaMemcpyDeviceToHost, sv->io);
  if (!e && depth) e = cudaMemcpyAsync(depth, sl.depth, n * 4, cudaMemcpyDeviceToHost, sv->io);
  if (!e) e = cudaStreamSynchronize(sv->io);
  lk.lock();
  sv->slots[r.slot].busy = false;
  sv->reqs.erase(id);
  sv->cv_work.notify_one();
  if (e) return set_err(sv->ctx, PIKO_ERR_CUDA, "%s", cudaGetErrorString(e));
  return PIKO_OK;
}

piko_status piko_server_stats_get(piko_server* sv, piko_server_stats* o)
{
  if (!sv || !o) return PIKO_ERR_INVALID;
  memset(o, 0, sizeof(*o));
  std::lock_guard<std::mutex> lk(sv->mu);
  o->submitted = sv->submitted;
  o->completed = sv->completed;
  o->failed = sv->failed;
  o->batches = sv->batches;
  o->mean_batch = sv->batches ? (double)sv->batched_reqs / (double)sv->batches : 0.0;
  o->span_s = sv->completed ? sv->last_done - sv->first_submit : 0.0;
  size_t scratch = 0;
  for (auto& l : sv->lanes)
    for (auto& kv : l.scr) scratch += scratch_bytes(kv.second);
  o->hbm_bytes = sv->hbm_used + scratch;
  o->slots = (uint32_t)sv->slots.size();
  if (!sv->latencies_ms.empty()) {
    std::vector<double> v = sv->latencies_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) {
      const size_t k = (size_t)std::min<double>((double)v.size() - 1, std::ceil(p * v.size()) - 1);
      return v[k];
    };
    o->p50_ms = pct(0.50);
    o->p99_ms = pct(0.99);
    o->max_ms = v.back();
    double s = 0;
    for (double x : v) s += x;
    o->mean_ms = s / (double)v.size();
  }
  return PIKO_OK;
}

piko_status piko_server_reset_stats(piko_server* sv)
{
  if (!sv) return PIKO_ERR_INVALID;
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->latencies_ms.clear();
  sv->submitted = sv->completed = sv->failed = sv->batches = sv->batched_reqs = 0;
  sv->first_submit = sv->last_done = 0;
  return PIKO_OK;
}

piko_status piko_server_destroy(piko_server* sv)
{
  if (!sv) return PIKO_ERR_INVALID;
  piko_server_drain(sv, 60000);
  sv->stop.store(true);
  sv->cv_work.notify_all();
  if (sv->worker.joinable()) sv->worker.join();
  for (auto& l : sv->lanes) {
    if (l.st) cudaStreamSynchronize(l.st);
    for (auto& kv : l.scr) kv.second.release();
    if (l.ev) cudaEventDestroy(l.ev);
    if (l.st) cudaStreamDestroy(l.st);
  }
  for (auto& s : sv->slots) {
    release_view(s);
    dfree(s.fb);
    dfree(s.depth);
  }
  for (auto& l : sv->lanes) reyes_buffers_free(l.reyes_buf);
  if (sv->io) cudaStreamDestroy(sv->io);
  delete sv;
  return PIKO_OK;
}

}  // extern "C"
