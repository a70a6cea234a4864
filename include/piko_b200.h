/*
 * piko_b200.h - C ABI of libpiko_b200.so: Piko's binned raster and Reyes
 * pipelines on one B200 (sm_100a).
 *
 * The reference's real boundary is source level: a pipeline is a C++ class
 * derived from PikoPipe whose Stage<binX, binY, threadsPerTile, In, Out>
 * members are wired with pikoConnect (pikoc/api/include/piko/pipe.h:8-15,
 * pikoc/api/include/piko/stage.h:138-391), and pikoc generates the host methods
 * allocate / prepare / run_single / destroy plus PikoScreen::getData
 * (pikoc/src/Backend/CPUBackend.cpp:272-571, pikoc/src/Backend/PTXBackend.cpp:741-1026).
 * Each entry point below names the reference method it replaces.
 *
 * Conventions: every call returns a piko_status; nothing calls exit() (the
 * reference's CUDACHECK does, pikoc/api/include/internal/cudaMacros.h:10-20).
 * Buffers passed in are caller-owned and copied; handles are library-owned.
 * One context per host thread, or external locking.  `stream` arguments are
 * cudaStream_t values passed as void* (NULL = the scene's own stream).
 * Device-side waits are bounded and report PIKO_ERR_TIMEOUT.
 */
#ifndef PIKO_B200_H
#define PIKO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum piko_status {
  PIKO_OK = 0,
  PIKO_ERR_INVALID = 1,        /* bad argument or descriptor */
  PIKO_ERR_OOM = 2,            /* device allocation failed */
  PIKO_ERR_QUEUE_OVERFLOW = 3, /* a bin queue outgrew its capacity (retried internally) */
  PIKO_ERR_TIMEOUT = 4,        /* a bounded device-side wait gave up */
  PIKO_ERR_CUDA = 5,           /* CUDA runtime error; see piko_last_error */
  PIKO_ERR_UNSUPPORTED = 6,    /* pipeline shape this build does not implement */
  PIKO_ERR_NO_DEVICE = 7,      /* no CUDA device */
  PIKO_ERR_LIMIT = 8           /* request beyond a fixed limit of the allocation-free entry point */
} piko_status;

typedef struct piko_ctx piko_ctx;
typedef struct piko_pipe piko_pipe;
typedef struct piko_scene piko_scene;
typedef struct piko_batch piko_batch;

/* ------------------------------------------------------------------ context */
typedef struct piko_ctx_opts {
  int device;        /* CUDA device ordinal */
  int time_kernels;  /* record CUDA events between the kernels of a frame */
} piko_ctx_opts;

/* Creates a context on opts->device (NULL opts = device 0, no timing). */
piko_status piko_ctx_create(const piko_ctx_opts* opts, piko_ctx** out);
piko_status piko_ctx_destroy(piko_ctx* ctx);
/* Last error message of this context (static storage, never NULL). */
const char* piko_last_error(const piko_ctx* ctx);
/* Library version string. */
const char* piko_version(void);

/* ------------------------------------------------------------------ pipeline
 * A pipeline descriptor is the compiled-in equivalent of the reference's
 * PikoPipe class: the Stage<> template arguments of each stage and the
 * pikoConnect calls of the constructor (rasterPipe.h:16-38, reyesPipe.h:12-32).
 * Bin size 0 means one full-screen bin (pikoc/include/PikoSummary.hpp:279). */
typedef enum piko_prim {
  PIKO_PRIM_RASTER_WTRI = 1, /* raster_wtri  (basicTypes/rasterTypes.h:8-34) */
  PIKO_PRIM_RASTER_STRI = 2, /* raster_stri  (basicTypes/rasterTypes.h:36-71) */
  PIKO_PRIM_PIXEL = 3,       /* Pixel        (piko/builtinTypes.h:52-72) */
  PIKO_PRIM_PATCH = 4,       /* piko_patch   (reyesPipe/pikoTypes.h:65-73) */
  PIKO_PRIM_UPOLY = 5        /* piko_upoly   (reyesPipe/pikoTypes.h:75-79) */
} piko_prim;

typedef struct piko_stage_desc {
  int bin_size_x, bin_size_y, threads_per_tile; /* Stage<binX, binY, threadsPerTile, ...> */
  int in_prim, out_prim;                        /* piko_prim */
} piko_stage_desc;

typedef struct piko_link {
  int out_stage, in_stage, out_port, in_port;   /* pikoConnect(out, in, outPort, inPort) */
} piko_link;

#define PIKO_MAX_STAGES 8

typedef struct piko_pipe_desc {
  int n_stages;
  piko_stage_desc stages[PIKO_MAX_STAGES];
  int n_links;
  piko_link links[PIKO_MAX_STAGES];
  /* device tuning, no counterpart in the reference (0 = default) */
  int tile_px;          /* raster tile edge: 8 (default), 16 or 32 pixels (Reyes shades per
                           micropolygon and ignores it) */
  int ctas_per_sm;      /* persistent raster CTAs per SM */
  /* Reyes constants the reference hard-codes (0 = the reference's value):
   * THRESHOLD_PIXELS 4.0f and the 20-split limit (split.pikostage:12,284), and
   * a fixed dice grid instead of the extent-derived nu, nv (split.pikostage:307-316),
   * 1..32 like the derived grids (larger values are PIKO_ERR_INVALID) */
  float split_threshold_px;
  int max_splits;
  int dice_grid;
  /* device tuning: list entries per work item of the 8x8 raster tile queue; a
   * tile with a longer list is split over several warps (0 = 32) */
  int chunk_entries;
  /* Reyes sampling and shading variants, no reference counterpart (0 = the
   * reference: one sample at the pixel centre, corners lit and averaged).
   * samples_per_pixel 4: one jittered sample per pixel quadrant, positions
   * from sample_seed; each sample has the reference's coverage test and depth
   * order, and a pixel takes the rounded mean of its samples' colours and its
   * nearest sample's depth.  phong 1: the micropolygon's corner normals are
   * interpolated to its centre and lit once (Phong) instead of lit per corner
   * and averaged (Gouraud). */
  int samples_per_pixel;   /* 0 or 1, or 4 */
  uint32_t sample_seed;
  int phong;
} piko_pipe_desc;

/* Fills desc with the reference's RasterPipe: VertexShaderStage<32,32,512,
 * raster_wtri, raster_stri> -> RasterStage<8,8,32, raster_stri, Pixel>. */
void piko_pipe_desc_raster(piko_pipe_desc* desc);
/* Fills desc with the reference's ReyesPipe: SplitStage<0,0,256> (self loop on
 * port 1) -> DiceStage<64,64,128> -> ShadeStage<64,64,512>. */
void piko_pipe_desc_reyes(piko_pipe_desc* desc);

/* Replaces the PikoPipe constructor + pikoConnect (pipe.h:8-12).
 * PIKO_ERR_UNSUPPORTED for shapes other than the two pipelines above. */
piko_status piko_pipe_create(piko_ctx* ctx, const piko_pipe_desc* desc, piko_pipe** out);
piko_status piko_pipe_destroy(piko_pipe* pipe);

/* ------------------------------------------------------------------ scenes */
typedef enum piko_scene_kind {
  PIKO_SCENE_TRIANGLES = 1, /* world-space SoA attributes; vertex shading on device */
  PIKO_SCENE_WTRI = 2,      /* the reference's pre-transformed raster_wtri payload */
  PIKO_SCENE_PATCHES = 3,   /* bicubic Bezier patches (Reyes) */
  PIKO_SCENE_WTRI_WORLD = 4 /* the raster_wtri payload of the pipe built without
                               VTX_PRETRANSFORM (rasterPipe.h:7 removed): world
                               positions that the vertex stage transforms with the
                               frame's view_proj (vtxTransform, rasterMacros.h:14-21;
                               vertexShader.pikostage:56-80).  The reference sets no
                               vertex colours in that mode; here they are 0, so
                               drawn pixels are 0xff000000 (coverage and depth are
                               the reference's) */
} piko_scene_kind;

typedef struct piko_scene_desc {
  int width, height;       /* framebuffer size (>= 32 x 32) */
  int kind;                /* piko_scene_kind */
  int count;               /* triangles or patches */
  /* PIKO_SCENE_TRIANGLES: float4 [3][count] per attribute, vertex slot major */
  const float* pos;        /* x, y, z, (w ignored) */
  const float* nrm;        /* normal x, y, z */
  const float* col;        /* material colour r, g, b; NULL: every vertex takes
                              the reference's fixed material colour (0.9, 0.9,
                              0.6), main.cpp:380-386, and nothing is uploaded */
  const float* uv;         /* optional float2 [3][count]: textured variant */
  const uint8_t* texture;  /* optional RGBA8 [tex_h][tex_w], power-of-two sides */
  int tex_w, tex_h;
  /* PIKO_SCENE_WTRI: screen x, y, z of 3 vertices [count][9] and ABGR colours
   * [count][3] (raster_wtri worldPos0..2, icol0..2 under VTX_PRETRANSFORM).
   * PIKO_SCENE_WTRI_WORLD: world x, y, z of 3 vertices [count][9] in
   * wtri_xyz; wtri_icol unused */
  const float* wtri_xyz;
  const uint32_t* wtri_icol;
  /* PIKO_SCENE_PATCHES: 16 float4 control points per patch [count][16][4] */
  const float* patches;
  /* PIKO_SCENE_TRIANGLES: nonzero = pos and nrm are float3 [3][count] (x, y, z;
   * 12 bytes per vertex) instead of float4: a quarter fewer bytes to upload,
   * the same image.  Kept for the life of the scene (uploads must match). */
  int packed;
} piko_scene_desc;

/* Replaces RasterPipe::allocate / ReyesPipe::allocate (CPUBackend.cpp:272-350):
 * copies the inputs to device memory and allocates the framebuffer, depth
 * buffer and bin queues. */
piko_status piko_scene_create(piko_pipe* pipe, const piko_scene_desc* desc, piko_scene** out);
/* Re-uploads the inputs of an existing scene (same kind and count), async on
 * stream; the host buffers must stay valid until the stream reaches it. */
piko_status piko_scene_upload(piko_scene* scene, const piko_scene_desc* desc, void* stream);
/* Replaces destroy() (CPUBackend.cpp:400-426). */
piko_status piko_scene_destroy(piko_scene* scene);

/* ConstantState (piko/builtinTypes.h:20-33) plus the lighting inputs of the
 * host pre-transform (main.cpp:358-392).  light_mode 0: light[] is the light
 * vector of every vertex; 1: light vector = normalize(eye - vertex). */
typedef struct piko_const_state {
  float view_proj[16]; /* column-major: clip.x = m[0]x + m[4]y + m[8]z + m[12] */
  int light_mode;
  float light[3];
  float eye[3];
} piko_const_state;

/* Replaces prepare() (CPUBackend.cpp:366-379): the state used by the next
 * frames.  The depth buffer is reset to 1.0f and the colour buffer to
 * 0xff663313 at the start of every frame. */
piko_status piko_frame_prepare(piko_scene* scene, const piko_const_state* state);
/* Replaces run_single() (CPUBackend.cpp:381-398): enqueues one frame on
 * `stream` and returns without waiting. */
piko_status piko_frame_run(piko_scene* scene, void* stream);
/* Waits for the scene's last frame and checks its status; a bin-queue
 * overflow grows the queues and re-renders the frame before returning OK. */
piko_status piko_frame_finish(piko_scene* scene);
/* Replaces pikoScreen.getData() (stage.h:108-117) and the depth buffer
 * readback: finishes the frame and copies W*H RGBA8 words (R in the low
 * byte, row 0 = bottom) and W*H floats; either pointer may be NULL. */
piko_status piko_frame_read(piko_scene* scene, uint32_t* rgba, float* depth);
/* Device pointers of the scene's framebuffer and depth buffer. */
piko_status piko_frame_device_buffers(piko_scene* scene, uint32_t** rgba, float** depth);

typedef struct piko_frame_stats {
  uint64_t prims_in;        /* triangles or patches submitted */
  uint64_t prims_kept;      /* triangles emitted by the vertex stage / Reyes leaves */
  uint64_t upolys;          /* Reyes micropolygons */
  uint64_t bin_entries;     /* raster: (primitive, tile) queue entries; Reyes: micropolygons
                               with more than 16 candidate pixels (shaded a warp each) */
  uint64_t covered;         /* covered samples (fragments) */
  uint64_t wrap_risk;       /* triangles whose edge values may wrap in int32 */
  uint32_t status;          /* device status bits of the last frame */
  uint32_t split_levels;    /* Reyes split levels run */
  int n_kernels;            /* entries of kernel_ms in use (time_kernels only) */
  float kernel_ms[8];       /* per-phase time of the last frame: raster [setup, scan,
                               scatter, tiles]; Reyes [split, dice + depth pass, key pass,
                               resolve pass] */
} piko_frame_stats;

/* Finishes the last frame and returns its counters. */
piko_status piko_frame_stats_get(piko_scene* scene, piko_frame_stats* out);

/* Parity support: re-renders the last prepared frame recording every covered
 * sample as (triangle index, pixel index); copies up to cap records and sets
 * *count to the total.  Order is unspecified. */
piko_status piko_frame_coverage(piko_scene* scene, uint32_t* tri, uint32_t* pix, uint64_t cap, uint64_t* count);

/* ------------------------------------------------------------------ batched form
 * Many raster scenes drawn by one set of launches over a global tile queue;
 * no reference counterpart (the reference renders one scene per run_single). */
piko_status piko_batch_create(piko_ctx* ctx, piko_scene* const* scenes, int n, piko_batch** out);
/* Enqueues one frame of every scene of the batch; capture=1 records the launch
 * sequence as a CUDA graph on first use and replays it afterwards. */
piko_status piko_batch_run(piko_batch* batch, void* stream, int use_graph);
/* Waits for the batch, checks the status (growing queues and re-rendering on
 * overflow) and returns the summed counters. */
piko_status piko_batch_finish(piko_batch* batch, piko_frame_stats* out);
piko_status piko_batch_destroy(piko_batch* batch);

/* ------------------------------------------------------------------ tuner
 * Launch-configuration tuner of the batched form; no reference counterpart
 * (the reference fixes bin sizes in the pipeline source).  Scenes fall into
 * PIKO_TUNE_BUCKETS buckets by resolution class (<= 256x256, <= 512x512,
 * <= 1280x720, larger) x triangle class (< 4K, < 16K, < 64K, more);
 * bucket = resolution_class * 4 + triangle_class.  Each bucket holds a tile
 * edge (8/16/32 px), persistent CTAs per SM (0 = occupancy) and 8x8-queue
 * chunk size (0 = 32).  Every configuration renders the identical image. */
#define PIKO_TUNE_BUCKETS 16
typedef struct piko_tuner piko_tuner;
typedef struct piko_tune_cfg {
  int tile_px;
  int ctas_per_sm;
  int chunk_entries;
  float ms;     /* median device time of the bucket's scenes when tuned */
  int tuned;    /* 1 once measured (or set) */
} piko_tune_cfg;

/* Bucket of a scene of width x height pixels and `triangles` triangles. */
int piko_tune_bucket(int width, int height, int triangles);
/* A tuner whose buckets all hold tile 8, occupancy CTAs, chunk 32 (untuned). */
piko_status piko_tuner_create(piko_tuner** out);
piko_status piko_tuner_destroy(piko_tuner* tuner);
piko_status piko_tuner_get(const piko_tuner* tuner, int bucket, piko_tune_cfg* out);
/* Sets one bucket (a saved table); PIKO_ERR_INVALID for other tile sizes or
 * out-of-range values. */
piko_status piko_tuner_set(piko_tuner* tuner, int bucket, const piko_tune_cfg* cfg);
/* Measures every candidate configuration on the scenes of each bucket present
 * in scenes[0..n) (as one batch, `reps` graph replays, median) and keeps the
 * fastest.  Synchronous; renders into the scenes' own buffers. */
piko_status piko_tuner_tune(piko_tuner* tuner, piko_ctx* ctx, piko_scene* const* scenes, int n, int reps);
/* A batch whose scenes are grouped by their bucket's configuration: one launch
 * sequence per group, the groups on parallel branches of the replayed graph. */
piko_status piko_batch_create_tuned(piko_ctx* ctx, piko_scene* const* scenes, int n, const piko_tuner* tuner,
                                    piko_batch** out);

/* ------------------------------------------------------------------ served form
 * A render-request loop with continuous batching; no reference counterpart.
 * A worker thread admits requests (a resident mesh = any piko_scene, a camera
 * state) into output slots against an HBM budget, batches whatever is queued
 * into one launch sequence per free stream lane, keeps several batches in
 * flight, and records each request's latency from submit to completion. */
typedef struct piko_server piko_server;

typedef struct piko_server_opts {
  size_t hbm_budget_bytes; /* slots + meshes + scratch (0 = 120 GiB) */
  int max_slots;           /* output slots (0 = 256) */
  int max_batch;           /* requests per launch sequence (0 = 64) */
  int lanes;               /* batches in flight on separate streams (0 = 3) */
  int max_pixels;          /* slot size in pixels (0 = 1920*1080; larger meshes get larger slots) */
  int poll_us;             /* worker idle wait (0 = 20 us) */
} piko_server_opts;

typedef struct piko_server_stats {
  uint64_t submitted, completed, failed, batches;
  double mean_batch;       /* requests per launch sequence */
  double p50_ms, p99_ms, mean_ms, max_ms;  /* submit-to-completion latency */
  double span_s;           /* first submit to last completion */
  uint64_t hbm_bytes;      /* slots + meshes + scratch held */
  uint32_t slots;
} piko_server_stats;

piko_status piko_server_create(piko_ctx* ctx, const piko_server_opts* opts, piko_server** out);
/* Queues one frame of `mesh` seen with `state`; keep_result=1 keeps the output
 * slot until piko_server_read.  Thread-safe. */
piko_status piko_server_submit(piko_server* server, piko_scene* mesh, const piko_const_state* state, int keep_result,
                               uint64_t* request_id);
/* Waits for one request (PIKO_ERR_TIMEOUT after timeout_ms). */
piko_status piko_server_wait(piko_server* server, uint64_t request_id, int timeout_ms);
/* Waits until every submitted request has completed. */
piko_status piko_server_drain(piko_server* server, int timeout_ms);
/* Copies a kept request's image and depth (W*H each) and frees its slot. */
piko_status piko_server_read(piko_server* server, uint64_t request_id, uint32_t* rgba, float* depth);
piko_status piko_server_stats_get(piko_server* server, piko_server_stats* out);
piko_status piko_server_reset_stats(piko_server* server);
piko_status piko_server_destroy(piko_server* server);

/* ------------------------------------------------------------------ scene and mesh files
 * Loaders without GL for the reference's `.scene` command files
 * (sceneParser/sceneParser.cpp:114-478: camera, camera_fov, zNear, zFar, light,
 * material, meshAttribute, translate, rotate, scale, reset, texture (ignored),
 * loadmesh, loadbez), its bezmesh `.dat` patches (bezmesh/bezmesh.cpp:23-150)
 * and Wavefront OBJ meshes, which replace the reference's assimp import (not
 * shipped).  Triangles are flattened as scene::flatten does
 * (basicTypes/scene.h:134-190): positions through the model transform in force
 * at their loadmesh, normals through its inverse transpose, unit length.
 * Host-side only; no device needed. */
typedef struct piko_asset piko_asset;
typedef struct piko_asset_info {
  int triangles, patches, has_uv, has_camera;
  float eye[3], target[3], up[3];   /* camera (defaults: (0,0,3) looking at the origin, y up) */
  float fovy_rad, znear, zfar;      /* defaults pi/3, 0.02, 100 (basicTypes/camera.h:40-45) */
  int lights, materials;
  float light_pos[3];               /* the first light's position */
} piko_asset_info;

/* Loads a .scene, .obj or .dat file.  Meshes named by a scene are looked up in
 * mesh_dir (NULL: the scene file's directory).  PIKO_ERR_INVALID with a
 * message in piko_asset_last_error() on a parse or file error. */
piko_status piko_asset_load(const char* path, const char* mesh_dir, piko_asset** out);
const char* piko_asset_last_error(void);
piko_status piko_asset_info_get(const piko_asset* asset, piko_asset_info* out);
/* Copies the flattened triangles into per-vertex-slot arrays (each may be
 * NULL): pos, nrm, col float4 [3][triangles], uv float2 [3][triangles].
 * colour_source 0: the reference's fixed material colour (0.9, 0.9, 0.6,
 * main.cpp:383); 1: each triangle's scene material diffuse colour. */
piko_status piko_asset_triangles(const piko_asset* asset, int colour_source, float* pos, float* nrm, float* col,
                                 float* uv);
/* Copies the patches: float4 [patches][16]. */
piko_status piko_asset_patches(const piko_asset* asset, float* patches);
/* The camera's view-projection matrix for a width x height target
 * (camera::updateCam, basicTypes/camera.h:73-120), column-major. */
piko_status piko_asset_view_proj(const piko_asset* asset, int width, int height, float* out16);
piko_status piko_asset_destroy(piko_asset* asset);
/* Writes an RGBA8 image (R in the low byte, row 0 = bottom) as a 24-bit BMP,
 * the screenshot format of the reference's EasyBMP; alpha is dropped. */
piko_status piko_image_write_bmp(const char* path, const uint32_t* rgba, int width, int height);

/* ------------------------------------------------------------------ allocation-free frame
 * No counterpart in the reference.  For callers that must not allocate device
 * memory while they run -- a plug-in inside a host application that reserves
 * all device memory in its own pool up front (a cudaMalloc from the plug-in
 * would fail or fragment that pool), or a real-time loop that cannot take the
 * synchronisation cudaMalloc/cudaFree may imply -- and so cannot use the entry
 * points above, which allocate and grow bin queues as needed.
 *
 * Renders one frame of the raster pipeline from the pre-transformed
 * raster_wtri payload (d_xyz: [count][9] floats, d_icol: [count][3] ABGR) into
 * d_rgba / d_depth (width*height each), all device pointers owned by the
 * caller, using only a fixed working area inside the library (about 23.5 MB of
 * device memory per GPU, held from library load until process exit).  Limits:
 * count <= 65,536 and width*height <= 1,048,576 (width, height >= 32); larger
 * requests return PIKO_ERR_LIMIT, and a frame whose bin queues would exceed
 * 2^20 entries (or 65,536 128-tile segments of large triangles) returns
 * PIKO_ERR_QUEUE_OVERFLOW.  The call waits for the frame.
 * The first call on a device looks up the working area's device address, so
 * make that first call before any stream capture.  Every call uses the same
 * working area: calls that could run on the GPU at the same time (other
 * streams, other threads) race and must be serialised by the caller. */
piko_status piko_raster_frame_noalloc(const float* d_xyz, const uint32_t* d_icol, int count, int width, int height,
                                      uint32_t* d_rgba, float* d_depth, void* stream);

/* Failure-path self-test (no counterpart in the reference): one CTA waits at
 * the Reyes split kernel's level barrier for a release that nothing sends.  The
 * wait is bounded (about a second); the kernel then records the timeout in its
 * status word and returns, and this call reports PIKO_ERR_TIMEOUT, as a frame
 * whose barrier gave up does.  The context stays usable afterwards.  Returns
 * PIKO_OK only if the wait was (wrongly) released. */
piko_status piko_selftest_wait_timeout(piko_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* PIKO_B200_H */
