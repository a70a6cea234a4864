"""ctypes binding of libpiko_b200.so (include/piko_b200.h).

The library is the product: this module only marshals arguments.  Importing
it never falls back to anything else; using it without the built library or
without a CUDA device raises :class:`PikoError`.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpiko_b200.so")

OK, ERR_INVALID, ERR_OOM, ERR_QUEUE_OVERFLOW, ERR_TIMEOUT, ERR_CUDA, ERR_UNSUPPORTED, ERR_NO_DEVICE, ERR_LIMIT = range(9)
STATUS_NAMES = {0: "PIKO_OK", 1: "PIKO_ERR_INVALID", 2: "PIKO_ERR_OOM", 3: "PIKO_ERR_QUEUE_OVERFLOW",
                4: "PIKO_ERR_TIMEOUT", 5: "PIKO_ERR_CUDA", 6: "PIKO_ERR_UNSUPPORTED", 7: "PIKO_ERR_NO_DEVICE",
                8: "PIKO_ERR_LIMIT"}

PRIM_RASTER_WTRI, PRIM_RASTER_STRI, PRIM_PIXEL, PRIM_PATCH, PRIM_UPOLY = 1, 2, 3, 4, 5
SCENE_TRIANGLES, SCENE_WTRI, SCENE_PATCHES, SCENE_WTRI_WORLD = 1, 2, 3, 4
MAX_STAGES = 8


class PikoError(RuntimeError):
    def __init__(self, status, message=""):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class CtxOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("time_kernels", ctypes.c_int)]


class StageDesc(ctypes.Structure):
    _fields_ = [("bin_size_x", ctypes.c_int), ("bin_size_y", ctypes.c_int), ("threads_per_tile", ctypes.c_int),
                ("in_prim", ctypes.c_int), ("out_prim", ctypes.c_int)]


class Link(ctypes.Structure):
    _fields_ = [("out_stage", ctypes.c_int), ("in_stage", ctypes.c_int), ("out_port", ctypes.c_int),
                ("in_port", ctypes.c_int)]


class PipeDesc(ctypes.Structure):
    _fields_ = [("n_stages", ctypes.c_int), ("stages", StageDesc * MAX_STAGES),
                ("n_links", ctypes.c_int), ("links", Link * MAX_STAGES),
                ("tile_px", ctypes.c_int), ("ctas_per_sm", ctypes.c_int),
                ("split_threshold_px", ctypes.c_float), ("max_splits", ctypes.c_int), ("dice_grid", ctypes.c_int),
                ("chunk_entries", ctypes.c_int), ("samples_per_pixel", ctypes.c_int),
                ("sample_seed", ctypes.c_uint32), ("phong", ctypes.c_int)]


class SceneDesc(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("kind", ctypes.c_int), ("count", ctypes.c_int),
                ("pos", ctypes.c_void_p), ("nrm", ctypes.c_void_p), ("col", ctypes.c_void_p), ("uv", ctypes.c_void_p),
                ("texture", ctypes.c_void_p), ("tex_w", ctypes.c_int), ("tex_h", ctypes.c_int),
                ("wtri_xyz", ctypes.c_void_p), ("wtri_icol", ctypes.c_void_p), ("patches", ctypes.c_void_p),
                ("packed", ctypes.c_int)]


class ConstState(ctypes.Structure):
    _fields_ = [("view_proj", ctypes.c_float * 16), ("light_mode", ctypes.c_int),
                ("light", ctypes.c_float * 3), ("eye", ctypes.c_float * 3)]


class FrameStats(ctypes.Structure):
    _fields_ = [("prims_in", ctypes.c_uint64), ("prims_kept", ctypes.c_uint64), ("upolys", ctypes.c_uint64),
                ("bin_entries", ctypes.c_uint64), ("covered", ctypes.c_uint64), ("wrap_risk", ctypes.c_uint64),
                ("status", ctypes.c_uint32), ("split_levels", ctypes.c_uint32), ("n_kernels", ctypes.c_int),
                ("kernel_ms", ctypes.c_float * 8)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "kernel_ms"}
        d["kernel_ms"] = list(self.kernel_ms)[: self.n_kernels]
        return d


class TuneCfg(ctypes.Structure):
    _fields_ = [("tile_px", ctypes.c_int), ("ctas_per_sm", ctypes.c_int), ("chunk_entries", ctypes.c_int),
                ("ms", ctypes.c_float), ("tuned", ctypes.c_int)]


class AssetInfo(ctypes.Structure):
    _fields_ = [("triangles", ctypes.c_int), ("patches", ctypes.c_int), ("has_uv", ctypes.c_int),
                ("has_camera", ctypes.c_int), ("eye", ctypes.c_float * 3), ("target", ctypes.c_float * 3),
                ("up", ctypes.c_float * 3), ("fovy_rad", ctypes.c_float), ("znear", ctypes.c_float),
                ("zfar", ctypes.c_float), ("lights", ctypes.c_int), ("materials", ctypes.c_int),
                ("light_pos", ctypes.c_float * 3)]


class ServerOpts(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("max_slots", ctypes.c_int), ("max_batch", ctypes.c_int),
                ("lanes", ctypes.c_int), ("max_pixels", ctypes.c_int), ("poll_us", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("batches", ctypes.c_uint64), ("mean_batch", ctypes.c_double), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("span_s", ctypes.c_double), ("hbm_bytes", ctypes.c_uint64), ("slots", ctypes.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# every symbol of include/piko_b200.h with its ctypes signature
_V, _I, _P = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER
SIGNATURES = {
    "piko_version": ([], ctypes.c_char_p),
    "piko_ctx_create": ([_P(CtxOpts), _P(_V)], _I),
    "piko_ctx_destroy": ([_V], _I),
    "piko_last_error": ([_V], ctypes.c_char_p),
    "piko_pipe_desc_raster": ([_P(PipeDesc)], None),
    "piko_pipe_desc_reyes": ([_P(PipeDesc)], None),
    "piko_pipe_create": ([_V, _P(PipeDesc), _P(_V)], _I),
    "piko_pipe_destroy": ([_V], _I),
    "piko_scene_create": ([_V, _P(SceneDesc), _P(_V)], _I),
    "piko_scene_upload": ([_V, _P(SceneDesc), _V], _I),
    "piko_scene_destroy": ([_V], _I),
    "piko_frame_prepare": ([_V, _P(ConstState)], _I),
    "piko_frame_run": ([_V, _V], _I),
    "piko_frame_finish": ([_V], _I),
    "piko_frame_read": ([_V, _V, _V], _I),
    "piko_frame_device_buffers": ([_V, _P(_V), _P(_V)], _I),
    "piko_frame_stats_get": ([_V, _P(FrameStats)], _I),
    "piko_frame_coverage": ([_V, _V, _V, ctypes.c_uint64, _P(ctypes.c_uint64)], _I),
    "piko_batch_create": ([_V, _P(_V), _I, _P(_V)], _I),
    "piko_batch_run": ([_V, _V, _I], _I),
    "piko_batch_finish": ([_V, _P(FrameStats)], _I),
    "piko_batch_destroy": ([_V], _I),
    "piko_tune_bucket": ([_I, _I, _I], _I),
    "piko_tuner_create": ([_P(_V)], _I),
    "piko_tuner_destroy": ([_V], _I),
    "piko_tuner_get": ([_V, _I, _P(TuneCfg)], _I),
    "piko_tuner_set": ([_V, _I, _P(TuneCfg)], _I),
    "piko_tuner_tune": ([_V, _V, _P(_V), _I, _I], _I),
    "piko_batch_create_tuned": ([_V, _P(_V), _I, _V, _P(_V)], _I),
    "piko_asset_load": ([ctypes.c_char_p, ctypes.c_char_p, _P(_V)], _I),
    "piko_asset_last_error": ([], ctypes.c_char_p),
    "piko_asset_info_get": ([_V, _P(AssetInfo)], _I),
    "piko_asset_triangles": ([_V, _I, _V, _V, _V, _V], _I),
    "piko_asset_patches": ([_V, _V], _I),
    "piko_asset_view_proj": ([_V, _I, _I, _V], _I),
    "piko_asset_destroy": ([_V], _I),
    "piko_image_write_bmp": ([ctypes.c_char_p, _V, _I, _I], _I),
    "piko_raster_frame_noalloc": ([_V, _V, _I, _I, _I, _V, _V, _V], _I),
    "piko_selftest_wait_timeout": ([_V], _I),
    "piko_server_create": ([_V, _P(ServerOpts), _P(_V)], _I),
    "piko_server_submit": ([_V, _V, _P(ConstState), _I, _P(ctypes.c_uint64)], _I),
    "piko_server_wait": ([_V, ctypes.c_uint64, _I], _I),
    "piko_server_drain": ([_V, _I], _I),
    "piko_server_read": ([_V, ctypes.c_uint64, _V, _V], _I),
    "piko_server_stats_get": ([_V, _P(ServerStats)], _I),
    "piko_server_reset_stats": ([_V], _I),
    "piko_server_destroy": ([_V], _I),
}

_lib = None


def load_library(path=LIB_PATH):
    """Loads the built library (raises PikoError if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise PikoError(ERR_UNSUPPORTED, f"{path} is not built (run piko-public_b200/build.py)")
    lib = ctypes.CDLL(path)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class Context:
    def __init__(self, device=0, time_kernels=False):
        self.lib = load_library()
        self.h = ctypes.c_void_p()
        opts = CtxOpts(device, 1 if time_kernels else 0)
        st = self.lib.piko_ctx_create(ctypes.byref(opts), ctypes.byref(self.h))
        if st != OK:
            raise PikoError(st, "piko_ctx_create")

    def check(self, st, what):
        if st != OK:
            raise PikoError(st, f"{what}: {self.lib.piko_last_error(self.h).decode()}")

    def close(self):
        if self.h:
            self.lib.piko_ctx_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Pipe:
    def __init__(self, ctx, kind="raster", tile_px=8, ctas_per_sm=0, split_threshold_px=0.0, max_splits=0,
                 dice_grid=0, desc=None, chunk_entries=0, samples_per_pixel=1, sample_seed=0, phong=False):
        self.ctx = ctx
        lib = ctx.lib
        if desc is None:
            desc = PipeDesc()
            (lib.piko_pipe_desc_raster if kind == "raster" else lib.piko_pipe_desc_reyes)(ctypes.byref(desc))
        desc.tile_px = tile_px
        desc.ctas_per_sm = ctas_per_sm
        desc.split_threshold_px = split_threshold_px
        desc.max_splits = max_splits
        desc.dice_grid = dice_grid
        desc.chunk_entries = chunk_entries
        desc.samples_per_pixel = samples_per_pixel
        desc.sample_seed = sample_seed & 0xFFFFFFFF
        desc.phong = 1 if phong else 0
        self.kind = kind
        self.h = ctypes.c_void_p()
        ctx.check(lib.piko_pipe_create(ctx.h, ctypes.byref(desc), ctypes.byref(self.h)), "piko_pipe_create")

    def close(self):
        if self.h:
            self.ctx.lib.piko_pipe_destroy(self.h)
            self.h = ctypes.c_void_p()


def scene_desc(scene, kind=None, packed=False):
    """piko_scene_desc for a scenes.RasterScene / PatchScene or a wtri payload
    dict {W, H, xyz [N,9], icol [N,3]}; returns (desc, keepalive).  packed:
    positions and normals as float3 (the scene's [3, N, 4] arrays cut to
    x, y, z, or [3, N, 3] arrays as they are)."""
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dt)
        keep.append(a)
        return _p(a)

    d = SceneDesc()
    if isinstance(scene, dict) and "xyz_world" in scene:
        # the raster_wtri payload without VTX_PRETRANSFORM: world positions,
        # transformed by the vertex stage with the frame's view-projection
        d.width, d.height, d.kind = scene["W"], scene["H"], SCENE_WTRI_WORLD
        d.count = int(scene["xyz_world"].shape[0])
        d.wtri_xyz = arr(scene["xyz_world"], np.float32)
        return d, keep
    if isinstance(scene, dict):
        d.width, d.height, d.kind = scene["W"], scene["H"], SCENE_WTRI
        d.count = int(scene["xyz"].shape[0])
        d.wtri_xyz = arr(scene["xyz"], np.float32)
        d.wtri_icol = arr(scene["icol"], np.uint32)
        return d, keep
    d.width, d.height = scene.W, scene.H
    d.count = scene.n
    if hasattr(scene, "patches"):
        d.kind = SCENE_PATCHES
        d.patches = arr(scene.patches, np.float32)
        return d, keep
    d.kind = SCENE_TRIANGLES
    if packed:
        d.packed = 1
        d.pos = arr(np.asarray(scene.pos)[..., :3], np.float32)
        d.nrm = arr(np.asarray(scene.nrm)[..., :3], np.float32)
    else:
        d.pos = arr(scene.pos, np.float32)
        d.nrm = arr(scene.nrm, np.float32)
    if scene.col is not None:          # None: the reference's fixed material colour
        d.col = arr(scene.col, np.float32)
    if scene.uv is not None:
        d.uv = arr(scene.uv, np.float32)
        d.texture = arr(scene.texture, np.uint8)
        d.tex_h, d.tex_w = int(scene.texture.shape[0]), int(scene.texture.shape[1])
    return d, keep


def const_state(scene=None, view_proj=None, light_mode=0, light=(0.5773, 0.5773, 0.5773), eye=(0, 0, 0)):
    cs = ConstState()
    if scene is not None and hasattr(scene, "light_mode"):
        view_proj, light_mode, light, eye = scene.view_proj, scene.light_mode, scene.light, scene.eye
    elif scene is not None:
        view_proj = scene.view_proj
    vp = np.eye(4, dtype=np.float32).reshape(16) if view_proj is None else np.asarray(view_proj, np.float32)
    for i in range(16):
        cs.view_proj[i] = float(vp[i])
    cs.light_mode = int(light_mode)
    for i in range(3):
        cs.light[i] = float(light[i])
        cs.eye[i] = float(eye[i])
    return cs


class Scene:
    """One scene: device-resident inputs, framebuffer and depth buffer."""

    def __init__(self, pipe, scene, packed=False):
        self.pipe = pipe
        self.ctx = pipe.ctx
        lib = self.ctx.lib
        desc, keep = scene_desc(scene, packed=packed)
        self.packed = packed
        self.W, self.H, self.N = desc.width, desc.height, desc.count
        self.h = ctypes.c_void_p()
        self.ctx.check(lib.piko_scene_create(pipe.h, ctypes.byref(desc), ctypes.byref(self.h)), "piko_scene_create")
        if not isinstance(scene, dict):
            self.prepare(const_state(scene))
        elif "view_proj" in scene:
            self.prepare(const_state(view_proj=scene["view_proj"]))

    def prepare(self, cs):
        self.ctx.check(self.ctx.lib.piko_frame_prepare(self.h, ctypes.byref(cs)), "piko_frame_prepare")

    def upload(self, scene_or_desc, stream=None):
        if isinstance(scene_or_desc, SceneDesc):
            desc, keep = scene_or_desc, None
        else:
            desc, keep = scene_desc(scene_or_desc, packed=self.packed)
        self._keep = keep
        self.ctx.check(self.ctx.lib.piko_scene_upload(self.h, ctypes.byref(desc), stream), "piko_scene_upload")

    def run(self, stream=None):
        self.ctx.check(self.ctx.lib.piko_frame_run(self.h, stream), "piko_frame_run")

    def finish(self):
        self.ctx.check(self.ctx.lib.piko_frame_finish(self.h), "piko_frame_finish")

    def read(self, out_fb=None, out_depth=None):
        fb = np.empty((self.H, self.W), np.uint32) if out_fb is None else out_fb
        depth = np.empty((self.H, self.W), np.float32) if out_depth is None else out_depth
        self.ctx.check(self.ctx.lib.piko_frame_read(self.h, _p(fb), _p(depth)), "piko_frame_read")
        return fb, depth

    def stats(self):
        st = FrameStats()
        self.ctx.check(self.ctx.lib.piko_frame_stats_get(self.h, ctypes.byref(st)), "piko_frame_stats_get")
        return st.as_dict()

    def device_buffers(self):
        fb, d = ctypes.c_void_p(), ctypes.c_void_p()
        self.ctx.check(self.ctx.lib.piko_frame_device_buffers(self.h, ctypes.byref(fb), ctypes.byref(d)), "buffers")
        return fb.value, d.value

    def coverage(self, cap=1 << 24):
        tri = np.zeros(cap, np.uint32)
        pix = np.zeros(cap, np.uint32)
        n = ctypes.c_uint64()
        self.ctx.check(self.ctx.lib.piko_frame_coverage(self.h, _p(tri), _p(pix), cap, ctypes.byref(n)),
                       "piko_frame_coverage")
        m = min(n.value, cap)
        return tri[:m], pix[:m], n.value

    def close(self):
        if self.h:
            self.ctx.lib.piko_scene_destroy(self.h)
            self.h = ctypes.c_void_p()


TUNE_BUCKETS = 16


def tune_bucket(width, height, triangles):
    """The tuner's scene-size bucket: resolution class * 4 + triangle class."""
    return load_library().piko_tune_bucket(int(width), int(height), int(triangles))


class Tuner:
    """Per scene-size bucket launch configuration of the batched form
    (piko_tuner_*): tile edge, persistent CTAs per SM, 8x8-queue chunk size.
    tune() measures; table()/load() save and restore a tuned table as plain
    data (JSON-ready)."""

    def __init__(self, table=None):
        self.lib = load_library()
        self.h = ctypes.c_void_p()
        st = self.lib.piko_tuner_create(ctypes.byref(self.h))
        if st != OK:
            raise PikoError(st, "piko_tuner_create")
        if table is not None:
            self.load(table)

    def tune(self, ctx, scenes, reps=5):
        arr = (ctypes.c_void_p * len(scenes))(*[s.h.value for s in scenes])
        ctx.check(self.lib.piko_tuner_tune(self.h, ctx.h, arr, len(scenes), reps), "piko_tuner_tune")
        return self

    def get(self, bucket):
        c = TuneCfg()
        st = self.lib.piko_tuner_get(self.h, bucket, ctypes.byref(c))
        if st != OK:
            raise PikoError(st, "piko_tuner_get")
        return {"tile_px": c.tile_px, "ctas_per_sm": c.ctas_per_sm, "chunk_entries": c.chunk_entries,
                "ms": c.ms, "tuned": bool(c.tuned)}

    def set(self, bucket, tile_px, ctas_per_sm=0, chunk_entries=0, ms=0.0, tuned=True):
        c = TuneCfg(tile_px, ctas_per_sm, chunk_entries, ms, 1 if tuned else 0)
        st = self.lib.piko_tuner_set(self.h, bucket, ctypes.byref(c))
        if st != OK:
            raise PikoError(st, f"piko_tuner_set(bucket {bucket})")

    def table(self, tuned_only=True):
        """{bucket: config} for the (tuned) buckets."""
        out = {}
        for b in range(TUNE_BUCKETS):
            c = self.get(b)
            if c["tuned"] or not tuned_only:
                out[b] = c
        return out

    def load(self, table):
        for b, c in table.items():
            self.set(int(b), c["tile_px"], c.get("ctas_per_sm", 0), c.get("chunk_entries", 0), c.get("ms", 0.0),
                     c.get("tuned", True))

    def close(self):
        if self.h:
            self.lib.piko_tuner_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_bmp(path, rgba):
    """Writes an RGBA8 framebuffer ([H, W] uint32, R in the low byte, row 0 =
    bottom) as a 24-bit BMP (piko_image_write_bmp)."""
    img = np.ascontiguousarray(rgba, np.uint32)
    lib = load_library()
    st = lib.piko_image_write_bmp(str(path).encode(), _p(img), int(img.shape[1]), int(img.shape[0]))
    if st != OK:
        raise PikoError(st, f"piko_image_write_bmp: {lib.piko_asset_last_error().decode()}")


class Asset:
    """A loaded .scene / .obj / .dat file (piko_asset_*): flattened triangles,
    Bezier patches, camera.  raster_scene() / patch_scene() give the inputs of
    Scene(pipe, ...) with the camera's view-projection for a W x H target and,
    for triangles, the reference's light (light vector toward the eye,
    main.cpp:372-378)."""

    def __init__(self, path, mesh_dir=None):
        self.lib = load_library()
        self.h = ctypes.c_void_p()
        st = self.lib.piko_asset_load(str(path).encode(), None if mesh_dir is None else str(mesh_dir).encode(),
                                      ctypes.byref(self.h))
        if st != OK:
            raise PikoError(st, f"piko_asset_load: {self.lib.piko_asset_last_error().decode()}")
        i = AssetInfo()
        self.lib.piko_asset_info_get(self.h, ctypes.byref(i))
        self.info = {k: (list(getattr(i, k)) if isinstance(getattr(i, k), ctypes.Array) else getattr(i, k))
                     for k, _ in AssetInfo._fields_}

    def view_proj(self, W, H):
        vp = np.zeros(16, np.float32)
        self.lib.piko_asset_view_proj(self.h, int(W), int(H), _p(vp))
        return vp

    def triangles(self, colour_source=0):
        n = self.info["triangles"]
        pos, nrm, col = (np.zeros((3, n, 4), np.float32) for _ in range(3))
        uv = np.zeros((3, n, 2), np.float32)
        st = self.lib.piko_asset_triangles(self.h, int(colour_source), _p(pos), _p(nrm), _p(col), _p(uv))
        if st != OK:
            raise PikoError(st, "piko_asset_triangles")
        return pos, nrm, col, uv

    def raster_scene(self, W, H, colour_source=0):
        from . import scenes
        pos, nrm, col, _ = self.triangles(colour_source)
        return scenes.RasterScene(W=W, H=H, pos=pos, nrm=nrm, col=col, view_proj=self.view_proj(W, H),
                                  light_mode=scenes.LIGHT_EYE, eye=np.array(self.info["eye"], np.float32),
                                  name="asset")

    def patch_scene(self, W, H):
        from . import scenes
        p = np.zeros((self.info["patches"], 16, 4), np.float32)
        if p.size:
            self.lib.piko_asset_patches(self.h, _p(p))
        return scenes.PatchScene(W=W, H=H, patches=p, view_proj=self.view_proj(W, H), name="asset")

    def close(self):
        if self.h:
            self.lib.piko_asset_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many raster scenes drawn by one launch sequence (optionally a CUDA graph);
    with a Tuner, one launch sequence per configuration group, on parallel
    branches of the graph."""

    def __init__(self, ctx, scenes, tuner=None):
        self.ctx = ctx
        self.scenes = list(scenes)
        arr = (ctypes.c_void_p * len(self.scenes))(*[s.h.value for s in self.scenes])
        self.h = ctypes.c_void_p()
        if tuner is None:
            ctx.check(ctx.lib.piko_batch_create(ctx.h, arr, len(self.scenes), ctypes.byref(self.h)),
                      "piko_batch_create")
        else:
            ctx.check(ctx.lib.piko_batch_create_tuned(ctx.h, arr, len(self.scenes), tuner.h, ctypes.byref(self.h)),
                      "piko_batch_create_tuned")

    def run(self, stream=None, graph=True):
        self.ctx.check(self.ctx.lib.piko_batch_run(self.h, stream, 1 if graph else 0), "piko_batch_run")

    def finish(self):
        st = FrameStats()
        self.ctx.check(self.ctx.lib.piko_batch_finish(self.h, ctypes.byref(st)), "piko_batch_finish")
        return st.as_dict()

    def close(self):
        if self.h:
            self.ctx.lib.piko_batch_destroy(self.h)
            self.h = ctypes.c_void_p()


class Server:
    """Continuous-batching request loop over resident scenes (piko_server_*)."""

    def __init__(self, ctx, hbm_budget_bytes=120 << 30, max_slots=256, max_batch=64, lanes=3,
                 max_pixels=1920 * 1080, poll_us=20):
        self.ctx = ctx
        o = ServerOpts(hbm_budget_bytes, max_slots, max_batch, lanes, max_pixels, poll_us)
        self.h = ctypes.c_void_p()
        ctx.check(ctx.lib.piko_server_create(ctx.h, ctypes.byref(o), ctypes.byref(self.h)), "piko_server_create")

    def submit(self, scene, state, keep=False):
        rid = ctypes.c_uint64()
        self.ctx.check(self.ctx.lib.piko_server_submit(self.h, scene.h, ctypes.byref(state), 1 if keep else 0,
                                                       ctypes.byref(rid)), "piko_server_submit")
        return rid.value

    def wait(self, rid, timeout_ms=60000):
        self.ctx.check(self.ctx.lib.piko_server_wait(self.h, rid, timeout_ms), "piko_server_wait")

    def drain(self, timeout_ms=120000):
        self.ctx.check(self.ctx.lib.piko_server_drain(self.h, timeout_ms), "piko_server_drain")

    def read(self, rid, W, H):
        fb = np.empty((H, W), np.uint32)
        depth = np.empty((H, W), np.float32)
        self.ctx.check(self.ctx.lib.piko_server_read(self.h, rid, _p(fb), _p(depth)), "piko_server_read")
        return fb, depth

    def stats(self):
        st = ServerStats()
        self.ctx.check(self.ctx.lib.piko_server_stats_get(self.h, ctypes.byref(st)), "piko_server_stats_get")
        return st.as_dict()

    def reset_stats(self):
        self.ctx.check(self.ctx.lib.piko_server_reset_stats(self.h), "piko_server_reset_stats")

    def close(self):
        if self.h:
            self.ctx.lib.piko_server_destroy(self.h)
            self.h = ctypes.c_void_p()
