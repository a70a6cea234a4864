"""TEST INFRASTRUCTURE — the oracle.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this package, and only as the checker (or the timed CPU reference); the
product path never does.

Two implementations live here:

* ``restated``: ``liboracle.so``, a plain-C restatement of the reference's
  raster and Reyes stage code (``oracle/src``), each function citing the
  reference file and lines it follows.
* ``ref``: ``_ref/libpiko_ref_raster.so`` and ``_ref/libpiko_ref_reyes.so``, the
  reference's own stage code compiled in place from its source tree with
  hand-written ``pikoc --target=CPU`` glue (``oracle/ref``).  They are built
  here (``make -C oracle``) and travel to the GPU host as built files; the
  source tree itself is never read at run time there.

The restatement is pinned against the reference build on every golden case
(``tests/test_oracle_pins.py``) and against the committed fixtures in
``tests/golden``.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_RESTATED = os.path.join(HERE, "liboracle.so")
LIB_REF_RASTER = os.path.join(HERE, "_ref", "libpiko_ref_raster.so")
LIB_REF_REYES = os.path.join(HERE, "_ref", "libpiko_ref_reyes.so")
# the raster pipe built without VTX_PRETRANSFORM: the vertex stage transforms
# world positions itself (no colours are set in that mode); see oracle/Makefile
LIB_REF_RASTER_WORLD = os.path.join(HERE, "_ref", "libpiko_ref_raster_world.so")
# the same Reyes pipe built with the Reyes workload's constants substituted into
# a build copy of split.pikostage (split below 16 px, at most 10 splits, fixed
# 16x16 dice grids); see oracle/Makefile
LIB_REF_REYES_C2 = os.path.join(HERE, "_ref", "libpiko_ref_reyes_c2.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_LL = ctypes.c_longlong


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


_lib = None


def restated():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(LIB_RESTATED)
        lib.oracle_r1_setup.argtypes = [_I, _I, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P]
        lib.oracle_raster_frame.argtypes = [_I, _I, _I, _P, _P, _P, _P, _I, _I, _P, _P, _P]
        lib.oracle_raster_coverage.argtypes = [_I, _I, _I, _P, _P, _P, _P, _P, _LL]
        lib.oracle_raster_coverage.restype = _LL
        lib.oracle_submission_order.argtypes = [_I, _I, _I, _P]
        lib.oracle_vs_world.argtypes = [_I, _I, _I, _P, _P, _P]
        lib.oracle_reyes_frame.argtypes = [_I, _I, _I, _P, _P, ctypes.c_float, _I, _I, _P, _P, _P, _P, _LL]
        lib.oracle_reyes_frame_ms.argtypes = [_I, _I, _I, _P, _P, ctypes.c_float, _I, _I, _I, ctypes.c_uint32, _I,
                                              _P, _P, _P]
        _lib = lib
    return _lib


def r1_setup(scene):
    """R1 on the CPU: world-space SoA attributes -> pre-transformed raster_wtri
    payload (xyz [N, 9] float32, icol [N, 3] uint32)."""
    n = scene.n
    xyz = np.zeros((n, 9), np.float32)
    icol = np.zeros((n, 3), np.uint32)
    pos = np.ascontiguousarray(scene.pos, np.float32)
    nrm = np.ascontiguousarray(scene.nrm, np.float32)
    col = None if scene.col is None else np.ascontiguousarray(scene.col, np.float32)
    vp = np.ascontiguousarray(scene.view_proj, np.float32)
    light = np.ascontiguousarray(scene.light, np.float32)
    eye = np.ascontiguousarray(scene.eye, np.float32)
    restated().oracle_r1_setup(n, scene.W, scene.H, _ptr(pos), _ptr(nrm), _ptr(col), _ptr(vp),
                               int(scene.light_mode), _ptr(light), _ptr(eye), _ptr(xyz), _ptr(icol))
    return xyz, icol


def world_xyz(scene):
    """A triangle scene's world positions as the reference's raster_wtri
    worldPos0..2 payload: [N, 9] float32."""
    return np.ascontiguousarray(scene.pos[:, :, :3].transpose(1, 0, 2).reshape(scene.n, 9), np.float32)


def vs_world(W, H, xyz_world, view_proj):
    """The vertex stage's transform without VTX_PRETRANSFORM: world positions
    [N, 9] -> screen x, y, depth [N, 9] (the pre-transformed payload)."""
    n = int(xyz_world.shape[0])
    out = np.zeros((n, 9), np.float32)
    w = np.ascontiguousarray(xyz_world, np.float32)
    vp = np.ascontiguousarray(view_proj, np.float32)
    restated().oracle_vs_world(n, W, H, _ptr(w), _ptr(vp), _ptr(out))
    return out


def uv_per_tri(scene):
    """[N, 6] float32 (u0, v0, u1, v1, u2, v2) or None."""
    if scene.uv is None:
        return None
    return np.ascontiguousarray(scene.uv.transpose(1, 0, 2).reshape(scene.n, 6), np.float32)


def raster_frame(W, H, xyz, icol, uv=None, texture=None):
    """Restated one-thread raster frame -> (fb uint32 [H, W], depth float32 [H, W], stats)."""
    n = int(xyz.shape[0])
    fb = np.zeros((H, W), np.uint32)
    depth = np.zeros((H, W), np.float32)
    stats = np.zeros(4, np.int64)
    xyz = np.ascontiguousarray(xyz, np.float32)
    icol = np.ascontiguousarray(icol, np.uint32)
    tex = None if texture is None else np.ascontiguousarray(texture, np.uint8)
    TW = 0 if tex is None else tex.shape[1]
    TH = 0 if tex is None else tex.shape[0]
    restated().oracle_raster_frame(W, H, n, _ptr(xyz), _ptr(icol), _ptr(uv), _ptr(tex), TW, TH,
                                   _ptr(fb), _ptr(depth), _ptr(stats))
    return fb, depth, dict(kept=int(stats[0]), pairs=int(stats[1]), covered=int(stats[2]), passed=int(stats[3]))


def raster_scene(scene):
    xyz, icol = r1_setup(scene)
    return raster_frame(scene.W, scene.H, xyz, icol, uv_per_tri(scene), scene.texture)


def raster_coverage(W, H, xyz, icol):
    """All non-empty (triangle, 8x8 bin) coverage masks, sorted by (tri, bin)."""
    n = int(xyz.shape[0])
    xyz = np.ascontiguousarray(xyz, np.float32)
    icol = np.ascontiguousarray(icol, np.uint32)
    lib = restated()
    total = lib.oracle_raster_coverage(W, H, n, _ptr(xyz), _ptr(icol), None, None, None, 0)
    tri = np.zeros(max(total, 1), np.int32)
    binv = np.zeros(max(total, 1), np.int32)
    mask = np.zeros(max(total, 1), np.uint64)
    lib.oracle_raster_coverage(W, H, n, _ptr(xyz), _ptr(icol), _ptr(tri), _ptr(binv), _ptr(mask), total)
    return tri[:total], binv[:total], mask[:total]


def submission_order(n, W, H):
    out = np.zeros(max(n, 1), np.int32)
    restated().oracle_submission_order(n, W, H, _ptr(out))
    return out[:n]


def reyes_frame(scene, threshold=4.0, max_splits=20, grid=0, leaf_cap=0):
    W, H = scene.W, scene.H
    fb = np.zeros((H, W), np.uint32)
    depth = np.zeros((H, W), np.float32)
    stats = np.zeros(7, np.int64)
    cps = np.ascontiguousarray(scene.patches, np.float32)
    vp = np.ascontiguousarray(scene.view_proj, np.float32)
    leaves = np.zeros((max(leaf_cap, 1), 4), np.int32) if leaf_cap else None
    restated().oracle_reyes_frame(W, H, scene.n, _ptr(cps), _ptr(vp), float(threshold), int(max_splits), int(grid),
                                  _ptr(fb), _ptr(depth), _ptr(stats), _ptr(leaves), int(leaf_cap))
    st = dict(leaves=int(stats[0]), upolys=int(stats[1]), pairs=int(stats[2]), covered=int(stats[3]),
              passed=int(stats[4]), hangs=int(stats[5]), levels=int(stats[6]))
    if leaf_cap:
        st["leaf_list"] = leaves[:min(leaf_cap, st["leaves"])]
    return fb, depth, st


def reyes_frame_ms(scene, threshold=4.0, max_splits=20, grid=0, spp=4, seed=0, phong=True):
    """The multi-sample / Phong Reyes variant (no reference counterpart):
    spp samples per pixel at jittered positions, the reference's per-sample
    coverage and depth loop, and (phong) lighting of the interpolated normal;
    pixels average their samples' colours and keep the nearest depth."""
    W, H = scene.W, scene.H
    fb = np.zeros((H, W), np.uint32)
    depth = np.zeros((H, W), np.float32)
    stats = np.zeros(7, np.int64)
    cps = np.ascontiguousarray(scene.patches, np.float32)
    vp = np.ascontiguousarray(scene.view_proj, np.float32)
    r = restated().oracle_reyes_frame_ms(W, H, scene.n, _ptr(cps), _ptr(vp), float(threshold), int(max_splits),
                                         int(grid), int(spp), int(seed) & 0xFFFFFFFF, 1 if phong else 0,
                                         _ptr(fb), _ptr(depth), _ptr(stats))
    if r != 0:
        raise ValueError("spp must be 1 or 4")
    st = dict(leaves=int(stats[0]), upolys=int(stats[1]), pairs=int(stats[2]), covered=int(stats[3]),
              passed=int(stats[4]), hangs=int(stats[5]), levels=int(stats[6]))
    return fb, depth, st


# ---------------------------------------------------------------- reference build
_ref_r = None
_ref_y = {}


def ref_available():
    return os.path.exists(LIB_REF_RASTER) and os.path.exists(LIB_REF_REYES)


def ref_raster():
    global _ref_r
    if _ref_r is None:
        lib = ctypes.CDLL(LIB_REF_RASTER)
        lib.piko_ref_raster_create.argtypes = [_I, _I, _P, _P, _I]
        lib.piko_ref_raster_frame.argtypes = [_I]
        lib.piko_ref_raster_frame.restype = _LL
        lib.piko_ref_raster_read.argtypes = [_P, _P]
        lib.piko_ref_raster_emitted.argtypes = [_I]
        lib.piko_ref_raster_emitted.restype = _LL
        lib.piko_ref_raster_coverage.argtypes = [_I, _P, _I]
        lib.piko_ref_raster_bins.argtypes = [_P, _P, _P]
        _ref_r = lib
    return _ref_r


def ref_c2_available():
    return os.path.exists(LIB_REF_REYES_C2)


def ref_reyes(workload_constants=False):
    path = LIB_REF_REYES_C2 if workload_constants else LIB_REF_REYES
    if path not in _ref_y:
        lib = ctypes.CDLL(path)
        lib.piko_ref_reyes_create.argtypes = [_I, _I, _P, _I, _P]
        lib.piko_ref_reyes_frame.argtypes = [_I, _I]
        lib.piko_ref_reyes_frame.restype = _LL
        lib.piko_ref_reyes_read.argtypes = [_P, _P]
        lib.piko_ref_reyes_counters.argtypes = [_P, _I]
        lib.piko_ref_reyes_leaves.argtypes = [_P, _LL]
        lib.piko_ref_reyes_leaves.restype = _LL
        _ref_y[path] = lib
    return _ref_y[path]


class RefRaster:
    """The reference's RasterPipe on the CPU (one instance at a time: the
    reference's generated code keeps its state in globals)."""

    def __init__(self, W, H, xyz, icol):
        self.W, self.H = W, H
        self.n = int(xyz.shape[0])
        self._xyz = np.ascontiguousarray(xyz, np.float32)
        self._icol = np.ascontiguousarray(icol, np.uint32)
        self.grown = ref_raster().piko_ref_raster_create(W, H, _ptr(self._xyz), _ptr(self._icol), self.n)
        if self.grown < 0:
            raise RuntimeError("piko_ref_raster_create failed")

    def frame(self, cpu_threads=1):
        """Runs one frame; returns its wall time in ns."""
        return int(ref_raster().piko_ref_raster_frame(int(cpu_threads)))

    def read(self):
        fb = np.zeros((self.H, self.W), np.uint32)
        depth = np.zeros((self.H, self.W), np.float32)
        ref_raster().piko_ref_raster_read(_ptr(fb), _ptr(depth))
        return fb, depth

    def emitted(self, reset=True):
        return int(ref_raster().piko_ref_raster_emitted(1 if reset else 0))

    def coverage(self, tri, cap=1 << 20):
        xy = np.zeros((cap, 2), np.int32)
        n = ref_raster().piko_ref_raster_coverage(int(tri), _ptr(xy), cap)
        return xy[:n]

    def close(self):
        ref_raster().piko_ref_raster_destroy()


def ref_world_available():
    return os.path.exists(LIB_REF_RASTER_WORLD)


_ref_w = None


class RefRasterWorld:
    """The reference's RasterPipe built without VTX_PRETRANSFORM, on the CPU:
    world positions in, the vertex stage's own transform.  The reference sets
    no vertex colours in that mode, so only depth and the emitted Pixel count
    are meaningful."""

    def __init__(self, W, H, xyz_world, view_proj):
        global _ref_w
        if _ref_w is None:
            lib = ctypes.CDLL(LIB_REF_RASTER_WORLD)
            lib.piko_ref_raster_create_world.argtypes = [_I, _I, _P, _P, _I]
            lib.piko_ref_raster_frame.argtypes = [_I]
            lib.piko_ref_raster_frame.restype = _LL
            lib.piko_ref_raster_read.argtypes = [_P, _P]
            lib.piko_ref_raster_emitted.argtypes = [_I]
            lib.piko_ref_raster_emitted.restype = _LL
            _ref_w = lib
        self._lib = _ref_w
        self.W, self.H = W, H
        self._xyz = np.ascontiguousarray(xyz_world, np.float32)
        self._vp = np.ascontiguousarray(view_proj, np.float32)
        if self._lib.piko_ref_raster_create_world(W, H, _ptr(self._xyz), _ptr(self._vp), int(self._xyz.shape[0])) < 0:
            raise RuntimeError("piko_ref_raster_create_world failed")

    def frame(self, cpu_threads=1):
        return int(self._lib.piko_ref_raster_frame(int(cpu_threads)))

    def read(self):
        fb = np.zeros((self.H, self.W), np.uint32)
        depth = np.zeros((self.H, self.W), np.float32)
        self._lib.piko_ref_raster_read(_ptr(fb), _ptr(depth))
        return fb, depth

    def emitted(self, reset=True):
        return int(self._lib.piko_ref_raster_emitted(1 if reset else 0))

    def close(self):
        self._lib.piko_ref_raster_destroy()


class RefReyes:
    """The reference's ReyesPipe on the CPU; workload_constants=True selects the
    build with the Reyes workload's split threshold, split limit and dice grid."""

    def __init__(self, scene, workload_constants=False):
        self.W, self.H = scene.W, scene.H
        self._lib = ref_reyes(workload_constants)
        self._cps = np.ascontiguousarray(scene.patches, np.float32)
        self._vp = np.ascontiguousarray(scene.view_proj, np.float32)
        r = self._lib.piko_ref_reyes_create(self.W, self.H, _ptr(self._cps), scene.n, _ptr(self._vp))
        if r < 0:
            raise RuntimeError("piko_ref_reyes_create failed")

    def frame(self, cpu_threads=1, record_leaves=False):
        return int(self._lib.piko_ref_reyes_frame(int(cpu_threads), 1 if record_leaves else 0))

    def read(self):
        fb = np.zeros((self.H, self.W), np.uint32)
        depth = np.zeros((self.H, self.W), np.float32)
        self._lib.piko_ref_reyes_read(_ptr(fb), _ptr(depth))
        return fb, depth

    def counters(self, reset=True):
        out = np.zeros(4, np.int64)
        self._lib.piko_ref_reyes_counters(_ptr(out), 1 if reset else 0)
        return dict(leaves=int(out[0]), upolys=int(out[1]), emitted=int(out[2]), levels=int(out[3]))

    def leaves(self):
        n = self._lib.piko_ref_reyes_leaves(None, 0)
        out = np.zeros((max(n, 1), 4), np.int32)
        self._lib.piko_ref_reyes_leaves(_ptr(out), n)
        return out[:n]

    def close(self):
        self._lib.piko_ref_reyes_destroy()
