"""pikoc.py: pipelines written in the reference's stage-file form (a PikoPipe
class header and .pikostage files, unchanged) compiled for the B200 -- stage
code by NVRTC against include/piko/, the pipe class's host methods generated
on the stage runtime -- and run with the reference's one-thread order.

* tests/golden/assets/splatpipe: a test pipeline in that form (points stamp
  2x2 pixel blocks; later points in the one-thread order win).
* the reference's own RasterPipe and ReyesPipe (pikoc/samples/), compiled by
  __graft_entry__.build() where the reference tree is present; their images
  must equal the reference's golden records bit for bit.
"""
import ctypes
import os

import numpy as np
import pytest

from helpers import golden, scene_from, sha

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUT = os.path.join(ROOT, "piko-public_b200", "_pikoc")
SPLAT_HEADER = os.path.join(ROOT, "tests", "golden", "assets", "splatpipe", "splatPipe.h")

RASTER_WTRI = np.dtype([("binID", "<u4"), ("launchIdx", "<u4"), ("id", "<i4"), ("xyz", "<f4", (9,)),
                        ("icol", "<u4", (3,))])
PIKO_PATCH = np.dtype([("binID", "<u4"), ("launchIdx", "<u4"), ("cp", "<f4", (16, 4)), ("numSplits", "<i4"),
                       ("nu", "<i4"), ("nv", "<i4"), ("id", "<i4"), ("bbmin", "<f4", (2,)), ("bbmax", "<f4", (2,))])
SPLAT_POINT = np.dtype([("binID", "<u4"), ("launchIdx", "<u4"), ("id", "<i4"), ("x", "<f4"), ("y", "<f4"),
                        ("color", "<u4")])


def _pikoc():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "piko-public_b200"))
    import pikoc
    sys.path.pop(0)
    return pikoc


def _lib(name, build_if_missing=None):
    path = os.path.join(OUT, name, f"libpikoc_{name}.so")
    if not os.path.exists(path):
        if build_if_missing is None:
            pytest.skip(f"{name} is compiled only where the reference tree is present")
        _pikoc().compile_pipe(build_if_missing, os.path.join(OUT, name))
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    lib.pikoc_new.restype = P
    lib.pikoc_delete.argtypes = [P]
    lib.pikoc_error.argtypes = [P]
    lib.pikoc_error.restype = ctypes.c_char_p
    lib.pikoc_allocate.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, ctypes.c_int]
    lib.pikoc_frame.argtypes = [P]
    lib.pikoc_read.argtypes = [P, P, P]
    lib.pikoc_processed.argtypes = [P, P, ctypes.c_int]
    return lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _run(lib, W, H, vp, items):
    h = lib.pikoc_new()
    try:
        assert lib.pikoc_allocate(h, W, H, _ptr(vp), _ptr(items), len(items)) == 0, lib.pikoc_error(h)
        assert lib.pikoc_frame(h) == 0, lib.pikoc_error(h)
        fb = np.zeros((H, W), np.uint32)
        depth = np.zeros((H, W), np.float32)
        assert lib.pikoc_read(h, _ptr(fb), _ptr(depth)) == 0, lib.pikoc_error(h)
        done = np.zeros(lib.pikoc_stages(), np.uint64)
        lib.pikoc_processed(h, _ptr(done), len(done))
        return fb, depth, done
    finally:
        lib.pikoc_delete(h)


def test_parse_finds_the_pipe_its_stages_and_its_input():
    info = _pikoc().parse(SPLAT_HEADER)
    assert info["pipe"] == "SplatPipe"
    assert info["members"] == [("SplatStage", "splat")]
    assert info["own_emit"] == {"SplatStage": True}
    assert info["input_type"] == "splat_point"


def test_compiled_pipe_exports_its_abi():
    lib = _lib("SplatPipe", SPLAT_HEADER)
    assert lib.pikoc_input_size() == SPLAT_POINT.itemsize and lib.pikoc_stages() == 1


def _splat_points(n, W, H, seed):
    g = np.random.Generator(np.random.Philox(seed))
    pts = np.zeros(n, SPLAT_POINT)
    pts["id"] = np.arange(n)
    pts["x"] = g.uniform(0, W, n).astype(np.float32)
    pts["y"] = g.uniform(0, H, n).astype(np.float32)
    pts["color"] = g.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32) | np.uint32(0xff000000)
    return pts


def _splat_cpu(pts, W, H):
    """The one-thread run: bins in index order (16x16 px, W // 16 per row),
    each bin's points in input order, each stamping its 2x2 block."""
    fb = np.full((H, W), 0xff663313, np.uint32)
    nbx, nby = max(1, W // 16), max(1, H // 16)
    x0 = np.floor(pts["x"]).astype(np.int64)
    y0 = np.floor(pts["y"]).astype(np.int64)
    bx, by = x0 // 16, y0 // 16
    ok = (bx < nbx) & (by < nby)
    order = sorted(np.nonzero(ok)[0].tolist(), key=lambda i: (int(by[i] * nbx + bx[i]), i))
    for i in order:
        for dy in range(2):
            for dx in range(2):
                x, y = x0[i] + dx, y0[i] + dy
                if x < W and y < H:
                    fb[y, x] = pts["color"][i]
    return fb, int(ok.sum())


@pytest.mark.gpu
@pytest.mark.parametrize("seed,n", [(1, 3000), (2, 20000)])
def test_splat_pipe_runs_in_one_thread_order(seed, n):
    """Many overlapping stamps: every pixel must hold the colour of the last
    stamp in the reference's one-thread order, whatever order the GPU ran."""
    lib = _lib("SplatPipe", SPLAT_HEADER)
    W, H = 200, 136
    pts = _splat_points(n, W, H, seed)
    fb, _, done = _run(lib, W, H, None, pts)
    want, assigned = _splat_cpu(pts, W, H)
    assert int(done[0]) == n
    bad = int(np.sum(fb != want))
    assert bad == 0, f"{bad} pixels differ from the one-thread order"


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["raster_plain4096_512", "raster_odd_size", "raster_depth_ties",
                                  "raster_order_wrap_256"])
def test_reference_raster_pipe_matches_reference(pk, oracle_mod, case):
    """The reference's RasterPipe (rasterPipe.h, vertexShader.pikostage,
    raster.pikostage, unchanged) on the B200 equals the reference's own CPU
    run, colour included."""
    lib = _lib("RasterPipe")
    rec = golden(case)
    sc = scene_from(pk, rec)
    xyz, icol = oracle_mod.r1_setup(sc)
    tris = np.zeros(sc.n, RASTER_WTRI)
    assert lib.pikoc_input_size() == RASTER_WTRI.itemsize
    tris["id"] = np.arange(sc.n)
    tris["xyz"] = xyz
    tris["icol"] = icol
    fb, depth, done = _run(lib, sc.W, sc.H, None, tris)
    assert sha(depth) == rec["depth_sha256"], "depth differs from the reference"
    assert sha(fb) == rec["fb_sha256"], "colour differs from the reference"
    assert int(done[0]) == sc.n


def _depths_positive(sc):
    """Every control point in front of the camera with a positive projected
    depth, so every micropolygon's depth is positive: the reference's Shade
    depth loop (shade.pikostage:232-237) ends only for such depths (for two
    negative depths it repeats forever), so nothing else is run."""
    cp = sc.patches.reshape(-1, 4).astype(np.float64)
    m = np.asarray(sc.view_proj, np.float64).reshape(4, 4).T
    clip = cp @ m.T
    return bool(np.all(clip[:, 3] > 0) and np.all(clip[:, 2] / clip[:, 3] > 0))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["reyes_sphere32_small", "reyes_sphere32_ref_constants"])
def test_reference_reyes_pipe_matches_reference(pk, case):
    """The reference's ReyesPipe (reyesPipe.h, split / dice / shade
    .pikostage, unchanged: its Split loop, 4 px threshold, 20 splits) on the
    B200 equals the reference's own CPU run."""
    lib = _lib("ReyesPipe")
    rec = golden(case)
    sc = scene_from(pk, rec)
    assert _depths_positive(sc), "a control point projects behind the camera"
    p = np.zeros(sc.n, PIKO_PATCH)
    assert lib.pikoc_input_size() == PIKO_PATCH.itemsize
    p["cp"] = sc.patches
    p["id"] = np.arange(sc.n)
    p["bbmin"] = 99999.0
    p["bbmax"] = -99999.0
    vp = np.ascontiguousarray(sc.view_proj, np.float32)
    fb, depth, done = _run(lib, sc.W, sc.H, vp, p)
    assert sha(depth) == rec["depth_sha256"], "depth differs from the reference"
    assert sha(fb) == rec["fb_sha256"], "colour differs from the reference"
    assert int(done[1]) == rec["leaves"] and int(done[2]) == rec["upolys"]
