"""The stage API of include/piko_stage.cuh (the reference's Stage /
assignBin / schedule / process / emit / pikoConnect interface) running user
pipelines: piko-public_b200/samples/stage_samples.cu, built into
libpiko_stage_samples.so.

raster2 restates the reference's RasterPipe stages through the API.  The
runtime orders every stage's work as the reference's one-thread CPU run does
and resolves the screen in that order, so the depth buffer, the covered-sample
count and the colour of every pixel equal the oracle's bit for bit -- also
where many fragments tie in depth, where the colour is the last tied fragment
in the reference's order.  subdivide checks a self-looping stage against a CPU
restatement."""
import ctypes
import os

import numpy as np
import pytest

from helpers import golden, scene_from

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "piko-public_b200", "libpiko_stage_samples.so")


@pytest.fixture(scope="module")
def samples():
    if not os.path.exists(LIB):
        pytest.fail("libpiko_stage_samples.so is not built (piko-public_b200/build.py)")
    lib = ctypes.CDLL(LIB)
    P = ctypes.c_void_p
    lib.piko_sample_raster.argtypes = [ctypes.c_int, ctypes.c_int, P, P, ctypes.c_int, P, P, P]
    lib.piko_sample_subdivide.argtypes = [ctypes.c_int, ctypes.c_int, P, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                          P, P, P, P]
    return lib


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_samples_library_exports_its_entry_points(samples):
    assert hasattr(samples, "piko_sample_raster") and hasattr(samples, "piko_sample_subdivide")


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["raster_plain4096_512", "raster_odd_size", "raster_depth_ties"])
def test_raster_through_the_stage_api_matches_the_oracle(pk, oracle_mod, samples, case):
    """raster_depth_ties draws many triangles at exactly equal depths: every
    tied fragment passes the reference's depth test and writes its colour, and
    the last one in the reference's one-thread order must win."""
    sc = scene_from(pk, golden(case))
    xyz, icol = oracle_mod.r1_setup(sc)
    fb = np.zeros((sc.H, sc.W), np.uint32)
    depth = np.zeros((sc.H, sc.W), np.float32)
    cov = np.zeros(1, np.uint64)
    assert samples.piko_sample_raster(sc.W, sc.H, ptr(np.ascontiguousarray(xyz)), ptr(np.ascontiguousarray(icol)),
                                      sc.n, ptr(fb), ptr(depth), ptr(cov)) == 0
    ofb, odepth, ost = oracle_mod.raster_frame(sc.W, sc.H, xyz, icol)
    assert np.array_equal(depth.view(np.uint32), odepth.view(np.uint32)), "depth differs from the oracle"
    assert int(cov[0]) == ost["covered"], "covered-sample count differs"
    bad = int(np.sum(fb != ofb))
    assert bad == 0, f"{bad} pixels differ from the oracle's colour"


def subdivide_cpu(segs, W, H, thr, max_depth):
    """The split stage's recursion in float32, returning the stamped pixels."""
    out = []
    stack = [(np.float32(a), np.float32(b), np.float32(c), np.float32(d), 0) for a, b, c, d in segs]
    half = np.float32(0.5)
    while stack:
        x0, y0, x1, y1, dep = stack.pop()
        dx, dy = np.float32(x1 - x0), np.float32(y1 - y0)
        if np.sqrt(np.float32(dx * dx + dy * dy), dtype=np.float32) >= np.float32(thr) and dep < max_depth:
            mx, my = np.float32((x0 + x1) * half), np.float32((y0 + y1) * half)
            stack.append((x0, y0, mx, my, dep + 1))
            stack.append((mx, my, x1, y1, dep + 1))
        else:
            out.append((int(np.floor(np.float32((x0 + x1) * half))), int(np.floor(np.float32((y0 + y1) * half)))))
    return out


@pytest.mark.gpu
def test_self_looping_stage_matches_the_recursion(samples):
    g = np.random.Generator(np.random.Philox(5))
    W, H = 200, 150
    segs = np.stack([g.uniform(0, W, 40), g.uniform(0, H, 40), g.uniform(0, W, 40), g.uniform(0, H, 40)], 1)
    segs = segs.astype(np.float32)
    thr, max_depth = 3.0, 12
    fb = np.zeros((H, W), np.uint32)
    leaves = np.zeros(1, np.uint64)
    rounds = np.zeros(1, np.int32)
    processed = np.zeros(1, np.uint64)
    assert samples.piko_sample_subdivide(W, H, ptr(segs), len(segs), thr, max_depth, ptr(fb), ptr(leaves),
                                         ptr(rounds), ptr(processed)) == 0
    pts = subdivide_cpu(segs, W, H, thr, max_depth)
    inside = [(x, y) for x, y in pts if 0 <= x < W and 0 <= y < H]
    assert int(leaves[0]) == len(inside)
    want = np.full((H, W), 0xFF000000, np.uint32)
    for x, y in inside:
        want[y, x] = 0xFFFFFFFF
    assert np.array_equal(fb, want)
    # every split doubles a segment: processed = leaves (all) + 2 * splits / 2 ... one round per split level
    assert 1 < int(rounds[0]) <= max_depth + 1
    assert int(processed[0]) == 2 * len(pts) - len(segs)
