"""piko_raster_frame_noalloc: one raster frame rendered entirely in the
library's fixed device arena, for callers that may not allocate device memory
while they run (for example a plug-in whose host application reserves all
device memory in its own pool, or a real-time loop that cannot take the
synchronisation cudaMalloc may imply).

It must produce exactly the frame the regular entry points produce, on every
call: the arena is reused, so the second call checks that nothing left over
from the first one leaks into it.  Runs last (file name) so that a failure
here leaves every other test already run."""
import ctypes

import numpy as np
import pytest

from helpers import golden, scene_from, sha

pytestmark = pytest.mark.gpu

STATUS_OVERFLOW = 3
STATUS_LIMIT = 8
CLEAR_COLOUR = 0xff663313


def _entry(pk):
    lib = pk.load_library()
    fn = lib.piko_raster_frame_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _regular(pk, ctx, W, H, xyz, icol):
    pipe = pk.Pipe(ctx, "raster")
    s = pk.Scene(pipe, {"W": W, "H": H, "xyz": xyz, "icol": icol})
    try:
        s.run()
        return s.read()
    finally:
        s.close()
        pipe.close()


@pytest.mark.parametrize("case", ["raster_plain4096_512", "raster_odd_size", "raster_depth_ties"])
def test_noalloc_matches_regular_path_twice(pk, ctx, oracle_mod, case):
    import torch
    rec = golden(case)
    sc = scene_from(pk, rec)
    xyz, icol = oracle_mod.r1_setup(sc)
    fb_ref, depth_ref = _regular(pk, ctx, sc.W, sc.H, xyz, icol)
    assert sha(fb_ref) == rec["fb_sha256"]
    fn = _entry(pk)
    d_xyz = torch.from_numpy(xyz).cuda()
    d_icol = torch.from_numpy(icol.view(np.int32)).cuda()
    for call in range(2):
        d_fb = torch.full((sc.H, sc.W), 7, dtype=torch.int32, device="cuda")
        d_z = torch.full((sc.H, sc.W), -3.0, dtype=torch.float32, device="cuda")
        st = fn(d_xyz.data_ptr(), d_icol.data_ptr(), sc.n, sc.W, sc.H, d_fb.data_ptr(), d_z.data_ptr(), None)
        assert st == 0, f"call {call}: status {st}"
        fb = d_fb.cpu().numpy().view(np.uint32)
        z = d_z.cpu().numpy()
        assert np.array_equal(fb, fb_ref), f"call {call}: colour differs"
        assert np.array_equal(z.view(np.uint32), depth_ref.view(np.uint32)), f"call {call}: depth differs"


def test_noalloc_rejects_sizes_beyond_its_limits(pk):
    import torch
    fn = _entry(pk)
    d = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = d.data_ptr()
    assert fn(p, p, 70000, 64, 64, p, p, None) == STATUS_LIMIT        # more than 65,536 triangles
    assert fn(p, p, 10, 2048, 1024, p, p, None) == STATUS_LIMIT       # more than 2^20 pixels


def _call(fn, xyz, icol, n, W, H):
    """One call on fresh output buffers filled with junk; (status, rgba, depth)."""
    import torch
    d_xyz = torch.from_numpy(np.ascontiguousarray(xyz)).cuda()
    d_icol = torch.from_numpy(np.ascontiguousarray(icol).view(np.int32)).cuda()
    d_fb = torch.full((H, W), 7, dtype=torch.int32, device="cuda")
    d_z = torch.full((H, W), -3.0, dtype=torch.float32, device="cuda")
    st = fn(d_xyz.data_ptr(), d_icol.data_ptr(), n, W, H, d_fb.data_ptr(), d_z.data_ptr(), None)
    torch.cuda.synchronize()
    return st, d_fb.cpu().numpy().view(np.uint32), d_z.cpu().numpy()


def test_noalloc_empty_frame_is_cleared(pk):
    """No triangles: every pixel takes the clear colour and depth 1.0."""
    fn = _entry(pk)
    xyz = np.zeros((1, 9), np.float32)
    icol = np.zeros((1, 3), np.uint32)
    st, fb, z = _call(fn, xyz, icol, 0, 96, 64)
    assert st == 0
    assert np.all(fb == CLEAR_COLOUR) and np.all(z == 1.0)


def test_noalloc_overflow_is_reported_and_the_arena_recovers(pk, oracle_mod):
    """3,000 screen-sized triangles need more than 2^20 (triangle, tile) entries
    and more than 65,536 large-triangle segments: the call reports the overflow
    instead of drawing a wrong frame.  The next call on the same arena draws a
    golden frame bit for bit."""
    fn = _entry(pk)
    n, W, H = 3000, 1024, 1024
    tri = np.array([-200.0, -200.0, 0.5, 1240.0, -200.0, 0.5, -200.0, 1240.0, 0.5], np.float32)
    xyz = np.tile(tri, (n, 1))
    xyz[:, 2::3] = np.linspace(0.1, 0.9, n, dtype=np.float32)[:, None]
    icol = np.full((n, 3), 0xff0000ff, np.uint32)
    st, _, _ = _call(fn, xyz, icol, n, W, H)
    assert st == STATUS_OVERFLOW
    rec = golden("raster_plain4096_512")
    sc = scene_from(pk, rec)
    gx, gi = oracle_mod.r1_setup(sc)
    st, fb, z = _call(fn, gx, gi, sc.n, sc.W, sc.H)
    assert st == 0
    assert sha(fb) == rec["fb_sha256"] and sha(z) == rec["depth_sha256"]
