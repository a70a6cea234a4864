"""The raster pipe built without VTX_PRETRANSFORM: the vertex stage transforms
world positions itself (vtxTransform, rasterMacros.h:14-21;
vertexShader.pikostage:56-80) and sets no vertex colours.  Coverage and depth
are pinned to the reference built that way (golden records from
oracle/_ref/libpiko_ref_raster_world.so); the device mode
(PIKO_SCENE_WTRI_WORLD) leaves the colours 0, which the oracle restates."""
import numpy as np
import pytest

from helpers import golden_cases, scene_from, sha

CASES = golden_cases("raster_world")


def _world(pk, oracle_mod, rec):
    sc = scene_from(pk, rec)
    xw = oracle_mod.world_xyz(sc)
    assert sha(xw) == rec["world_sha256"]
    assert np.array_equal(np.asarray(rec["view_proj"], np.float32), sc.view_proj)
    return sc, xw


@pytest.mark.parametrize("rec", CASES, ids=lambda r: r["case"])
def test_restatement_matches_reference_world_build(pk, oracle_mod, rec):
    sc, xw = _world(pk, oracle_mod, rec)
    xyz = oracle_mod.vs_world(sc.W, sc.H, xw, sc.view_proj)
    fb, depth, st = oracle_mod.raster_frame(sc.W, sc.H, xyz, np.zeros((sc.n, 3), np.uint32))
    assert sha(depth) == rec["depth_sha256"]
    assert st["passed"] == rec["emitted"]


def test_world_transform_equals_the_host_pretransform(pk, oracle_mod):
    """The vertex stage's transform and the host pre-transform of main.cpp
    (inPlaceTransform) are the same float sequence."""
    sc = pk.scenes.forest_scene()
    xyz, _ = oracle_mod.r1_setup(sc)
    assert np.array_equal(oracle_mod.vs_world(sc.W, sc.H, oracle_mod.world_xyz(sc), sc.view_proj), xyz)


@pytest.mark.gpu
@pytest.mark.parametrize("tile", [8, 16])
@pytest.mark.parametrize("rec", CASES, ids=lambda r: r["case"])
def test_device_world_mode_matches_reference(pk, ctx, oracle_mod, rec, tile):
    sc, xw = _world(pk, oracle_mod, rec)
    pipe = pk.Pipe(ctx, "raster", tile_px=tile)
    s = pk.Scene(pipe, {"W": sc.W, "H": sc.H, "xyz_world": xw, "view_proj": sc.view_proj})
    try:
        s.run()
        fb, depth = s.read()
        st = s.stats()
    finally:
        s.close()
        pipe.close()
    assert sha(depth) == rec["depth_sha256"], "depth differs from the reference"
    xyz = oracle_mod.vs_world(sc.W, sc.H, xw, sc.view_proj)
    ofb, odepth, ost = oracle_mod.raster_frame(sc.W, sc.H, xyz, np.zeros((sc.n, 3), np.uint32))
    assert np.array_equal(fb, ofb), "colour differs from the restatement (vertex colours 0)"
    assert st["covered"] == ost["covered"] and st["prims_kept"] == ost["kept"]
