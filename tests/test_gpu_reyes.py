"""Device Reyes path vs the oracle: bit-exact image, depth, leaf and
micropolygon counts."""
import numpy as np
import pytest

from helpers import golden, golden_cases, scene_from, sha

pytestmark = pytest.mark.gpu


def render(pk, ctx, sc, **kw):
    pipe = pk.Pipe(ctx, "reyes", **kw)
    s = pk.Scene(pipe, sc)
    try:
        s.run()
        fb, depth = s.read()
        st = s.stats()
    finally:
        s.close()
        pipe.close()
    return fb, depth, st


@pytest.mark.parametrize("rec", golden_cases("reyes"), ids=lambda r: r["case"])
def test_matches_reference_golden(pk, ctx, rec):
    sc = scene_from(pk, rec)
    if sc is None:
        pytest.skip("reference fixture mesh not present on this host")
    fb, depth, st = render(pk, ctx, sc)
    assert st["prims_kept"] == rec["leaves"]
    assert st["upolys"] == rec["upolys"]
    assert st["split_levels"] == rec["levels"]
    assert sha(fb) == rec["fb_sha256"], "colour buffer differs from the reference"
    assert sha(depth) == rec["depth_sha256"], "depth buffer differs from the reference"


@pytest.mark.parametrize("thr,max_splits,grid", [(16.0, 10, 16), (16.0, 1, 2), (64.0, 3, 0)],
                         ids=["workload", "huge-upolys", "adaptive-grid"])
def test_workload_parameters_match_restatement(pk, ctx, oracle_mod, thr, max_splits, grid):
    """The Reyes workload's parameters (split below 16 px, at most 10 splits,
    fixed 16x16 dice grids; the reference hard-codes 4 px / 20 / adaptive), and
    two settings whose micropolygons span tens of pixels, which are shaded a
    warp per micropolygon."""
    sc = pk.scenes.sphere_patches()
    fb, depth, st = render(pk, ctx, sc, split_threshold_px=thr, max_splits=max_splits, dice_grid=grid)
    ofb, odepth, ost = oracle_mod.reyes_frame(sc, threshold=thr, max_splits=max_splits, grid=grid)
    assert st["prims_kept"] == ost["leaves"] and st["upolys"] == ost["upolys"]
    assert np.array_equal(depth.view(np.uint32), odepth.view(np.uint32))
    assert np.array_equal(fb, ofb)
    assert st["covered"] == ost["covered"]
    if max_splits < 10:
        assert st["bin_entries"] > 0, "no micropolygon took the warp path"


@pytest.mark.parametrize("seed", [31, 32, 33])
def test_random_spheres(pk, ctx, oracle_mod, seed):
    g = np.random.Generator(np.random.Philox(seed))
    W, H = int(g.integers(64, 400)), int(g.integers(64, 300))
    sc = pk.scenes.sphere_patches(W=W, H=H, seed=seed, amplitude=float(g.uniform(0.0, 0.3)))
    thr = float(g.choice([4.0, 8.0]))
    fb, depth, st = render(pk, ctx, sc, split_threshold_px=thr)
    ofb, odepth, ost = oracle_mod.reyes_frame(sc, threshold=thr)
    assert np.array_equal(fb, ofb)
    assert np.array_equal(depth.view(np.uint32), odepth.view(np.uint32))


def test_reference_interface_mirror(pk, ctx):
    rec = golden("reyes_sphere32_small")
    sc = scene_from(pk, rec)
    patches = np.zeros(sc.n, pk.piko_patch)
    patches["CP"] = sc.patches
    patches["id"] = np.arange(sc.n)
    cs = pk.ConstantState(sc.W, sc.H)
    cs.viewProjMatrix = sc.view_proj
    ms = pk.MutableState(sc.W, sc.H)
    pipe = pk.ReyesPipe(ctx)
    pipe.allocate(cs, ms, patches, sc.n)
    pipe.prepare()
    pipe.run_single()
    data = pipe.pikoScreen.getData()
    assert sha(data.reshape(sc.H, sc.W)) == rec["fb_sha256"]
    assert sha(ms.zBuffer.reshape(sc.H, sc.W)) == rec["depth_sha256"]
    pipe.destroy()
