"""The oracle's C restatement, pinned to the reference's own stage code.

Two anchors: the committed golden records (made by tests/golden/make_golden.py
from the reference pipeline compiled in place), and, where oracle/_ref is
built, a live comparison with the reference on the same inputs."""
import numpy as np
import pytest

from helpers import golden_cases, masks_from_pixels, scene_from, sha


@pytest.mark.parametrize("rec", golden_cases("raster"), ids=lambda r: r["case"])
def test_raster_restatement_matches_golden(pk, oracle_mod, rec):
    sc = scene_from(pk, rec)
    xyz, icol = oracle_mod.r1_setup(sc)
    assert sha(xyz) + ":" + sha(icol) == rec["r1_sha256"]
    fb, depth, st = oracle_mod.raster_frame(sc.W, sc.H, xyz, icol)
    assert sha(fb) == rec["fb_sha256"]
    assert sha(depth) == rec["depth_sha256"]
    assert st["passed"] == rec["emitted"]
    for x, y, c, d in rec["samples"]:
        assert int(fb[y, x]) == c and int(depth.view(np.uint32)[y, x]) == d


@pytest.mark.parametrize("rec", golden_cases("reyes"), ids=lambda r: r["case"])
def test_reyes_restatement_matches_golden(pk, oracle_mod, rec):
    sc = scene_from(pk, rec)
    assert sc is not None, "fixture mesh missing"
    c = rec.get("constants", {})
    fb, depth, st = oracle_mod.reyes_frame(sc, threshold=c.get("split_threshold_px", 4.0),
                                           max_splits=c.get("max_splits", 20), grid=c.get("dice_grid", 0),
                                           leaf_cap=1 << 20)
    assert sha(fb) == rec["fb_sha256"]
    assert sha(depth) == rec["depth_sha256"]
    assert st["passed"] == rec["emitted"]
    assert st["leaves"] == rec["leaves"] and st["upolys"] == rec["upolys"] and st["levels"] == rec["levels"]
    if "leaves_sha256" in rec:
        # leaves in the order Split emits them (the restatement lists Dice order)
        assert st["hangs"] == 0


def _ref_or_skip(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built here")


def test_live_reference_raster_random_sizes(pk, oracle_mod):
    _ref_or_skip(oracle_mod)
    for seed, (n, W, H) in enumerate([(700, 64, 48), (2500, 128, 96), (9000, 200, 120)]):
        sc = pk.scenes.plain_scene(n=n, W=W, H=H, seed=100 + seed, edge_median=0.08)
        xyz, icol = oracle_mod.r1_setup(sc)
        fb, depth, st = oracle_mod.raster_frame(W, H, xyz, icol)
        r = oracle_mod.RefRaster(W, H, xyz, icol)
        r.frame(1)
        fb2, d2 = r.read()
        emitted = r.emitted()
        r.close()
        assert np.array_equal(fb, fb2)
        assert np.array_equal(depth.view(np.uint32), d2.view(np.uint32))
        assert emitted == st["passed"]


def test_live_reference_coverage_masks(pk, oracle_mod):
    """Per-triangle coverage of the restatement == what the reference's own
    RasterStage::process emits for that triangle alone."""
    _ref_or_skip(oracle_mod)
    sc = pk.scenes.plain_scene(n=600, W=256, H=256, seed=11, edge_median=0.15, xy_range=1.2)
    xyz, icol = oracle_mod.r1_setup(sc)
    tri, binv, mask = oracle_mod.raster_coverage(sc.W, sc.H, xyz, icol)
    ours = {(int(t), int(b)): int(m) for t, b, m in zip(tri, binv, mask)}
    r = oracle_mod.RefRaster(sc.W, sc.H, xyz, icol)
    try:
        for t in range(0, 600, 3):
            xy = r.coverage(t)
            pix = (xy[:, 1] * sc.W + xy[:, 0]).astype(np.int64)
            ref = masks_from_pixels(np.full(len(pix), t), pix, sc.W)
            mine = {k: v for k, v in ours.items() if k[0] == t}
            assert ref == mine, t
    finally:
        r.close()


def test_live_reference_reyes_parameters(pk, oracle_mod):
    """Reyes restatement == reference on a second seed, and the split/dice
    generalisation collapses to the reference at its own constants."""
    _ref_or_skip(oracle_mod)
    sc = pk.scenes.sphere_patches(W=256, H=160, seed=21)
    fb, depth, st = oracle_mod.reyes_frame(sc, threshold=4.0, max_splits=20, grid=0, leaf_cap=1 << 20)
    r = oracle_mod.RefReyes(sc)
    try:
        r.frame(1, record_leaves=True)
        fb2, d2 = r.read()
        c = r.counters()
        leaves = r.leaves()
    finally:
        r.close()
    assert np.array_equal(fb, fb2)
    assert np.array_equal(depth.view(np.uint32), d2.view(np.uint32))
    assert c["leaves"] == st["leaves"] and c["upolys"] == st["upolys"]
    # same multiset of leaves (Split emission order vs Dice processing order)
    a = sorted(map(tuple, leaves.tolist()))
    b = sorted(map(tuple, st["leaf_list"].tolist()))
    assert a == b


def test_restated_r1_matches_numpy_float32(pk, oracle_mod):
    """R1's viewport transform, restated in C, agrees with a float32 numpy
    evaluation of the same left-to-right expression on the identity camera."""
    sc = pk.scenes.plain_scene(n=256, W=320, H=200, seed=9)
    xyz, icol = oracle_mod.r1_setup(sc)
    x = sc.pos[:, :, 0].T.astype(np.float32)
    halfW = np.float32(0.5) * np.float32(320)
    ref = (x * np.float32(1.0) + np.float32(1.0)) * halfW
    assert np.array_equal(xyz[:, 0::3], ref)
    assert np.all((icol >> 24) == 0xFF)


def test_multisample_restatement_reduces_to_the_pinned_one(pk, oracle_mod):
    """The oracle's multi-sample / Phong Reyes variant with one centre sample
    and the reference's shading is the pinned restatement, bit for bit; with 4
    samples the jitter is seeded (same seed, same image; another seed, another
    sample pattern)."""
    rec = [r for r in golden_cases("reyes") if r["case"] == "reyes_sphere32_small"][0]
    sc = scene_from(pk, rec)
    fb, depth, st = oracle_mod.reyes_frame(sc)
    fb1, depth1, st1 = oracle_mod.reyes_frame_ms(sc, spp=1, seed=99, phong=False)
    assert np.array_equal(fb, fb1) and np.array_equal(depth.view(np.uint32), depth1.view(np.uint32))
    assert st == st1
    a = oracle_mod.reyes_frame_ms(sc, spp=4, seed=1, phong=True)
    b = oracle_mod.reyes_frame_ms(sc, spp=4, seed=1, phong=True)
    c = oracle_mod.reyes_frame_ms(sc, spp=4, seed=2, phong=True)
    assert np.array_equal(a[0], b[0]) and a[2] == b[2]
    assert a[2]["covered"] != c[2]["covered"] or not np.array_equal(a[0], c[0])
    # about four times the samples of the one-sample frame
    assert 3.5 * st["covered"] < a[2]["covered"] < 4.5 * st["covered"]
