"""Device raster path vs the oracle: bit-exact framebuffer, depth buffer,
coverage and fragment counts, through the C ABI."""
import numpy as np
import pytest

from helpers import golden_cases, masks_from_pixels, scene_from, sha

pytestmark = pytest.mark.gpu


def render(pk, ctx, sc, tile=16, **kw):
    pipe = pk.Pipe(ctx, "raster", tile_px=tile, **kw)
    s = pk.Scene(pipe, sc)
    try:
        s.run()
        fb, depth = s.read()
        st = s.stats()
    finally:
        s.close()
        pipe.close()
    return fb, depth, st


@pytest.mark.parametrize("rec", golden_cases("raster"), ids=lambda r: r["case"])
def test_matches_reference_golden(pk, ctx, oracle_mod, rec):
    sc = scene_from(pk, rec)
    fb, depth, st = render(pk, ctx, sc)
    assert sha(fb) == rec["fb_sha256"], "colour buffer differs from the reference"
    assert sha(depth) == rec["depth_sha256"], "depth buffer differs from the reference"
    xyz, icol = oracle_mod.r1_setup(sc)
    _, _, ost = oracle_mod.raster_frame(sc.W, sc.H, xyz, icol)
    assert st["prims_kept"] == ost["kept"]
    assert st["covered"] == ost["covered"], "fragment count differs"


@pytest.mark.parametrize("tile", [8, 32])
@pytest.mark.parametrize("case", ["raster_plain4096_512", "raster_guard_giants", "raster_odd_size"])
def test_tile_sizes_agree(pk, ctx, tile, case):
    from helpers import golden
    rec = golden(case)
    sc = scene_from(pk, rec)
    fb, depth, st = render(pk, ctx, sc, tile=tile)
    assert sha(fb) == rec["fb_sha256"] and sha(depth) == rec["depth_sha256"]


@pytest.mark.parametrize("case", ["raster_plain4096_512", "raster_guard_giants", "raster_order_wrap_256"])
def test_coverage_masks_match_oracle(pk, ctx, oracle_mod, case):
    from helpers import golden
    sc = scene_from(pk, golden(case))
    pipe = pk.Pipe(ctx, "raster")
    s = pk.Scene(pipe, sc)
    try:
        tri, pix, n = s.coverage(cap=1 << 24)
    finally:
        s.close()
        pipe.close()
    assert n == len(tri)
    gpu = masks_from_pixels(tri.astype(np.int64), pix.astype(np.int64), sc.W)
    xyz, icol = oracle_mod.r1_setup(sc)
    t, b, m = oracle_mod.raster_coverage(sc.W, sc.H, xyz, icol)
    ref = {(int(a), int(c)): int(d) for a, c, d in zip(t, b, m)}
    assert gpu == ref


def test_pretransformed_wtri_input(pk, ctx, oracle_mod):
    """The reference's own input format (raster_wtri) gives the same frame."""
    from helpers import golden
    rec = golden("raster_plain4096_512")
    sc = scene_from(pk, rec)
    xyz, icol = oracle_mod.r1_setup(sc)
    fb, depth, _ = render(pk, ctx, {"W": sc.W, "H": sc.H, "xyz": xyz, "icol": icol})
    assert sha(fb) == rec["fb_sha256"] and sha(depth) == rec["depth_sha256"]


def test_textured_forest_matches_restatement(pk, ctx, oracle_mod):
    """Textured variant (no reference counterpart): coverage and depth pinned to
    the reference through the Gouraud golden, colour to the restatement, which
    the kernel reproduces exactly (the tolerance of 1/255 is not needed)."""
    from helpers import golden
    sc = pk.scenes.forest_scene()
    fb, depth, _ = render(pk, ctx, sc)
    ofb, odepth, _ = oracle_mod.raster_scene(sc)
    assert np.array_equal(depth.view(np.uint32), odepth.view(np.uint32))
    assert sha(depth) == golden("raster_forest_gouraud")["depth_sha256"]
    diff = np.abs(fb.view(np.uint8).astype(int) - ofb.view(np.uint8).astype(int)).max()
    assert diff <= 1
    assert np.array_equal(fb, ofb)


@pytest.mark.parametrize("seed", range(6))
def test_random_small_scenes(pk, ctx, oracle_mod, seed):
    g = np.random.Generator(np.random.Philox(1000 + seed))
    W = int(g.integers(32, 300))
    H = int(g.integers(32, 300))
    n = int(g.integers(1, 20000))
    sc = pk.scenes.plain_scene(n=n, W=W, H=H, seed=seed, edge_median=float(g.uniform(0.01, 0.6)),
                               xy_range=float(g.uniform(0.5, 1.4)), flat_z=0.25 if seed % 3 == 0 else None)
    fb, depth, st = render(pk, ctx, sc, tile=int(g.choice([8, 16, 32])))
    xyz, icol = oracle_mod.r1_setup(sc)
    ofb, odepth, ost = oracle_mod.raster_frame(W, H, xyz, icol)
    assert np.array_equal(fb, ofb)
    assert np.array_equal(depth.view(np.uint32), odepth.view(np.uint32))
    assert st["covered"] == ost["covered"]


def test_empty_scene_clears(pk, ctx):
    sc = pk.scenes.plain_scene(n=0, W=64, H=64, seed=0)
    fb, depth, st = render(pk, ctx, sc)
    assert np.all(fb == 0xFF663313) and np.all(depth == 1.0)
    assert st["covered"] == 0


def test_batch_equals_alone(pk, ctx, oracle_mod):
    """Every scene of a batched launch (and of its graph replay) renders exactly
    as it does alone."""
    scs = [pk.scenes.plain_scene(n=n, W=W, H=H, seed=i, edge_median=0.05)
           for i, (n, W, H) in enumerate([(3000, 256, 256), (20000, 512, 512), (500, 64, 96), (9000, 333, 197)])]
    pipe = pk.Pipe(ctx, "raster")
    scenes = [pk.Scene(pipe, s) for s in scs]
    b = pk.Batch(ctx, scenes)
    try:
        for graph in (False, True, True):
            b.run(graph=graph)
            b.finish()
            for s, sc in zip(scenes, scs):
                fb, depth = s.read()
                xyz, icol = oracle_mod.r1_setup(sc)
                ofb, odepth, _ = oracle_mod.raster_frame(sc.W, sc.H, xyz, icol)
                assert np.array_equal(fb, ofb)
                assert np.array_equal(depth.view(np.uint32), odepth.view(np.uint32))
    finally:
        b.close()
        for s in scenes:
            s.close()
        pipe.close()


def test_reference_interface_mirror(pk, ctx, oracle_mod):
    """allocate / prepare / run_single / pikoScreen.getData as the reference's
    main.cpp drives them, on the raster_wtri input of the plain case."""
    from helpers import golden
    rec = golden("raster_plain4096_512")
    sc = scene_from(pk, rec)
    xyz, icol = oracle_mod.r1_setup(sc)
    tris = np.zeros(sc.n, pk.raster_wtri)
    tris["id"] = np.arange(sc.n)
    tris["worldPos0"], tris["worldPos1"], tris["worldPos2"] = xyz[:, 0:3], xyz[:, 3:6], xyz[:, 6:9]
    tris["icol0"], tris["icol1"], tris["icol2"] = icol[:, 0], icol[:, 1], icol[:, 2]
    cs = pk.ConstantState(sc.W, sc.H)
    ms = pk.MutableState(sc.W, sc.H)
    pipe = pk.RasterPipe(ctx)
    pipe.allocate(cs, ms, tris, sc.n)
    for _ in range(2):
        pipe.prepare()
        pipe.run_single()
        data = pipe.pikoScreen.getData()
        assert sha(data.reshape(sc.H, sc.W)) == rec["fb_sha256"]
        assert sha(ms.zBuffer.reshape(sc.H, sc.W)) == rec["depth_sha256"]
    pipe.destroy()


def test_queue_overflow_is_retried(pk, ctx, oracle_mod):
    """A frame whose bin lists outgrow the first capacity guess is re-rendered
    with grown queues and still matches (guard-band giants cover many tiles)."""
    from helpers import golden
    rec = golden("raster_guard_giants")
    sc = scene_from(pk, rec)
    fb, depth, st = render(pk, ctx, sc, tile=8)
    assert sha(fb) == rec["fb_sha256"]
    assert st["bin_entries"] > 4 * sc.n


def test_no_colour_array_matches_explicit_material_colour(pk, ctx, oracle_mod):
    """A triangle scene without a colour array renders as with every vertex
    given the reference's fixed material colour, and as the oracle does."""
    import copy
    sc = pk.scenes.plain_scene(n=5000, W=320, H=240, seed=6)
    sc.col = None
    explicit = copy.copy(sc)
    explicit.col = np.ones((3, sc.n, 4), np.float32)
    explicit.col[:, :, :3] = pk.scenes.REF_MATCOL
    fb0, depth0, _ = render(pk, ctx, sc)
    fb1, depth1, _ = render(pk, ctx, explicit)
    assert np.array_equal(fb0, fb1) and np.array_equal(depth0.view(np.uint32), depth1.view(np.uint32))
    ofb, odepth, _ = oracle_mod.raster_scene(sc)
    assert np.array_equal(fb0, ofb) and np.array_equal(depth0.view(np.uint32), odepth.view(np.uint32))


@pytest.mark.parametrize("case", ["raster_plain4096_512", "raster_guard_giants"])
def test_packed_float3_input_equals_float4(pk, ctx, case):
    """Positions and normals uploaded as float3 (piko_scene_desc.packed) draw
    the reference's golden image, and a re-upload keeps the layout."""
    from helpers import golden
    rec = golden(case)
    sc = scene_from(pk, rec)
    pipe = pk.Pipe(ctx, "raster", tile_px=8)
    s = pk.Scene(pipe, sc, packed=True)
    try:
        s.run()
        fb, depth = s.read()
        assert sha(fb) == rec["fb_sha256"] and sha(depth) == rec["depth_sha256"]
        s.upload(sc)
        s.run()
        fb2, depth2 = s.read()
        assert np.array_equal(fb2, fb) and np.array_equal(depth2.view(np.uint32), depth.view(np.uint32))
    finally:
        s.close()
        pipe.close()


def test_packed_textured_forest_equals_float4(pk, ctx):
    sc = pk.scenes.forest_scene()
    fb, depth, _ = render(pk, ctx, sc, tile=8)
    pipe = pk.Pipe(ctx, "raster", tile_px=8)
    s = pk.Scene(pipe, sc, packed=True)
    try:
        s.run()
        pfb, pdepth = s.read()
    finally:
        s.close()
        pipe.close()
    assert np.array_equal(pfb, fb) and np.array_equal(pdepth.view(np.uint32), depth.view(np.uint32))
