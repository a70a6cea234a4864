"""The launch-configuration tuner of the batched form: scene-size buckets, the
configuration table (set / get / saved as plain data), and on the GPU that a
tuned batch -- scenes split into 8, 16 and 32 px launch groups on parallel
graph branches -- renders every scene exactly as the oracle does."""
import json

import numpy as np
import pytest


def test_buckets_follow_resolution_and_triangle_classes(pk):
    b = pk.tune_bucket
    assert b(256, 256, 1000) == 0
    assert b(256, 256, 4096) == 1
    assert b(512, 512, 20000) == 4 + 2
    assert b(1280, 720, 70000) == 8 + 3
    assert b(1920, 1080, 174000) == 12 + 3
    assert b(1920, 1080, 3000) == 12
    # every config of the 64-scene mix lands in a bucket in range
    for sc in pk.scenes.batch_mix(64):
        assert 0 <= b(sc.W, sc.H, sc.n) < 16


def test_table_round_trips_through_json(pk):
    t = pk.Tuner()
    assert t.table() == {}
    assert t.get(5)["tile_px"] == 8 and not t.get(5)["tuned"]
    t.set(5, 16, ctas_per_sm=1, ms=0.25)
    t.set(12, 8, chunk_entries=64, ms=1.5)
    saved = json.loads(json.dumps(t.table()))
    u = pk.Tuner(table=saved)
    assert u.table() == t.table()
    assert u.get(12)["chunk_entries"] == 64 and u.get(5)["ctas_per_sm"] == 1
    t.close()
    u.close()


def test_invalid_configurations_are_rejected(pk):
    t = pk.Tuner()
    with pytest.raises(pk.PikoError):
        t.set(3, 12)
    with pytest.raises(pk.PikoError):
        t.set(16, 8)
    with pytest.raises(pk.PikoError):
        t.set(2, 8, chunk_entries=-1)
    t.close()


def _mixed_scenes(pk):
    dims = [(3000, 256, 256), (20000, 512, 512), (500, 64, 96), (9000, 333, 197), (70000, 1280, 720),
            (1500, 512, 512), (30000, 256, 256)]
    return [pk.scenes.plain_scene(n=n, W=W, H=H, seed=40 + i, edge_median=0.04) for i, (n, W, H) in enumerate(dims)]


def _check_against_oracle(oracle_mod, scenes, scs):
    for s, sc in zip(scenes, scs):
        fb, depth = s.read()
        xyz, icol = oracle_mod.r1_setup(sc)
        ofb, odepth, _ = oracle_mod.raster_frame(sc.W, sc.H, xyz, icol)
        assert np.array_equal(fb, ofb), f"colour differs ({sc.n} triangles, {sc.W}x{sc.H})"
        assert np.array_equal(depth.view(np.uint32), odepth.view(np.uint32)), "depth differs"


@pytest.mark.gpu
def test_mixed_tile_groups_equal_the_oracle(pk, ctx, oracle_mod):
    scs = _mixed_scenes(pk)
    pipe = pk.Pipe(ctx, "raster")
    scenes = [pk.Scene(pipe, s) for s in scs]
    t = pk.Tuner()
    # force three launch groups: 8 px (chunk 16), 16 px and 32 px tiles
    for bucket in range(16):
        tile = (8, 16, 32)[bucket % 3]
        t.set(bucket, tile, ctas_per_sm=0, chunk_entries=16 if tile == 8 else 0)
    b = pk.Batch(ctx, scenes, tuner=t)
    try:
        for graph in (False, True, True):
            b.run(graph=graph)
            st = b.finish()
            assert st["status"] == 0
            _check_against_oracle(oracle_mod, scenes, scs)
    finally:
        b.close()
        t.close()
        for s in scenes:
            s.close()
        pipe.close()


@pytest.mark.gpu
def test_tuned_batch_equals_the_oracle(pk, ctx, oracle_mod):
    scs = _mixed_scenes(pk)
    pipe = pk.Pipe(ctx, "raster")
    scenes = [pk.Scene(pipe, s) for s in scs]
    t = pk.Tuner().tune(ctx, scenes, reps=3)
    table = t.table()
    assert set(table) == {pk.tune_bucket(s.W, s.H, s.n) for s in scs}
    assert all(c["ms"] > 0 and c["tile_px"] in (8, 16, 32) for c in table.values())
    b = pk.Batch(ctx, scenes, tuner=t)
    try:
        b.run(graph=True)
        b.finish()
        _check_against_oracle(oracle_mod, scenes, scs)
    finally:
        b.close()
        t.close()
        for s in scenes:
            s.close()
        pipe.close()
