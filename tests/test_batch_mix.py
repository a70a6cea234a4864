"""The batched form's 64-scene mix (1K-200K triangles per scene, 256^2 to
1920x1080, seeds 0..63) against the reference's own digests
(tests/golden/batch_mix64.json, made by make_golden.py from the reference
build, one CPU thread).  The mix holds 200K-triangle scenes at 256^2, where the
reference's submission order wraps over its vertex-shader bins many times
(pikoc/api/include/internal/datatypes.h:88-93), and the tuned batch splits it
into launch groups of different tile sizes.

CPU: the oracle's restatement equals every scene's reference digest.
GPU: the tuned batch (graph replay), the single-configuration batch and the
plain per-scene path all equal the same digests."""
import numpy as np
import pytest

from helpers import golden, sha


def _mix(pk):
    rec = golden("batch_mix64")
    mix = pk.scenes.batch_mix(rec["kwargs"]["count"])
    for sc, r in zip(mix, rec["scenes"]):
        assert (sc.n, sc.W, sc.H) == (r["n"], r["W"], r["H"])
    return rec, mix


def test_restatement_matches_reference_digests(pk, oracle_mod):
    rec, mix = _mix(pk)
    for sc, r in zip(mix, rec["scenes"]):
        xyz, icol = oracle_mod.r1_setup(sc)
        fb, depth, st = oracle_mod.raster_frame(sc.W, sc.H, xyz, icol)
        assert sha(fb) == r["fb_sha256"], f"scene {r['index']}: colour"
        assert sha(depth) == r["depth_sha256"], f"scene {r['index']}: depth"
        assert st["passed"] == r["emitted"]


def _check(scenes, rec, what):
    bad = []
    for i, (s, r) in enumerate(zip(scenes, rec["scenes"])):
        fb, depth = s.read()
        if sha(fb) != r["fb_sha256"] or sha(depth) != r["depth_sha256"]:
            bad.append(i)
    assert not bad, f"{what}: scenes {bad} differ from the reference"


@pytest.mark.gpu
def test_tuned_batch_of_the_mix_matches_reference(pk, ctx):
    rec, mix = _mix(pk)
    pipe = pk.Pipe(ctx, "raster")
    scenes = [pk.Scene(pipe, s) for s in mix]
    t = pk.Tuner().tune(ctx, scenes, reps=3)
    b = pk.Batch(ctx, scenes, tuner=t)
    u = pk.Batch(ctx, scenes)
    try:
        for graph in (False, True, True):
            b.run(graph=graph)
            st = b.finish()
            assert st["status"] == 0
            _check(scenes, rec, f"tuned batch (graph={graph})")
        u.run(graph=True)
        u.finish()
        _check(scenes, rec, "single-configuration batch")
        for s in scenes:
            s.run()
        _check(scenes, rec, "plain per-scene frames")
    finally:
        b.close()
        u.close()
        t.close()
        for s in scenes:
            s.close()
        pipe.close()
