"""Served form: requests that arrive while others are on the GPU are batched and
overlap on the device, and every request's image equals the image of the same
request rendered alone (bit for bit: coverage, depth and colour)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_each_request_equals_rendering_alone(pk):
    from piko_b200 import serve
    ctx = pk.Context()
    rpipe = pk.Pipe(ctx, "raster")
    ypipe = pk.Pipe(ctx, "reyes", split_threshold_px=16.0, max_splits=10, dice_grid=16)
    rsc = [pk.scenes.plain_scene(n=n, W=W, H=H, seed=40 + i, edge_median=0.05)
           for i, (n, W, H) in enumerate([(3000, 256, 256), (20000, 640, 360), (800, 96, 64)])]
    ysc = [pk.scenes.sphere_patches(W=320, H=192, seed=41)]
    rs = [pk.Scene(rpipe, s) for s in rsc]
    ys = [pk.Scene(ypipe, s) for s in ysc]
    server = pk.Server(ctx, lanes=3, max_batch=8, max_slots=64, max_pixels=640 * 360)
    try:
        stream = serve.make_stream(seed=5, n_raster_scenes=len(rs), rate_hz=2000.0, seconds=0.03)
        assert len(stream) >= 20
        ids, states = serve.replay(server, stream, rs, ys, keep=True)
        server.drain()
        st = server.stats()
        assert st["completed"] == len(stream) and st["failed"] == 0
        assert st["p50_ms"] > 0 and st["p99_ms"] >= st["p50_ms"]
        for k, (rid, (t, kind, i, _), state) in enumerate(zip(ids, stream, states)):
            scene = rs[i] if kind == "raster" else ys[i]
            fb, depth = server.read(rid, scene.W, scene.H)
            scene.prepare(state)
            try:
                scene.run()
                afb, adepth = scene.read()
            except pk.PikoError as e:
                raise AssertionError(f"request {k} ({kind} scene {i}) rendered alone: {e}") from e
            assert np.array_equal(fb, afb), (kind, i)
            assert np.array_equal(depth.view(np.uint32), adepth.view(np.uint32)), (kind, i)
    finally:
        server.close()
        for s in rs + ys:
            s.close()
        rpipe.close()
        ypipe.close()
        ctx.close()


def test_admission_respects_slot_limit(pk):
    """With fewer output slots than queued requests, requests wait for slots
    instead of failing, and all complete."""
    ctx = pk.Context()
    pipe = pk.Pipe(ctx, "raster")
    sc = pk.Scene(pipe, pk.scenes.plain_scene(n=2000, W=128, H=128, seed=3))
    server = pk.Server(ctx, lanes=2, max_batch=4, max_slots=2, max_pixels=128 * 128)
    try:
        cs = pk.const_state()
        ids = [server.submit(sc, cs) for _ in range(50)]
        server.drain()
        st = server.stats()
        assert st["completed"] == 50 and st["slots"] <= 2
        assert ids == sorted(ids)
    finally:
        server.close()
        sc.close()
        pipe.close()
        ctx.close()
