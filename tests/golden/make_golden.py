"""Generates tests/golden/*.json from the reference's own stage code.

    python tests/golden/make_golden.py

Each case names a seeded scene (the generator and its arguments), runs the
reference pipeline built in place from its source tree (oracle/_ref, one CPU
thread; the Reyes workload's constants from the build with them substituted
into the split stage) and records the SHA-256 of the framebuffer and depth buffer bytes,
the reference's count of emitted Pixels, and a handful of sample pixels.  The
restatement in oracle/ and the device kernels are both checked against these
records, so the reference itself need not be present where the tests run.
"""
import hashlib
import json
import os
import shutil
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import piko_loader  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE = os.environ.get("PIKO_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))
# the reference's own Reyes fixture; copied into assets/ so that the tests
# (and the GPU host, which has no reference tree) can read it
TEAPOT_SRC = os.path.join(REFERENCE, "meshes", "tpt.dat")
TEAPOT = os.path.join(HERE, "assets", "tpt.dat")

RASTER_CASES = {
    "raster_plain4096_512": ("plain_scene", dict(n=4096, W=512, H=512, seed=0)),
    "raster_order_wrap_256": ("plain_scene", dict(n=40000, W=256, H=256, seed=3)),
    "raster_guard_giants": ("plain_scene", dict(n=3000, W=512, H=384, seed=4, edge_median=0.4, xy_range=1.3)),
    "raster_depth_ties": ("plain_scene", dict(n=5000, W=256, H=256, seed=5, flat_z=0.5, edge_median=0.1)),
    "raster_odd_size": ("plain_scene", dict(n=6000, W=333, H=197, seed=6, edge_median=0.05)),
    "raster_forest_gouraud": ("forest_scene", dict()),
}
REYES_CASES = {
    "reyes_sphere32_ref_constants": ("sphere_patches", dict()),
    "reyes_sphere32_small": ("sphere_patches", dict(W=320, H=192, seed=7)),
}
# the Reyes workload's constants (split below 16 px, at most 10 splits, fixed
# 16x16 dice grids), rendered by the reference build with those constants
# substituted into its split stage (oracle/_ref/libpiko_ref_reyes_c2.so)
REYES_C2_CONSTANTS = dict(split_threshold_px=16.0, max_splits=10, dice_grid=16)
REYES_C2_CASES = {
    "reyes_sphere32_c2_constants": ("sphere_patches", dict()),
}
BATCH_MIX = 64
# the raster pipe built without VTX_PRETRANSFORM (oracle/_ref/libpiko_ref_raster_world.so):
# world positions through the vertex stage's own transform; the reference sets
# no colours in that mode, so only depth and the emitted Pixel count are recorded
RASTER_WORLD_CASES = {
    "raster_world_forest": ("forest_scene", dict()),
    "raster_world_plain": ("plain_scene", dict(n=3000, W=320, H=240, seed=9, edge_median=0.06)),
}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def samples(fb, depth, k=16, seed=0):
    g = np.random.Generator(np.random.Philox(seed))
    H, W = fb.shape
    ys = g.integers(0, H, k)
    xs = g.integers(0, W, k)
    return [[int(x), int(y), int(fb[y, x]), int(depth.view(np.uint32)[y, x])] for x, y in zip(xs, ys)]


def make_scene(pk, gen, kw):
    if gen == "forest_scene":
        sc = pk.scenes.forest_scene(**kw)
        sc.uv = None        # the reference has no texturing: Gouraud only
        sc.texture = None
        return sc
    return getattr(pk.scenes, gen)(**kw)


def main():
    pk = piko_loader.load()
    import oracle
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref is not built: make -C oracle ref")
    for name, (gen, kw) in RASTER_CASES.items():
        sc = make_scene(pk, gen, kw)
        xyz, icol = oracle.r1_setup(sc)
        r = oracle.RefRaster(sc.W, sc.H, xyz, icol)
        r.frame(1)
        fb, depth = r.read()
        emitted = r.emitted()
        r.close()
        rec = dict(case=name, pipeline="raster", generator=gen, kwargs=kw, W=sc.W, H=sc.H, n=sc.n,
                   r1_sha256=sha(xyz) + ":" + sha(icol), fb_sha256=sha(fb), depth_sha256=sha(depth),
                   emitted=emitted, samples=samples(fb, depth))
        with open(os.path.join(HERE, name + ".json"), "w") as f:
            json.dump(rec, f, indent=1)
        print(name, emitted)
    for name, (gen, kw) in REYES_CASES.items():
        sc = make_scene(pk, gen, kw)
        r = oracle.RefReyes(sc)
        r.frame(1, record_leaves=True)
        fb, depth = r.read()
        c = r.counters()
        leaves = r.leaves()
        r.close()
        rec = dict(case=name, pipeline="reyes", generator=gen, kwargs=kw, W=sc.W, H=sc.H, n=sc.n,
                   fb_sha256=sha(fb), depth_sha256=sha(depth), emitted=c["emitted"], leaves=c["leaves"],
                   upolys=c["upolys"], levels=c["levels"], leaves_sha256=sha(leaves.astype(np.int32)),
                   samples=samples(fb, depth))
        with open(os.path.join(HERE, name + ".json"), "w") as f:
            json.dump(rec, f, indent=1)
        print(name, c)
    if oracle.ref_c2_available():
        for name, (gen, kw) in REYES_C2_CASES.items():
            sc = make_scene(pk, gen, kw)
            r = oracle.RefReyes(sc, workload_constants=True)
            r.frame(1, record_leaves=True)
            fb, depth = r.read()
            c = r.counters()
            leaves = r.leaves()
            r.close()
            rec = dict(case=name, pipeline="reyes", generator=gen, kwargs=kw, constants=REYES_C2_CONSTANTS,
                       W=sc.W, H=sc.H, n=sc.n, fb_sha256=sha(fb), depth_sha256=sha(depth), emitted=c["emitted"],
                       leaves=c["leaves"], upolys=c["upolys"], levels=c["levels"],
                       leaves_sha256=sha(leaves.astype(np.int32)), samples=samples(fb, depth))
            with open(os.path.join(HERE, name + ".json"), "w") as f:
                json.dump(rec, f, indent=1)
            print(name, c)
    if oracle.ref_world_available():
        for name, (gen, kw) in RASTER_WORLD_CASES.items():
            sc = make_scene(pk, gen, kw)
            xw = oracle.world_xyz(sc)
            r = oracle.RefRasterWorld(sc.W, sc.H, xw, sc.view_proj)
            r.frame(1)
            _, depth = r.read()
            emitted = r.emitted()
            r.close()
            rec = dict(case=name, pipeline="raster_world", generator=gen, kwargs=kw, W=sc.W, H=sc.H, n=sc.n,
                       world_sha256=sha(xw), view_proj=[float(v) for v in sc.view_proj],
                       depth_sha256=sha(depth), emitted=emitted)
            with open(os.path.join(HERE, name + ".json"), "w") as f:
                json.dump(rec, f, indent=1)
            print(name, emitted)
    # the batched form's 64-scene mix: one record per scene (its generator
    # arguments and the reference's digests), in one file
    mix = pk.scenes.batch_mix(BATCH_MIX)
    recs = []
    for i, sc in enumerate(mix):
        xyz, icol = oracle.r1_setup(sc)
        r = oracle.RefRaster(sc.W, sc.H, xyz, icol)
        r.frame(1)
        fb, depth = r.read()
        emitted = r.emitted()
        r.close()
        recs.append(dict(index=i, n=sc.n, W=sc.W, H=sc.H, kwargs=dict(n=sc.n, W=sc.W, H=sc.H, seed=i),
                         fb_sha256=sha(fb), depth_sha256=sha(depth), emitted=emitted))
    with open(os.path.join(HERE, "batch_mix64.json"), "w") as f:
        json.dump(dict(case="batch_mix64", pipeline="raster_batch", generator="batch_mix",
                       kwargs=dict(count=BATCH_MIX), scenes=recs), f, indent=1)
    print("batch_mix64", sum(r["emitted"] for r in recs))
    if os.path.exists(TEAPOT_SRC):
        # the reference's own Reyes fixture (its 32 teapot patches), copied
        # byte for byte so that the GPU tests can render it where the
        # reference tree is absent
        shutil.copyfile(TEAPOT_SRC, TEAPOT)
    if os.path.exists(TEAPOT):
        cps = pk.scenes.read_bez(TEAPOT)
        sc = pk.scenes.teapot_scene(cps)
        r = oracle.RefReyes(sc)
        r.frame(1)
        fb, depth = r.read()
        c = r.counters()
        r.close()
        rec = dict(case="reyes_teapot_tpt", pipeline="reyes", generator="teapot_scene", kwargs={}, W=sc.W, H=sc.H,
                   n=sc.n, patches_sha256=sha(cps), fb_sha256=sha(fb), depth_sha256=sha(depth),
                   emitted=c["emitted"], leaves=c["leaves"], upolys=c["upolys"], levels=c["levels"],
                   samples=samples(fb, depth))
        with open(os.path.join(HERE, "reyes_teapot_tpt.json"), "w") as f:
            json.dump(rec, f, indent=1)
        print("teapot", c)


if __name__ == "__main__":
    main()
