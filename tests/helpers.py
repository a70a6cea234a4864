"""Shared helpers of the test suite (golden records, scene rebuild, digests)."""
import glob
import hashlib
import json
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# the reference's Reyes fixture (meshes/tpt.dat), copied by make_golden.py
TEAPOT = os.path.join(GOLDEN_DIR, "assets", "tpt.dat")


def golden(name):
    with open(os.path.join(GOLDEN_DIR, name + ".json")) as f:
        return json.load(f)


def golden_cases(pipeline):
    out = []
    for p in sorted(glob.glob(os.path.join(GOLDEN_DIR, "*.json"))):
        with open(p) as f:
            rec = json.load(f)
        if rec["pipeline"] == pipeline:
            out.append(rec)
    return out


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def scene_from(pk, rec, textured=False):
    """Rebuilds the seeded scene of a golden record (None if its data is absent)."""
    gen, kw = rec["generator"], rec["kwargs"]
    if gen == "teapot_scene":
        if not os.path.exists(TEAPOT):
            return None
        return pk.scenes.teapot_scene(pk.scenes.read_bez(TEAPOT))
    sc = getattr(pk.scenes, gen)(**kw)
    if gen == "forest_scene" and not textured:
        sc.uv = None
        sc.texture = None
    return sc


def masks_from_pixels(tri, pix, W):
    """{(tri, 8x8 bin): 64-bit mask} from (triangle, pixel index) samples."""
    nBx = W // 8
    x = pix % W
    y = pix // W
    b = (y // 8) * nBx + (x // 8)
    bit = (y % 8) * 8 + (x % 8)
    out = {}
    for t, bb, k in zip(tri.tolist(), b.tolist(), bit.tolist()):
        out[(t, bb)] = out.get((t, bb), 0) | (1 << k)
    return out
