"""Seeded workload generators: sizes, layouts and determinism."""
import numpy as np


def test_plain_case_shapes(pk):
    sc = pk.scenes.plain_scene()
    assert sc.n == 4096 and (sc.W, sc.H) == (512, 512)
    assert sc.pos.shape == (3, 4096, 4) and sc.pos.dtype == np.float32
    assert np.all(sc.pos[:, :, 3] == 1.0)
    assert np.all((sc.pos[:, :, 2] >= 0.1) & (sc.pos[:, :, 2] <= 0.9))
    n = np.linalg.norm(sc.nrm[:, :, :3], axis=2)
    assert np.allclose(n, 1.0, atol=1e-5)
    again = pk.scenes.plain_scene()
    assert np.array_equal(sc.pos, again.pos) and np.array_equal(sc.col, again.col)


def test_forest_has_174000_triangles(pk):
    sc = pk.scenes.forest_scene()
    assert sc.n == 174000 == pk.scenes.FOREST_TRIS
    assert (sc.W, sc.H) == (1920, 1080)
    assert sc.texture.shape == (512, 512, 4) and sc.uv.shape == (3, 174000, 2)
    assert sc.light_mode == pk.scenes.LIGHT_EYE


def test_batch_mix_distribution(pk):
    mix = pk.scenes.batch_mix(count=64)
    assert len(mix) == 64
    ns = np.array([s.n for s in mix])
    assert ns.min() >= 1000 and ns.max() <= 200000
    sizes = {(s.W, s.H) for s in mix}
    assert sizes <= {(256, 256), (512, 512), (1280, 720), (1920, 1080)}
    assert len(sizes) >= 3


def test_sphere_patches(pk):
    sc = pk.scenes.sphere_patches()
    assert sc.patches.shape == (32, 16, 4) and (sc.W, sc.H) == (1280, 720)
    r = np.linalg.norm(sc.patches[:, :, :3], axis=2)
    assert r.min() > 0.8 and r.max() < 1.2


def test_no_colour_array_means_the_reference_material_colour(pk, oracle_mod):
    """col None (no colour array uploaded) lights every vertex with the
    reference's fixed material colour (0.9, 0.9, 0.6), main.cpp:380-386: the
    oracle's R1 equals the one given that colour explicitly, bit for bit."""
    import copy
    sc = pk.scenes.plain_scene(n=3000, W=256, H=192, seed=4)
    sc.col = None
    explicit = copy.copy(sc)
    explicit.col = np.ones((3, sc.n, 4), np.float32)
    explicit.col[:, :, :3] = pk.scenes.REF_MATCOL
    xyz0, icol0 = oracle_mod.r1_setup(sc)
    xyz1, icol1 = oracle_mod.r1_setup(explicit)
    assert np.array_equal(xyz0.view(np.uint32), xyz1.view(np.uint32))
    assert np.array_equal(icol0, icol1)
    assert sc.attribute_bytes() == explicit.attribute_bytes() - explicit.col.nbytes
