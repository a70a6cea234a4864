"""Scene and mesh files without GL (piko_asset_*): the reference's .scene
commands with a CPU matrix stack, OBJ meshes in place of assimp, bezmesh .dat
patches; flattened as scene::flatten does.  Fixtures: tests/golden/assets,
written by tests/golden/make_assets.py."""
import os

import numpy as np
import pytest

ASSETS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "assets")


def path(name):
    return os.path.join(ASSETS, name)


def rot_y(deg):
    a = np.radians(deg)
    m = np.eye(4)
    m[0, 0], m[0, 2], m[2, 0], m[2, 2] = np.cos(a), np.sin(a), -np.sin(a), np.cos(a)
    return m


def tr(x, y, z):
    m = np.eye(4)
    m[:3, 3] = (x, y, z)
    return m


def sc(s):
    m = np.eye(4)
    m[0, 0] = m[1, 1] = m[2, 2] = s
    return m


def obj_fan(path_):
    """Fan-triangulated corner indices of an OBJ file, read independently."""
    V, faces = [], []
    for line in open(path_):
        t = line.split("#")[0].split()
        if not t:
            continue
        if t[0] == "v":
            V.append([float(x) for x in t[1:4]])
        elif t[0] == "f":
            idx = [int(c.split("/")[0]) for c in t[1:]]
            idx = [i - 1 if i > 0 else len(V) + i for i in idx]
            for k in range(1, len(idx) - 1):
                faces.append((idx[0], idx[k], idx[k + 1]))
    return np.array(V), faces


def test_obj_cube_fans_normals_and_uvs(pk):
    a = pk.Asset(path("cube.obj"))
    assert a.info["triangles"] == 12 and a.info["has_uv"] == 1 and a.info["has_camera"] == 0
    pos, nrm, col, uv = a.triangles()
    V, faces = obj_fan(path("cube.obj"))
    for t, f in enumerate(faces):
        for k in range(3):
            assert np.array_equal(pos[k, t, :3], V[f[k]].astype(np.float32))
    assert np.allclose(np.linalg.norm(nrm[:, :, :3], axis=-1), 1.0, atol=1e-6)
    # each quad's two triangles keep its face normal; the reference's fixed colour
    assert np.array_equal(nrm[0, 0, :3], [0, 0, -1]) and np.array_equal(nrm[2, 11, :3], [1, 0, 0])
    assert np.allclose(col[:, :, :3], [0.9, 0.9, 0.6])
    assert np.array_equal(uv[1, 0], [0.0, 1.0])


def test_obj_without_normals_gets_face_normals_and_negative_indices(pk):
    a = pk.Asset(path("tetra.obj"))
    pos, nrm, _, _ = a.triangles()
    assert a.info["triangles"] == 4
    V, faces = obj_fan(path("tetra.obj"))
    assert faces[-1] == (1, 2, 3)
    for t, f in enumerate(faces):
        n = np.cross(V[f[1]] - V[f[0]], V[f[2]] - V[f[0]])
        n /= np.linalg.norm(n)
        for k in range(3):
            assert np.allclose(nrm[k, t, :3], n, atol=1e-6)


def test_scene_commands_transforms_camera_and_materials(pk):
    from piko_b200 import camera
    a = pk.Asset(path("test.scene"))
    i = a.info
    assert (i["triangles"], i["patches"], i["lights"], i["materials"]) == (16, 2, 1, 2)
    assert np.isclose(i["fovy_rad"], np.radians(50.0)) and np.isclose(i["znear"], 0.1) and i["zfar"] == 50.0
    assert i["eye"] == [0.0, 1.0, 5.0] and i["light_pos"] == [2.0, 3.0, 4.0]
    pos, nrm, col, _ = a.triangles(colour_source=1)
    # cube under translate * rotate * scale (GL post-multiplication), tetra under translate
    M = tr(1, 0, 0) @ rot_y(30) @ sc(2)
    V, faces = obj_fan(path("cube.obj"))
    Nt = np.linalg.inv(M)[:3, :3].T
    for t, f in enumerate(faces):
        for k in range(3):
            p = (M @ np.append(V[f[k]], 1.0))[:3]
            assert np.allclose(pos[k, t, :3], p, rtol=0, atol=2e-7 * max(1.0, np.abs(p).max()))
        assert np.allclose(col[0, t, :3], [0.8, 0.2, 0.2])
    n0 = Nt @ np.array([0.0, 0.0, -1.0])
    assert np.allclose(nrm[0, 0, :3], n0 / np.linalg.norm(n0), atol=1e-6)
    Vt, ft = obj_fan(path("tetra.obj"))
    assert np.allclose(pos[0, 12:, :3], Vt[[f[0] for f in ft]] + [-1, 0, 0], atol=1e-7)
    assert np.allclose(col[0, 12:, :3], [0.2, 0.8, 0.2])
    # camera matrix as camera::updateCam builds it
    vp = camera.view_proj((0, 1, 5), (0, 0, 0), (0, 1, 0), np.radians(50.0), 64, 48, 0.1, 50.0)
    assert np.allclose(a.view_proj(64, 48), vp, rtol=1e-6, atol=1e-7)


def test_bez_patches_follow_the_bezmesh_reader(pk):
    a = pk.Asset(path("two_patches.dat"))
    p = a.patch_scene(64, 64).patches
    assert p.shape == (2, 16, 4)
    assert np.array_equal(p, pk.scenes.read_bez(path("two_patches.dat")))
    # in the scene file the patches come after `reset` and `scale [0.5 0.5 0.5]`
    s = pk.Asset(path("test.scene")).patch_scene(64, 64).patches
    assert np.allclose(s[:, :, :3], 0.5 * p[:, :, :3]) and np.all(s[:, :, 3] == 1.0)


def test_reference_teapot_fixture(pk):
    """The reference's own Reyes fixture (meshes/tpt.dat, 32 bicubic patches,
    copied into the assets by make_golden.py) reads the same through the C ABI
    loader and the bezmesh reader, and is the file the golden record was made
    from."""
    from helpers import golden, sha
    a = pk.Asset(path("tpt.dat"))
    assert a.info["patches"] == 32
    p = a.patch_scene(64, 64).patches
    q = pk.scenes.read_bez(path("tpt.dat"))
    assert np.array_equal(p, q)
    assert sha(q) == golden("reyes_teapot_tpt")["patches_sha256"]


@pytest.mark.parametrize("text,what", [("camera [ 0 0 1 ] [ 0 0 0 ]\n", "bad camera"),
                                       ("frobnicate 3\n", "unknown command"),
                                       ("loadmesh missing.obj\n", "cannot open"),
                                       ("loadmesh teapot.3DS\n", "only OBJ")])
def test_errors_are_reported(pk, tmp_path, text, what):
    f = tmp_path / "bad.scene"
    f.write_text(text)
    with pytest.raises(pk.PikoError) as e:
        pk.Asset(str(f))
    assert what in str(e.value)


@pytest.mark.gpu
def test_loaded_scene_renders_like_the_oracle(pk, ctx, oracle_mod):
    """The test scene's triangles through the device pipeline equal the
    oracle's frame on the same inputs, bit for bit."""
    a = pk.Asset(path("test.scene"))
    sc_ = a.raster_scene(320, 240)
    pipe = pk.Pipe(ctx, "raster")
    s = pk.Scene(pipe, sc_)
    try:
        s.run()
        fb, depth = s.read()
    finally:
        s.close()
        pipe.close()
    xyz, icol = oracle_mod.r1_setup(sc_)
    ofb, odepth, ost = oracle_mod.raster_frame(sc_.W, sc_.H, xyz, icol)
    assert ost["covered"] > 1000, "the test scene should cover part of the frame"
    assert np.array_equal(fb, ofb)
    assert np.array_equal(depth.view(np.uint32), odepth.view(np.uint32))


def test_bmp_writer_layout(pk, tmp_path):
    """24-bit BMP, bottom-up rows (the framebuffer's row 0 is the file's first
    row), rows padded to 4 bytes, B G R byte order."""
    H, W = 3, 5
    img = (np.arange(H * W, dtype=np.uint32) * 0x010203 + 0xFF000000).reshape(H, W)
    f = tmp_path / "t.bmp"
    pk.write_bmp(f, img)
    b = f.read_bytes()
    assert b[:2] == b"BM" and int.from_bytes(b[2:6], "little") == len(b)
    assert int.from_bytes(b[18:22], "little") == W and int.from_bytes(b[22:26], "little") == H
    assert int.from_bytes(b[28:30], "little") == 24
    row = (W * 3 + 3) & ~3
    for y in range(H):
        for x in range(W):
            c = int(img[y, x])
            o = 54 + y * row + 3 * x
            assert tuple(b[o:o + 3]) == ((c >> 16) & 255, (c >> 8) & 255, c & 255)
