"""Seeded synthetic scenes for the raster and Reyes pipelines.

The reference renders scenes parsed from ``.scene`` files through assimp (whose
library is not shipped) and a GL matrix stack; there is no dataset here, so the
workloads are generated from a counter-based PRNG (numpy's Philox4x32-10), with
the sizes and value distributions of the workloads being measured:

* :func:`plain_scene`   - the plain binned-raster case: clip-space triangles
  (x, y ~ U[-1, 1], z ~ U[0.1, 0.9], w = 1) with log-normal edge length
  (median 0.02 NDC, sigma 0.8), random unit normals, RGB ~ U[0, 1], one fixed
  directional light.  4,096 triangles at 512x512 with seed 0 is the small case
  the reference itself renders on the CPU; the same generator with other
  seeds, counts and resolutions builds the 64-scene batched mix.
* :func:`forest_scene`  - the scene-scale raster case: 1,700 cones (102
  triangles each) and 300 quads = 174,000 triangles on a 100x100 ground grid,
  heights log-normal (median 1, sigma 0.6), positions, normals and UVs,
  a 60-degree perspective camera at 1920x1080 and a seeded 512x512 RGBA8
  noise texture.
* :func:`sphere_patches` - the Reyes case: 32 bicubic Bezier patches laid out
  like a unit sphere (8 longitude x 4 latitude bands) with a seeded smooth
  radial deformation of amplitude 0.15, 1280x720.

Vertex attributes are structure-of-arrays per vertex slot: ``pos[k, t]`` is the
float4 position of vertex ``k`` (0..2) of triangle ``t``, so that thread ``t`` of
a warp reading slot ``k`` makes one coalesced 16-byte access.
"""
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import camera

LIGHT_DIRECTIONAL = 0   # the same light vector for every vertex
LIGHT_EYE = 1           # light vector = normalize(eye - vertex), as main.cpp:372-378

# the reference's fixed light vector and material colour (main.cpp:383-384)
REF_LIGHT = (0.5773, 0.5773, 0.5773)
REF_MATCOL = (0.9, 0.9, 0.6)


def _rng(seed):
    return np.random.Generator(np.random.Philox(int(seed)))


@dataclass
class RasterScene:
    W: int
    H: int
    pos: np.ndarray                    # float32 [3, N, 4]
    nrm: np.ndarray                    # float32 [3, N, 4]
    col: Optional[np.ndarray]          # float32 [3, N, 4] material colour per vertex;
                                       # None: the reference's fixed (0.9, 0.9, 0.6)
    view_proj: np.ndarray              # float32 [16], column-major
    light_mode: int = LIGHT_DIRECTIONAL
    light: np.ndarray = field(default_factory=lambda: np.array(REF_LIGHT, np.float32))
    eye: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))
    uv: Optional[np.ndarray] = None    # float32 [3, N, 2]
    texture: Optional[np.ndarray] = None  # uint8 [TH, TW, 4]
    name: str = "scene"

    @property
    def n(self):
        return int(self.pos.shape[1])

    def attribute_bytes(self):
        """Bytes of vertex attributes the setup kernel consumes per frame."""
        b = self.pos.nbytes + self.nrm.nbytes
        if self.uv is not None:
            b += self.uv.nbytes
        if self.col is not None:
            b += self.col.nbytes
        return b


@dataclass
class PatchScene:
    W: int
    H: int
    patches: np.ndarray                # float32 [P, 16, 4] control points (w = 1)
    view_proj: np.ndarray              # float32 [16]
    name: str = "patches"

    @property
    def n(self):
        return int(self.patches.shape[0])


def plain_scene(n=4096, W=512, H=512, seed=0, edge_median=0.02, edge_sigma=0.8, flat_z=None, xy_range=1.0):
    """Clip-space triangles of the plain rasterizer case (identity camera).

    edge_median / edge_sigma set the log-normal edge length in NDC; flat_z
    puts every vertex at one depth (every overlap is a depth tie); xy_range
    widens the centroid range past the screen into the guard band."""
    g = _rng(seed)
    cx = g.uniform(-xy_range, xy_range, n)
    cy = g.uniform(-xy_range, xy_range, n)
    z = g.uniform(0.1, 0.9, (3, n))
    if flat_z is not None:
        z[:] = flat_z
    ell = g.lognormal(np.log(edge_median), edge_sigma, n)
    theta0 = g.uniform(0.0, 2.0 * np.pi, n)
    jitter = g.uniform(-0.35, 0.35, (3, n))
    winding = np.where(g.uniform(0.0, 1.0, n) < 0.5, -1.0, 1.0)
    r = ell / np.sqrt(3.0)  # circumradius of a triangle with edge ell
    pos = np.zeros((3, n, 4), np.float64)
    for k in range(3):
        a = theta0 + winding * (k * 2.0 * np.pi / 3.0) + jitter[k]
        pos[k, :, 0] = cx + r * np.cos(a)
        pos[k, :, 1] = cy + r * np.sin(a)
        pos[k, :, 2] = z[k]
        pos[k, :, 3] = 1.0
    nv = g.standard_normal((3, n, 3))
    nv /= np.linalg.norm(nv, axis=2, keepdims=True)
    nrm = np.zeros((3, n, 4), np.float64)
    nrm[:, :, :3] = nv
    col = np.zeros((3, n, 4), np.float64)
    col[:, :, :3] = g.uniform(0.0, 1.0, (3, n, 3))
    col[:, :, 3] = 1.0
    return RasterScene(W=W, H=H, pos=pos.astype(np.float32), nrm=nrm.astype(np.float32),
                       col=col.astype(np.float32), view_proj=camera.identity(),
                       light_mode=LIGHT_DIRECTIONAL, name=f"plain{n}_{W}x{H}_s{seed}")


def _cone(x, z, h, segs, yaw):
    """102-triangle cone: segs side triangles + segs base triangles."""
    r = 0.35 * h
    ang = yaw + np.arange(segs + 1) * (2.0 * np.pi / segs)
    bx, bz = x + r * np.cos(ang), z + r * np.sin(ang)
    apex = np.array([x, h, z])
    tris, nrms, uvs = [], [], []
    for k in range(segs):
        b0 = np.array([bx[k], 0.0, bz[k]])
        b1 = np.array([bx[k + 1], 0.0, bz[k + 1]])
        # outward side normals (smooth), counter-clockwise seen from outside
        n0 = np.array([np.cos(ang[k]) * h, r, np.sin(ang[k]) * h])
        n1 = np.array([np.cos(ang[k + 1]) * h, r, np.sin(ang[k + 1]) * h])
        am = 0.5 * (ang[k] + ang[k + 1])
        na = np.array([np.cos(am) * h, r, np.sin(am) * h])
        tris.append([b1, b0, apex]); nrms.append([n1, n0, na])
        uvs.append([[(k + 1) / segs, 0.0], [k / segs, 0.0], [(k + 0.5) / segs, 1.0]])
        c = np.array([x, 0.0, z])
        down = np.array([0.0, -1.0, 0.0])
        tris.append([c, b0, b1]); nrms.append([down, down, down])
        uvs.append([[0.5, 0.5], [0.5 + 0.5 * np.cos(ang[k]), 0.5 + 0.5 * np.sin(ang[k])],
                    [0.5 + 0.5 * np.cos(ang[k + 1]), 0.5 + 0.5 * np.sin(ang[k + 1])]])
    return tris, nrms, uvs


def _quad(x, z, h, yaw):
    w = 0.8 * h
    d = np.array([np.cos(yaw), 0.0, np.sin(yaw)]) * (0.5 * w)
    nrm = np.array([-np.sin(yaw), 0.0, np.cos(yaw)])
    p0 = np.array([x, 0.0, z]) - d
    p1 = np.array([x, 0.0, z]) + d
    p2 = p1 + np.array([0.0, h, 0.0])
    p3 = p0 + np.array([0.0, h, 0.0])
    tris = [[p0, p1, p2], [p0, p2, p3]]
    nrms = [[nrm, nrm, nrm]] * 2
    uvs = [[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]]
    return tris, nrms, uvs


FOREST_CONES = 1700
FOREST_QUADS = 300
FOREST_CONE_SEGS = 51      # 51 side + 51 base triangles = 102 per cone
FOREST_TRIS = FOREST_CONES * 2 * FOREST_CONE_SEGS + FOREST_QUADS * 2   # 174,000


def forest_scene(seed=1, W=1920, H=1080, fovy_deg=60.0):
    """Procedural forest of cones and quads (textured Lambert)."""
    g = _rng(seed)
    kinds = np.array([0] * FOREST_CONES + [1] * FOREST_QUADS)
    g.shuffle(kinds)
    xs = g.uniform(0.0, 100.0, kinds.size)
    zs = g.uniform(0.0, 100.0, kinds.size)
    hs = g.lognormal(0.0, 0.6, kinds.size)
    yaws = g.uniform(0.0, 2.0 * np.pi, kinds.size)
    T, N, U = [], [], []
    for kind, x, z, h, yaw in zip(kinds, xs, zs, hs, yaws):
        t, n, u = _cone(x, z, h, FOREST_CONE_SEGS, yaw) if kind == 0 else _quad(x, z, h, yaw)
        T += t; N += n; U += u
    T = np.asarray(T).transpose(1, 0, 2)  # [3, N, 3]
    Nv = np.asarray(N, np.float64).transpose(1, 0, 2)
    Nv /= np.linalg.norm(Nv, axis=2, keepdims=True)
    Uv = np.asarray(U, np.float64).transpose(1, 0, 2)
    n = T.shape[1]
    pos = np.ones((3, n, 4), np.float32); pos[:, :, :3] = T
    nrm = np.zeros((3, n, 4), np.float32); nrm[:, :, :3] = Nv
    eye = np.array([50.0, 8.0, -12.0])
    vp = camera.view_proj(eye, (50.0, 0.0, 40.0), (0.0, 1.0, 0.0), np.radians(fovy_deg), W, H, 0.5, 300.0)
    tex = g.integers(0, 256, (512, 512, 4), dtype=np.uint8)
    tex[:, :, 3] = 255
    # every vertex takes the reference's fixed material colour (col None)
    return RasterScene(W=W, H=H, pos=pos, nrm=nrm, col=None, view_proj=vp,
                       light_mode=LIGHT_EYE, eye=eye.astype(np.float32),
                       uv=Uv.astype(np.float32), texture=tex, name=f"forest{n}_{W}x{H}_s{seed}")


def batch_mix(count=64, seed_base=0):
    """The batched mix: scene i has seed i, log-uniform [1K, 200K] triangles and a
    resolution drawn from {256^2, 512^2, 1280x720, 1920x1080}."""
    g = _rng(10_000 + seed_base)
    res = [(256, 256), (512, 512), (1280, 720), (1920, 1080)]
    scenes = []
    for i in range(count):
        n = int(round(np.exp(g.uniform(np.log(1000.0), np.log(200000.0)))))
        W, H = res[int(g.integers(0, len(res)))]
        scenes.append(plain_scene(n=n, W=W, H=H, seed=seed_base + i))
    return scenes


def sphere_patches(seed=2, W=1280, H=720, amplitude=0.15, fovy_deg=60.0):
    """32 bicubic patches on a radially deformed unit sphere."""
    g = _rng(seed)
    omega = g.standard_normal((4, 3)) * 2.5
    phase = g.uniform(0.0, 2.0 * np.pi, 4)
    amp = g.uniform(0.5, 1.0, 4)
    amp /= amp.sum()

    def radius(d):
        return 1.0 + amplitude * np.sum(amp * np.sin(d @ omega.T + phase), axis=-1)

    lat_edges = np.radians([-80.0, -40.0, 0.0, 40.0, 80.0])
    lon_edges = np.linspace(0.0, 2.0 * np.pi, 9)
    patches = []
    for b in range(4):
        for a in range(8):
            th = lat_edges[b] + (lat_edges[b + 1] - lat_edges[b]) * np.arange(4) / 3.0
            ph = lon_edges[a] + (lon_edges[a + 1] - lon_edges[a]) * np.arange(4) / 3.0
            cps = np.zeros((16, 4))
            for r_ in range(4):          # v direction (latitude)
                for c_ in range(4):      # u direction (longitude)
                    d = np.array([np.cos(th[r_]) * np.cos(ph[c_]), np.sin(th[r_]),
                                  np.cos(th[r_]) * np.sin(ph[c_])])
                    cps[r_ * 4 + c_, :3] = radius(d) * d
                    cps[r_ * 4 + c_, 3] = 1.0
            patches.append(cps)
    vp = camera.view_proj((0.0, 0.3, 3.2), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), np.radians(fovy_deg), W, H, 0.5, 10.0)
    return PatchScene(W=W, H=H, patches=np.asarray(patches, np.float32), view_proj=vp,
                      name=f"sphere32_{W}x{H}_s{seed}")


def read_bez(path, scale=1.0, swapyz=False):
    """Bicubic patches of a RenderMan-style ``.dat`` file as the reference's
    bezmesh reader loads them (bezmesh/bezmesh.cpp:23-80,130-150): every
    ``Patch "bicubic"`` line is followed by four lines of four x y z points
    (w = 1), then all coordinates are scaled by scale / maxcoord, where maxcoord
    is updated with the signed coordinate whenever its magnitude exceeds the
    current value (the reader's own rule).  Returns float32 [P, 16, 4]."""
    patches = []
    with open(path) as f:
        lines = f.readlines()
    i = 0
    while i < len(lines):
        tok = lines[i].split()
        i += 1
        if len(tok) >= 2 and tok[0] == "Patch" and tok[1] == '"bicubic"':
            cp = np.zeros((4, 4, 4), np.float32)
            for r in range(4):
                vals = lines[i].split()
                i += 1
                for c in range(4):
                    x, y, z = (np.float32(float(v)) for v in vals[3 * c: 3 * c + 3])
                    if swapyz:
                        y, z = z, y
                    cp[r, c] = (x, y, z, 1.0)
            patches.append(cp)
    cps = np.asarray(patches, np.float32).reshape(-1, 16, 4)
    if scale != 0.0:
        maxcoord = np.float32(0.0)
        for p in cps:
            for v in p:
                for c in range(3):
                    if abs(v[c]) > maxcoord:
                        maxcoord = v[c]
        factor = np.float32(scale) / maxcoord
        cps[:, :, :3] = cps[:, :, :3] * factor
    return cps


def teapot_scene(cps, W=1024, H=768):
    """The reference's Reyes fixture (scenes/bezteapot.scene): the patches
    translated by (0, -0.5, 1) and rotated -90 degrees about x, seen from
    (0, 0, 3) with the camera's default 60-degree field of view."""
    a = np.radians(-90.0)
    rot = np.array([[1, 0, 0, 0], [0, np.cos(a), -np.sin(a), 0], [0, np.sin(a), np.cos(a), 0], [0, 0, 0, 1.0]])
    tr = np.eye(4)
    tr[:3, 3] = (0.0, -0.5, 1.0)
    m = tr @ rot
    p = cps.astype(np.float64).reshape(-1, 4)
    w = (p @ m.T).astype(np.float32).reshape(cps.shape)
    w[:, :, 3] = 1.0
    vp = camera.view_proj((0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), np.pi / 3.0, W, H, 0.02, 100.0)
    return PatchScene(W=W, H=H, patches=w, view_proj=vp, name=f"teapot{len(cps)}_{W}x{H}")
