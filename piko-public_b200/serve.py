"""Request streams for the served form (piko_server_*).

A render request names a resident scene and a camera.  The raster scenes of the
served workload are the 64-scene batched mix (clip-space geometry); each request
re-seeds its camera as a small random similarity transform of clip space.  The
Reyes requests orbit the camera around the deformed sphere.
"""
import time

import numpy as np

from . import camera
from .runtime import const_state


def raster_camera(g, base=None):
    """Column-major view-projection: rotation about the view axis, uniform
    scale and a shift, all in clip space (w stays 1)."""
    th = g.uniform(-0.3, 0.3)
    s = g.uniform(0.85, 1.15)
    tx, ty = g.uniform(-0.1, 0.1, 2)
    m = np.eye(4)
    m[0, 0], m[0, 1] = s * np.cos(th), -s * np.sin(th)
    m[1, 0], m[1, 1] = s * np.sin(th), s * np.cos(th)
    m[0, 3], m[1, 3] = tx, ty
    return np.ascontiguousarray(m.T.reshape(16), np.float32)


def reyes_camera(g, W, H):
    phi = g.uniform(-0.6, 0.6)
    eye = (3.2 * np.sin(phi), g.uniform(0.0, 0.5), 3.2 * np.cos(phi))
    return camera.view_proj(eye, (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), np.radians(60.0), W, H, 0.5, 10.0)


def make_stream(seed, n_raster_scenes, rate_hz, seconds, reyes_fraction=0.2):
    """Poisson arrivals: list of (t_seconds, kind, scene index, seed)."""
    g = np.random.Generator(np.random.Philox(seed))
    t = 0.0
    out = []
    while True:
        t += g.exponential(1.0 / rate_hz)
        if t >= seconds:
            break
        if g.uniform() < reyes_fraction:
            out.append((t, "reyes", 0, int(g.integers(1 << 31))))
        else:
            out.append((t, "raster", int(g.integers(n_raster_scenes)), int(g.integers(1 << 31))))
    return out


def request_state(kind, scene, rseed):
    g = np.random.Generator(np.random.Philox(rseed))
    if kind == "raster":
        return const_state(view_proj=raster_camera(g), light_mode=0, light=(0.5773, 0.5773, 0.5773))
    return const_state(view_proj=reyes_camera(g, scene.W, scene.H))


def replay(server, stream, raster_scenes, reyes_scenes, keep=False):
    """Submits the stream in real time (busy-waiting for each arrival) and
    returns the request ids in submission order."""
    states = [request_state(k, (raster_scenes[i] if k == "raster" else reyes_scenes[i]), s)
              for (_, k, i, s) in stream]
    ids = []
    t0 = time.perf_counter()
    for (t, k, i, _), st in zip(stream, states):
        while time.perf_counter() - t0 < t:
            pass
        scene = raster_scenes[i] if k == "raster" else reyes_scenes[i]
        ids.append(server.submit(scene, st, keep=keep))
    return ids, states
