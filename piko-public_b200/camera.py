"""Host-side camera matrices (no GL).

The reference builds its view-projection matrix with gluPerspective/gluLookAt and
reads it back with glGetFloatv (pikoc/samples/rasterPipelineFixPt/main.cpp:268-297);
there is no GL here, so the matrix is computed on the CPU the way
``camera::updateCam`` does it (pikoc/samples/rasterPipelineFixPt/basicTypes/camera.h:73-120):
a GL perspective matrix times a look-at matrix, stored column-major so that
``clip.x = m[0]*x + m[4]*y + m[8]*z + m[12]`` (piko/math.h:365-373).

The 16 floats are an input shared by the device pipeline and the oracle, so
their own rounding does not enter the parity comparison.
"""
import numpy as np


def perspective(fovy_rad, aspect, znear, zfar):
    """GL perspective matrix (row-major 4x4, float64)."""
    f = 1.0 / np.tan(fovy_rad / 2.0)
    d = 1.0 / (znear - zfar)
    m = np.zeros((4, 4))
    m[0, 0] = f / aspect
    m[1, 1] = f
    m[2, 2] = (znear + zfar) * d
    m[2, 3] = 2.0 * znear * zfar * d
    m[3, 2] = -1.0
    return m


def look_at(eye, target, up):
    """GL look-at matrix (row-major 4x4, float64)."""
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    up = np.asarray(up, np.float64)
    up = up / np.linalg.norm(up)
    s = np.cross(f, up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    m = np.eye(4)
    m[0, :3] = s
    m[1, :3] = u
    m[2, :3] = -f
    m[:3, 3] = -m[:3, :3] @ eye
    return m


def view_proj(eye, target, up, fovy_rad, W, H, znear, zfar):
    """Column-major float32[16] view-projection matrix for a W x H target."""
    m = perspective(fovy_rad, W / float(H), znear, zfar) @ look_at(eye, target, up)
    return np.ascontiguousarray(m.T.reshape(16), dtype=np.float32)


def identity():
    return np.eye(4, dtype=np.float32).reshape(16).copy()
