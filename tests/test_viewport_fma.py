"""The Reyes split maps a projected control point to the screen as the
reference's C++ does, `(x + 1.0) * 0.5 * W` in double rounded to float
(split.pikostage:240-343 reads the double literal 1.0), with one float fma,
`fmaf(x, W/2, W/2)` (csrc/reyes_kernels.cu, split_measure).  The fma rounds the
exact value x*W/2 + W/2 once; the double sequence computes that exact value
whenever it lies near a float rounding boundary (the bits of x*W/2 + W/2 then
span fewer than 53), so both round it the same way.  This checks the identity
on random floats over a wide exponent range and on the floats next to every
rounding midpoint of random screen values, for the screen sizes in use and a
few odd ones, with exact rational arithmetic standing in for the fma."""
from fractions import Fraction

import numpy as np


def _round_f32(fr):
    """Correctly rounded (ties to even) float32 of a Fraction."""
    f = np.float32(float(fr))
    best = None
    for c in (np.nextafter(f, np.float32(-np.inf)), f, np.nextafter(f, np.float32(np.inf))):
        d = abs(Fraction(float(c)) - fr)
        if best is None or d < best[0] or (d == best[0] and (int(np.float32(c).view(np.uint32)) & 1) == 0):
            best = (d, c)
    return np.float32(best[1])


def _cases(rng, W, n_random, n_mid):
    e = rng.integers(-60, 12, n_random)
    m = rng.integers(1 << 23, 1 << 24, n_random)
    xs = (m.astype(np.float64) * np.exp2(e - 23.0) * rng.choice([-1.0, 1.0], n_random)).astype(np.float32)
    near = []
    half = Fraction(W, 2)
    for _ in range(n_mid):
        v = np.float32(rng.uniform(-2.0 * W, 2.0 * W))
        mid = Fraction(float(v)) + Fraction(float(np.spacing(v))) / 2
        x = np.float32(float(mid / half - 1))
        for step in (-2, -1, 0, 1, 2):
            xx = x
            for _ in range(abs(step)):
                xx = np.nextafter(xx, np.float32(np.inf) if step > 0 else np.float32(-np.inf))
            near.append(np.float32(xx))
    return np.concatenate([xs, np.array(near, np.float32)])


def test_fma_viewport_equals_double_sequence():
    rng = np.random.default_rng(7)
    for W in (256, 512, 720, 1080, 1280, 1920, 333, 16384):
        xs = _cases(rng, W, 3000, 300)
        ref = ((xs.astype(np.float64) + 1.0) * 0.5 * np.float64(W)).astype(np.float32)
        half = Fraction(W, 2)
        for x, r in zip(xs, ref):
            f = _round_f32(Fraction(float(x)) * half + half)
            assert f.view(np.uint32) == r.view(np.uint32), (W, float(x))
