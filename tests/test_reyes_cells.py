"""The two facts the device Reyes coverage pass rests on, checked on the CPU
with IEEE single-precision arithmetic (numpy float32 rounds every operation
and never contracts a multiply-add):

* the reversed-winding edge values equal the forward ones negated, so the
  kernel's rearranged test (`upoly_covers` in reyes_kernels.cu) equals the
  reference's eight-edge test (shade.pikostage:161-235) bit for bit;
* with every corner coordinate >= 32 and an extent < 16 px per axis, no sample
  strictly outside the corners' bounding box passes that test, which is why
  the dice kernel tests only the pixel cells (quadrants with 4 samples) that
  meet the open box there.
"""
import numpy as np

f32 = np.float32


def reference_covers(X, Y, px, py):
    """The reference's test: four edges of either winding strictly positive."""
    def edge(a, b):
        return (py - Y[a]) * (X[b] - X[a]) - (px - X[a]) * (Y[b] - Y[a])
    r1 = (edge(0, 1) > 0) & (edge(1, 2) > 0) & (edge(2, 3) > 0) & (edge(3, 0) > 0)
    r2 = (edge(0, 3) > 0) & (edge(3, 2) > 0) & (edge(2, 1) > 0) & (edge(1, 0) > 0)
    return r1 | r2


def rearranged_covers(X, Y, px, py):
    dX = [X[(i + 1) & 3] - X[i] for i in range(4)]
    dY = [Y[(i + 1) & 3] - Y[i] for i in range(4)]
    r1 = np.ones(px.shape, bool)
    r2 = np.ones(px.shape, bool)
    for i in range(4):
        ay, bx = py - Y[i], px - X[i]
        r1 &= ay * dX[i] - bx * dY[i] > 0
        r2 &= ay * dX[(i + 3) & 3] - bx * dY[(i + 3) & 3] < 0
    return r1 | r2


def quads(g, n):
    """Corners around random centres: ordinary micropolygons, slivers,
    degenerate (repeated / collinear) corners, and coordinates near the
    exact-region bounds."""
    mode = g.integers(0, 4, n)
    cx = np.where(mode == 0, g.uniform(-40, 2000, n), np.where(mode == 1, g.uniform(30, 40, n),
                                                               g.uniform(32, 4000, n)))
    cy = np.where(mode == 0, g.uniform(-40, 1200, n), np.where(mode == 1, g.uniform(30, 40, n),
                                                               g.uniform(32, 4000, n)))
    sz = np.where(mode == 1, g.uniform(0, 20, n), np.where(mode == 2, g.uniform(0, 1e-3, n),
                                                           g.uniform(0, 2, n)))
    X = [(cx + g.uniform(-1, 1, n) * sz).astype(f32) for _ in range(4)]
    Y = [(cy + g.uniform(-1, 1, n) * sz).astype(f32) for _ in range(4)]
    rep = g.random(n) < 0.1
    X[1] = np.where(rep, X[0], X[1])
    Y[1] = np.where(rep, Y[0], Y[1])
    col = g.random(n) < 0.1
    X[2] = np.where(col, X[0] + (X[1] - X[0]) * f32(2), X[2])
    Y[2] = np.where(col, Y[0] + (Y[1] - Y[0]) * f32(2), Y[2])
    return X, Y


def samples(g, X, Y):
    n = X[0].shape[0]
    mnx, mxx = np.minimum.reduce(X), np.maximum.reduce(X)
    mny, mxy = np.minimum.reduce(Y), np.maximum.reduce(Y)
    t = g.integers(0, 3, n)
    px = (mnx + (mxx - mnx + f32(2)) * g.random(n).astype(f32) - f32(1)).astype(f32)
    py = (mny + (mxy - mny + f32(2)) * g.random(n).astype(f32) - f32(1)).astype(f32)
    # samples on and just outside the box edges
    px = np.where(t == 1, np.where(g.random(n) < 0.5, mnx, mxx), px)
    px = np.where(t == 2, np.where(g.random(n) < 0.5, np.nextafter(mnx, f32(-1e9)), np.nextafter(mxx, f32(1e9))), px)
    return px.astype(f32), py.astype(f32), (mnx, mxx, mny, mxy)


def test_rearranged_test_equals_reference():
    g = np.random.Generator(np.random.Philox(101))
    total = 0
    for _ in range(8):
        X, Y = quads(g, 200_000)
        px, py, _ = samples(g, X, Y)
        a = reference_covers(X, Y, px, py)
        b = rearranged_covers(X, Y, px, py)
        assert np.array_equal(a, b)
        total += int(a.sum())
    assert total > 1000, "the sample mix never hit a micropolygon"


def test_no_sample_outside_the_box_passes_in_the_exact_region():
    g = np.random.Generator(np.random.Philox(202))
    checked = 0
    for _ in range(8):
        X, Y = quads(g, 200_000)
        px, py, (mnx, mxx, mny, mxy) = samples(g, X, Y)
        exact = ((mnx >= 32) & (mny >= 32) & (mxx - mnx < 16) & (mxy - mny < 16) &
                 (mxx < 4194304) & (mxy < 4194304))
        cov = reference_covers(X, Y, px, py)
        inside = (px > mnx) & (px < mxx) & (py > mny) & (py < mxy)
        assert not np.any(exact & cov & ~inside)
        checked += int(exact.sum())
    assert checked > 100_000


def test_cell_division_by_multiply_shift_is_exact():
    """cell_xy: dy = (li * (2^16 / cw + 1)) >> 16 equals li / cw for every cell
    index li < 64 of a rectangle cw <= 64 cells wide."""
    for cw in range(1, 65):
        m = 0x10000 // cw + 1
        for li in range(64):
            assert (li * m) >> 16 == li // cw, (cw, li)


def test_cell_ranges_equal_the_box_predicate():
    """The dice kernel's closed forms for the cells whose sample range meets the
    open box (mnx, mxx): quadrant q (4 samples, range [q/2, q/2 + 1/2]) is kept
    iff floor(2 mnx) <= q <= ceil(2 mxx) - 1; pixel x (centre x + 1/2) iff
    floor(mnx - 1/2) + 1 <= x <= ceil(mxx - 1/2) - 1.  Checked against the
    predicate itself on float32 bounds, including bounds on cell edges."""
    g = np.random.Generator(np.random.Philox(303))
    lo = g.uniform(32, 4000, 20000).astype(f32)
    lo = np.where(g.random(lo.size) < 0.3, np.round(lo * 2) / 2, lo).astype(f32)   # on half-pixel edges
    hi = (lo + g.uniform(0, 16, lo.size).astype(f32)).astype(f32)
    hi = np.where(g.random(lo.size) < 0.3, np.round(hi * 2) / 2, hi).astype(f32)
    hi = np.maximum(hi, lo)
    for mnx, mxx in zip(lo.tolist(), hi.tolist()):
        mnx, mxx = f32(mnx), f32(mxx)
        # quadrants
        q0 = int(np.floor(f32(2) * mnx))
        q1 = int(np.ceil(f32(2) * mxx)) - 1
        for q in range(int(mnx * 2) - 2, int(mxx * 2) + 3):
            keep = (q * 0.5 < float(mxx)) and (q * 0.5 + 0.5 > float(mnx))
            assert keep == (q0 <= q <= q1), (mnx, mxx, q)
        # pixel centres
        x0 = int(np.floor(mnx - f32(0.5))) + 1
        x1 = int(np.ceil(mxx - f32(0.5))) - 1
        for x in range(int(mnx) - 2, int(mxx) + 3):
            keep = (x + 0.5 > float(mnx)) and (x + 0.5 < float(mxx))
            assert keep == (x0 <= x <= x1), (mnx, mxx, x)
