"""Failure detection on the device without a fault: the Reyes split kernel's
level barrier is a bounded wait.  A self-test CTA waits for a release that
nothing sends; the wait gives up after about a second, the kernel records the
timeout and returns, the call reports PIKO_ERR_TIMEOUT, and the same context
then renders a frame that matches the oracle."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_survives(pk, ctx, oracle_mod):
    rt = pk.runtime
    lib = rt.load_library()
    t0 = time.perf_counter()
    st = lib.piko_selftest_wait_timeout(ctx.h)
    dt = time.perf_counter() - t0
    assert st == rt.ERR_TIMEOUT, rt.STATUS_NAMES.get(st, st)
    assert 0.5 < dt < 30.0, f"the wait gave up after {dt:.2f} s"
    sc = pk.scenes.sphere_patches(W=160, H=120, seed=4)
    pipe = pk.Pipe(ctx, "reyes")
    s = pk.Scene(pipe, sc)
    try:
        s.run()
        fb, depth = s.read()
    finally:
        s.close()
        pipe.close()
    ofb, odepth, _ = oracle_mod.reyes_frame(sc)
    assert np.array_equal(fb, ofb)
    assert np.array_equal(depth.view(np.uint32), odepth.view(np.uint32))
