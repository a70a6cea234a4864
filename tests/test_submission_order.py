"""The closed-form submission rank used by the setup kernel equals the order in
which the reference's one-thread CPU backend fills the raster bins."""
import numpy as np
import pytest


def submission_rank(ids, N, nVS):
    # same integer formula as submission_rank() in csrc/raster_kernels.cu
    ids = np.asarray(ids, np.int64)
    C = (N + 511) // 512
    c = ids // 512
    b = c % nVS
    q, rem = C // nVS, C % nVS
    lastbin = (C - 1) % nVS
    deficit = C * 512 - N
    start = 512 * (b * q + np.minimum(b, rem)) - np.where(lastbin < b, deficit, 0)
    return start + (c // nVS) * 512 + ids % 512


@pytest.mark.parametrize("N,W,H", [(1, 32, 32), (512, 32, 32), (513, 32, 32), (4096, 512, 512),
                                   (40000, 256, 256), (200000, 256, 256), (174000, 1920, 1080),
                                   (99999, 64, 96), (65537, 128, 32), (1000, 33, 65)])
def test_rank_matches_oracle_order(oracle_mod, N, W, H):
    nVS = (W // 32) * (H // 32)
    order = oracle_mod.submission_order(N, W, H)
    assert sorted(order.tolist()) == list(range(N))
    rank = submission_rank(np.arange(N), N, nVS)
    inv = np.empty(N, np.int64)
    inv[order] = np.arange(N)
    assert np.array_equal(rank, inv)
