"""The library's seeded streams (product code, no GPU needed) against the
oracle's restatement of rand 0.9 (itself pinned by the reference's RMSE
known answers)."""
import ctypes as C

import numpy as np
import pytest

from netflix_prize_b200 import native
from oracle import pyoracle as po


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.mark.parametrize("n,seed,epoch", [(1, 42, 1), (2, 42, 1), (20, 42, 3), (1000, 7, 13), (480189, 42, 2)])
def test_user_order_matches_oracle(n, seed, epoch):
    L = native.load()
    out = np.zeros(n, np.uint32)
    assert L.tsvd_user_order_for_seed(n, 1, seed, epoch, _p(out)) == 0
    assert np.array_equal(out, po.get_users(n, True, seed, epoch))


def test_user_order_unshuffled_is_identity():
    L = native.load()
    out = np.zeros(50, np.uint32)
    assert L.tsvd_user_order_for_seed(50, 0, 1, 1, _p(out)) == 0
    assert np.array_equal(out, np.arange(50))


@pytest.mark.parametrize("seed,sigma", [(42, 0.001), (64, 0.005), (1, 1.0), (2400, 0.0)])
def test_normal_stream_matches_oracle(seed, sigma):
    L = native.load()
    n = 200000
    out = np.zeros(n, np.float32)
    assert L.tsvd_normal_stream(seed, sigma, n, _p(out)) == 0
    ref = po.normal_stream(seed, sigma, n)
    assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))


def test_normal_stream_moments():
    ref = po.normal_stream(123, 1.0, 400000).astype(np.float64)
    assert abs(ref.mean()) < 0.01 and abs(ref.std() - 1.0) < 0.01
    # tails beyond the ziggurat's base layer (R = 3.654) are produced
    assert (np.abs(ref) > 3.7).sum() > 0
