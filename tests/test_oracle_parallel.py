"""The oracle's threaded stratified epoch (test infrastructure for the
full-shape FP64 runs) against its one-thread form: every table bitwise equal
after each epoch, in FP32 and FP64, since both sum in the same order."""
import numpy as np
import pytest

from netflix_prize_b200.config import run_lm
from netflix_prize_b200.data import MaskedDataset
from oracle import pyoracle as po

TABLES = ["ubias", "ibias", "ufeat", "ufeat2", "ifeat", "yfeat", "alpha_u", "but_bin", "bit_bin", "ybias",
          "ubias_day", "ibias_freq", "ifeat_freq", "cu", "cut", "ycache", "ycache_bias"]


@pytest.mark.parametrize("fp64", [False, True])
def test_threaded_epoch_is_bitwise_the_one_thread_epoch(fp64):
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=600, n_items=200, n_train=30000, seed=11)
    cfg = run_lm(24, 3, n_time_bins=30)
    a = po.OracleModel(tr, MaskedDataset(pr), cfg, fp64=fp64)
    b = po.OracleModel(tr, MaskedDataset(pr), cfg, fp64=fp64)
    for e in (1, 2, 3):
        a.fit_epoch(e, po.SCHED_P, nsvd_norm_exp=1.0, n_threads=1)
        b.fit_epoch_parallel(e, nsvd_norm_exp=1.0, workers=3)
        for n in TABLES:
            x, y = np.asarray(a.get_param(n)), np.asarray(b.get_param(n))
            assert x.shape == y.shape and np.array_equal(x, y), (e, n)
    assert a.calc_rmse(pr) == b.calc_rmse(pr)


def test_threaded_epoch_needs_low_memory():
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=300, n_items=100, n_train=12000, seed=2)
    cfg = run_lm(8, 1, n_time_bins=30, low_memory=False)
    m = po.OracleModel(tr, MaskedDataset(pr), cfg)
    with pytest.raises(RuntimeError, match="low_memory"):
        m.fit_epoch_parallel(1)
