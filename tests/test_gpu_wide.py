"""Factor counts outside 1..256, through the C ABI, against the oracle: the
bias-only jobs (n_feat = 0, src/bin/tsvdx4-new.rs:206,523) and the wide
jobs (400 ... 4800, :19-22; tsvdx4p up to 16000), whose rows the kernels take
in 256-column slices. And every base job of the reference's dispatcher
(:18-40) constructs and trains through tsvd_create with default options.

Tolerances as in test_gpu_parity: the seeded init bitwise, one epoch within
2e-5 of the oracle per parameter, predictions from identical parameters
within 1e-5.
"""
import numpy as np
import pytest

from netflix_prize_b200.abi import SCHED_SEQUENTIAL, SCHED_STRATIFIED
from netflix_prize_b200.config import run_lm
from netflix_prize_b200.data import MaskedDataset
from netflix_prize_b200.model import TxModel
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

PARAMS = ["ubias", "ibias", "ufeat", "ufeat2", "ifeat", "yfeat", "alpha_u", "but_bin", "bit_bin", "ybias",
          "ubias_day", "ibias_freq", "ifeat_freq", "cu", "cut"]


def _sets():
    from tests.conftest import small_sets
    return small_sets(n_users=400, n_items=150, n_train=16000, seed=17)


def _close(g, o, names, tol):
    for n in names:
        a = np.asarray(g.get_param(n), np.float64).ravel()
        b = np.asarray(o.get_param(n), np.float64).ravel()
        assert a.shape == b.shape, n
        if a.size:
            assert np.max(np.abs(a - b)) < tol, (n, float(np.max(np.abs(a - b))))


@pytest.mark.parametrize("f", [0, 400, 1600])
def test_initial_state_bitwise(f):
    tr, pr = _sets()
    cfg = run_lm(f, 1, n_time_bins=30)
    g = TxModel(tr, MaskedDataset(pr), cfg)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    for n in ["ufeat", "ifeat", "yfeat", "ifeat_freq", "tu_mean", "cu", "gbias"]:
        a = np.asarray(g.get_param(n), np.float32).ravel()
        b = np.asarray(o.get_param(n), np.float32).ravel()
        assert a.shape == b.shape, n
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), n


@pytest.mark.parametrize("f", [0, 300, 400, 1600])
def test_stratified_epochs_match_oracle_tsvdx4p(f):
    tr, pr = _sets()
    cfg = run_lm(f, 2, n_time_bins=30)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED)
    for e in (1, 2):
        o.fit_epoch(e, po.SCHED_P, nsvd_norm_exp=1.0, n_threads=1)
        g.fit_epoch(tr, pr, e)
    _close(g, o, PARAMS + ["ycache", "ycache_bias"], 2e-5)
    assert abs(g.calc_rmse(pr) - o.calc_rmse(pr)) < 1e-5


@pytest.mark.parametrize("f", [0, 400, 1000])
def test_sequential_epoch_matches_oracle(f):
    """The sequential schedule (and so the seq_epochs of the tsvdx4p jobs,
    src/bin/tsvdx4p-new.rs:14-19) with wide rows."""
    tr, pr = _sets()
    cfg = run_lm(f, 1, n_time_bins=30)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_SEQUENTIAL)
    o.fit_epoch(1, po.SCHED_SEQ)
    g.fit_epoch(tr, pr, 1)
    _close(g, o, PARAMS + ["ycache", "ycache_bias"], 2e-5)


@pytest.mark.parametrize("f", [0, 400, 1600])
def test_predict_parity_given_trained_oracle_params(f):
    tr, pr = _sets()
    cfg = run_lm(f, 1, n_time_bins=30)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    o.fit_epoch(1, po.SCHED_P, nsvd_norm_exp=1.0, n_threads=1)
    g = TxModel(tr, MaskedDataset(pr), cfg)
    for n in PARAMS:
        g.set_param(n, np.asarray(o.get_param(n), np.float32).ravel())
    g.rebuild_ycache()
    want = o.predict_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    got = g.predict_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    assert np.max(np.abs(got - want)) < 1e-5
    ws = o.predict_subscores_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    gs = g.predict_subscores_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    assert np.max(np.abs(gs - ws)) < 1e-5
    assert abs(g.calc_rmse(pr) - o.calc_rmse(pr)) < 1e-6


def test_every_tsvdx4_base_job_constructs_and_trains():
    """Each job's TxConfig, as the reference's dispatcher builds it, through
    tsvd_create with default options (the stratified schedule), one epoch."""
    from netflix_prize_b200.jobs import JOBS
    tr, pr = _sets()
    assert len(JOBS) == 19
    for name, job in JOBS.items():
        g = TxModel(tr, MaskedDataset(pr), job.config)
        g.fit_epoch(tr, pr, 1)
        r = g.calc_rmse(pr)
        assert np.isfinite(r) and r < 2.0, (name, r)
        g.close()


def test_hogwild_rejects_wide_rows():
    from netflix_prize_b200.abi import SCHED_HOGWILD
    from netflix_prize_b200.native import TsvdError
    tr, pr = _sets()
    with pytest.raises(TsvdError, match="above 256"):
        TxModel(tr, MaskedDataset(pr), run_lm(400, 1), schedule=SCHED_HOGWILD)
