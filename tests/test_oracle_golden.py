"""The CPU oracle against the reference's own known answers.

tests/regressors_test.rs:75-93 and :157-175 pin bit-exact f32 arithmetic and
the rand 0.9 streams (init and per-epoch shuffle) end to end;
tests/lib_test.rs pins the fixture invariants, offsets and gbias.
"""
import numpy as np
import pytest

from netflix_prize_b200.config import regression_test_config
from netflix_prize_b200.data import MaskedDataset, calc_gbias, calc_user_offsets
from oracle import pyoracle as po


def test_tsvdx4_probe_rmse_regression(tiny, golden):
    tr, pr = tiny
    m = po.OracleModel(tr, MaskedDataset(pr), regression_test_config())
    for e in range(1, m.n_epochs() + 1):
        m.fit_epoch(e, po.SCHED_SEQ)
    assert m.calc_rmse(pr) == golden["tsvdx4_probe_rmse"]


def test_tsvdx4p_probe_rmse_regression(tiny, golden):
    tr, pr = tiny
    m = po.OracleModel(tr, MaskedDataset(pr), regression_test_config())
    for e in range(1, m.n_epochs() + 1):
        m.fit_epoch(e, po.SCHED_P, nsvd_norm_exp=0.5, n_threads=1)
    assert m.calc_rmse(pr) == golden["tsvdx4p_probe_rmse"]


def test_chacha20_rfc7539_block():
    # RFC 7539 section 2.3.2 test vector (20 rounds) for the ChaCha core.
    key = [int.from_bytes(bytes(range(4 * k, 4 * k + 4)), "little") for k in range(8)]
    st = [0x61707865, 0x3320646e, 0x79622d32, 0x6b206574] + key + [1, 0x09000000, 0x4a000000, 0]
    out = po.chacha_block(st, 20)
    assert [int(x) for x in out[:4]] == [0xe4e7f110, 0x15593bd1, 0x1fdd0f50, 0xc47120a3]
    assert [int(x) for x in out[12:]] == [0xd19c12b5, 0xb94e16de, 0xe883d0cb, 0x4e3c50a2]


def test_tiny_train_sorted_by_user_date(tiny):
    tr, _ = tiny
    key = tr.user_idxs.astype(np.int64) * 100000 + tr.dates
    assert np.all(np.diff(key) >= 0)


def test_tiny_probe_sorted_by_item(tiny):
    _, pr = tiny
    assert np.all(np.diff(pr.item_idxs) >= 0)


def test_user_item_pairs_unique_across_train_and_probe(tiny):
    tr, pr = tiny
    k = np.concatenate([tr.user_idxs * 100 + tr.item_idxs, pr.user_idxs * 100 + pr.item_idxs])
    assert len(np.unique(k)) == len(k)


def test_user_offsets_raises_on_unsorted(tiny):
    _, pr = tiny
    with pytest.raises(ValueError, match="not user-sorted"):
        calc_user_offsets(pr)


def test_user_offsets_span_equals_user_cnts(tiny):
    tr, _ = tiny
    off = calc_user_offsets(tr)
    assert np.array_equal(np.diff(off), tr.user_cnts)


def test_gbias_equals_residuals_mean(tiny):
    tr, _ = tiny
    assert calc_gbias(tr) == np.float32(tr.residuals.astype(np.float64).sum() / tr.n_ratings)


def test_oracle_gbias_param_matches(tiny):
    tr, pr = tiny
    m = po.OracleModel(tr, MaskedDataset(pr), regression_test_config())
    assert np.float32(m.get_param("gbias")[0]) == calc_gbias(tr)


def test_oracle_fp64_twin_tracks_f32(tiny):
    tr, pr = tiny
    cfg = regression_test_config()
    a = po.OracleModel(tr, MaskedDataset(pr), cfg)
    b = po.OracleModel(tr, MaskedDataset(pr), cfg, fp64=True)
    for e in range(1, 4):
        a.fit_epoch(e)
        b.fit_epoch(e)
    assert abs(a.calc_rmse(pr) - b.calc_rmse(pr)) < 1e-5


def test_oracle_low_memory_quirk_trains_bin0_only(small):
    """low_memory: training always uses frequency bin 0 (src/tx.rs:834,873)."""
    from netflix_prize_b200.config import run_lm
    tr, pr = small
    cfg = run_lm(8, 1, n_time_bins=30, low_memory=True)
    m = po.OracleModel(tr, MaskedDataset(pr), cfg)
    before = m.get_param("ifeat_freq").reshape(tr.n_items, 16, 8).copy()
    ibf_before = m.get_param("ibias_freq").reshape(tr.n_items, 16).copy()
    m.fit_epoch(1)
    after = m.get_param("ifeat_freq").reshape(tr.n_items, 16, 8)
    ibf_after = m.get_param("ibias_freq").reshape(tr.n_items, 16)
    assert np.array_equal(before[:, 1:], after[:, 1:])
    assert np.array_equal(ibf_before[:, 1:], ibf_after[:, 1:])
    assert not np.array_equal(before[:, 0], after[:, 0])
