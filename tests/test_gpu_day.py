"""Per-day terms (low_memory = false) and the sequential schedule on the GPU,
against the CPU oracle, through the C ABI.

Tolerances:
  * sequential schedule vs the oracle's sequential TxModel: parameters within
    2e-5 absolute, held-out RMSE within 1e-5 (FP32 warp-tree dot products and
    FMA contraction against the oracle's sequential sums);
  * the reference's own known answer (tests/regressors_test.rs:75-93,
    low_memory = false, full_su, ufeat_day trained): RMSE within 1e-5;
  * ycache_day rebuild: bitwise (same adds in the same order, IEEE sqrt and
    division);
  * predictions from identical parameters: 1e-5 absolute;
  * Hogwild with per-day terms, disjoint item blocks (race-free): parameters
    within 2e-5 of the sequential oracle; on shared items, held-out RMSE
    within 0.001 of it.
"""
import numpy as np
import pytest

from netflix_prize_b200.abi import SCHED_HOGWILD, SCHED_SEQUENTIAL
from netflix_prize_b200.config import OrdinalHeadConfig, regression_test_config, run_lm
from netflix_prize_b200.data import MaskedDataset
from netflix_prize_b200.model import TxModel
from oracle import pyoracle as po
from tests.test_gpu_parity import PARAMS, disjoint_sets

pytestmark = pytest.mark.gpu

DAY_PARAMS = PARAMS + ["yfeat_day", "ufeat_day", "ycache_day", "ycache", "ycache_bias"]


def day_cfg(f=16, epochs=2, **kw):
    return run_lm(f, epochs, n_time_bins=30).replace(low_memory=False, lr_ud=0.001, reg_ud=0.04, lr_yd=0.0002,
                                                      reg_yd=0.02, sigma_yd=0.009, **kw)


def assert_params_close(g, o, names, tol=2e-5, rtol=1e-6):
    for n in names:
        a = np.asarray(g.get_param(n), np.float64).ravel()
        b = np.asarray(o.get_param(n), np.float64).ravel()
        assert a.shape == b.shape, n
        err = np.max(np.abs(a - b) - rtol * np.abs(b)) if a.size else 0.0
        assert err < tol, (n, err)


def test_initial_state_with_yfeat_day_bitwise(small):
    """yfeat_day is drawn between yfeat and ifeat_freq (src/tx.rs:610-612)."""
    tr, pr = small
    cfg = day_cfg(f=40)
    g = TxModel(tr, MaskedDataset(pr), cfg)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    for n in ["ufeat", "ifeat", "yfeat", "yfeat_day", "ifeat_freq", "ufeat_day", "ycache_day"]:
        a = np.asarray(g.get_param(n), np.float32).ravel()
        b = np.asarray(o.get_param(n), np.float32).ravel()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), n


def test_sequential_reproduces_reference_known_answer(tiny, golden):
    """tsvdx4_probe_rmse_regression (tests/regressors_test.rs:75-93) on the GPU:
    3 epochs, n_feat 10, low_memory = false, full_su, ufeat_day trained."""
    tr, pr = tiny
    cfg = regression_test_config()
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_SEQUENTIAL)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    for e in range(1, cfg.n_epochs + 1):
        g.fit_epoch(tr, pr, e)
        o.fit_epoch(e, po.SCHED_SEQ)
    assert abs(g.calc_rmse(pr) - golden["tsvdx4_probe_rmse"]) < 1e-5
    assert_params_close(g, o, DAY_PARAMS)


@pytest.mark.parametrize("low_memory", [True, False])
def test_sequential_matches_oracle(small, low_memory):
    tr, pr = small
    cfg = day_cfg(f=32, epochs=2) if not low_memory else run_lm(32, 2, n_time_bins=30)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_SEQUENTIAL)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    for e in (1, 2):
        g.fit_epoch(tr, pr, e)
        o.fit_epoch(e, po.SCHED_SEQ)
    names = DAY_PARAMS if not low_memory else PARAMS + ["ycache", "ycache_bias"]
    assert_params_close(g, o, names, tol=5e-5)
    assert abs(g.calc_rmse(pr) - o.calc_rmse(pr)) < 1e-5


def test_sequential_trains_ordinal_thresholds(small):
    """lr_t != 0 moves the four thresholds after every rating
    (src/tx.rs:963-972); only the sequential schedule takes it."""
    tr, pr = small
    cfg = run_lm(16, 2, n_time_bins=30).replace(
        ordinal_head=OrdinalHeadConfig((1.5, 2.5, 3.5, 4.5), 0.05, 0.002, 0.001))
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_SEQUENTIAL)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    for e in (1, 2):
        g.fit_epoch(tr, pr, e)
        o.fit_epoch(e, po.SCHED_SEQ)
    th_g, th_o = np.asarray(g.get_param("thresholds")), np.asarray(o.get_param("thresholds"))
    assert np.max(np.abs(th_g - th_o)) < 1e-4, (th_g, th_o)
    assert not np.allclose(th_o, [1.5, 2.5, 3.5, 4.5])
    assert_params_close(g, o, PARAMS, tol=1e-4, rtol=1e-5)
    with pytest.raises(Exception):
        TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_HOGWILD)


@pytest.mark.parametrize("f", [8, 40, 256])
def test_rebuild_ycache_day_bitwise(small, f):
    tr, pr = small
    cfg = day_cfg(f=f)
    g = TxModel(tr, MaskedDataset(pr), cfg)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    rng = np.random.default_rng(f)
    yd = rng.normal(0, 0.1, (tr.n_items, f)).astype(np.float32)
    g.set_param("yfeat_day", yd.ravel())
    o.set_param("yfeat_day", yd.ravel())
    g.rebuild_ycache()
    o.rebuild_ycache()
    a = np.asarray(g.get_param("ycache_day"), np.float32).ravel()
    b = np.asarray(o.get_param("ycache_day"), np.float32).ravel()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("f", [10, 64, 256])
def test_predict_parity_per_day(small, f):
    tr, pr = small
    cfg = day_cfg(f=f, epochs=2)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    for e in (1, 2):
        o.fit_epoch(e)
    g = TxModel(tr, MaskedDataset(pr), cfg)
    for n in PARAMS + ["yfeat_day", "ufeat_day"]:
        g.set_param(n, np.asarray(o.get_param(n), np.float32).ravel())
    g.rebuild_ycache()
    for u, i, d in ((pr.user_idxs, pr.item_idxs, pr.dates), (tr.user_idxs, tr.item_idxs, tr.dates),
                    (pr.user_idxs, pr.item_idxs, (pr.dates + 7).astype(np.int16))):
        assert np.max(np.abs(g.predict_batch(u, i, d) - o.predict_batch(u, i, d))) < 1e-5
        assert np.max(np.abs(g.predict_subscores_batch(u, i, d) - o.predict_subscores_batch(u, i, d))) < 1e-5
    assert abs(g.calc_rmse(pr) - o.calc_rmse(pr)) < 1e-6


@pytest.mark.parametrize("f", [16, 64])
def test_hogwild_day_equals_sequential_without_races(f):
    tr, pr = disjoint_sets()
    cfg = day_cfg(f=f, epochs=2)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_HOGWILD)
    for e in (1, 2):
        o.fit_epoch(e, po.SCHED_SEQ)
        g.fit_epoch(tr, pr, e)
    assert_params_close(g, o, DAY_PARAMS)
    assert abs(g.calc_rmse(pr) - o.calc_rmse(pr)) < 1e-5


def test_hogwild_day_heldout_rmse_within_0p001_of_sequential_reference():
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=3000, n_items=800, n_train=200000, seed=11)
    cfg = day_cfg(f=32, epochs=8)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_HOGWILD)
    for e in range(1, 9):
        o.fit_epoch(e, po.SCHED_SEQ)
        g.fit_epoch(tr, pr, e)
    ro, rg = o.calc_rmse(pr), g.calc_rmse(pr)
    print(f"held-out RMSE: oracle {ro:.6f}, GPU Hogwild per-day {rg:.6f}")
    assert abs(rg - ro) <= 0.001
