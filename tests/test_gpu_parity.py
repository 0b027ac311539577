"""GPU parity against the CPU oracle, through the C ABI.

Tolerances (floating point, FP32 kernels):
  * initial state and ycache rebuilds: bitwise (same adds in the same order,
    IEEE division and square root);
  * predictions/subscores from identical parameters: 1e-5 absolute (the
    warp-tree dot product and CUDA powf differ from the sequential f32 sum
    and glibc powf in the last bits);
  * one stratified epoch from identical state: parameters within 2e-5
    absolute of the oracle's tsvdx4p epoch (FMA contraction and reduction
    order);
  * training: held-out RMSE within +-0.001 of the oracle's sequential
    TxModel at the same hyperparameters and epoch count.
"""
import numpy as np
import pytest

from netflix_prize_b200.abi import SCHED_HOGWILD, SCHED_STRATIFIED
from netflix_prize_b200.config import run_lm, regression_test_config
from netflix_prize_b200.data import MaskedDataset
from netflix_prize_b200.model import TxModel
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

PARAMS = ["ubias", "ibias", "ufeat", "ufeat2", "ifeat", "yfeat", "alpha_u", "but_bin", "bit_bin", "ybias",
          "ubias_day", "ibias_freq", "ifeat_freq", "cu", "cut"]


def lm_cfg(f=16, epochs=3, **kw):
    return run_lm(f, epochs, n_time_bins=30).replace(**kw)


def copy_params(src, dst):
    for n in PARAMS:
        dst.set_param(n, np.asarray(src.get_param(n), np.float32).ravel())


def test_initial_state_bitwise(small):
    tr, pr = small
    cfg = lm_cfg(f=40)
    g = TxModel(tr, MaskedDataset(pr), cfg)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    for n in ["ufeat", "ifeat", "yfeat", "ifeat_freq", "tu_mean", "cu", "gbias"]:
        a = np.asarray(g.get_param(n), np.float32).ravel()
        b = np.asarray(o.get_param(n), np.float32).ravel()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), n


def test_user_order_matches_reference_shuffle(small):
    tr, pr = small
    g = TxModel(tr, MaskedDataset(pr), lm_cfg())
    for e in (1, 2, 13):
        assert np.array_equal(g.get_user_order(e), po.get_users(tr.n_users, True, 42, e))


@pytest.mark.parametrize("f", [8, 32, 60, 64, 128, 256])
def test_rebuild_ycache_bitwise(small, f):
    tr, pr = small
    cfg = lm_cfg(f=f)
    g = TxModel(tr, MaskedDataset(pr), cfg)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    rng = np.random.default_rng(f)
    yb = rng.normal(0, 0.1, tr.n_items).astype(np.float32)
    g.set_param("ybias", yb)
    o.set_param("ybias", yb)
    g.rebuild_ycache()
    o.rebuild_ycache()
    for n in ("ycache", "ycache_bias"):
        a = np.asarray(g.get_param(n), np.float32).ravel()
        b = np.asarray(o.get_param(n), np.float32).ravel()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), n


@pytest.mark.parametrize("f", [10, 32, 64, 256])
def test_predict_parity_given_trained_oracle_params(small, f):
    tr, pr = small
    cfg = lm_cfg(f=f, epochs=2)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    for e in (1, 2):
        o.fit_epoch(e)
    g = TxModel(tr, MaskedDataset(pr), cfg)
    copy_params(o, g)
    g.rebuild_ycache()
    want = o.predict_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    got = g.predict_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    assert np.max(np.abs(got - want)) < 1e-5
    ws = o.predict_subscores_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    gs = g.predict_subscores_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    assert np.max(np.abs(gs - ws)) < 1e-5
    assert abs(g.calc_rmse(pr) - o.calc_rmse(pr)) < 1e-6
    # training rows (save_train path) and days absent from SparseUD
    want = o.predict_batch(tr.user_idxs, tr.item_idxs, tr.dates)
    got = g.predict_batch(tr.user_idxs, tr.item_idxs, tr.dates)
    assert np.max(np.abs(got - want)) < 1e-5
    odd = (pr.dates + 7).astype(np.int16)
    assert np.max(np.abs(g.predict_batch(pr.user_idxs, pr.item_idxs, odd)
                         - o.predict_batch(pr.user_idxs, pr.item_idxs, odd))) < 1e-5


def test_gen_preds_offsets(tiny):
    tr, pr = tiny
    cfg = regression_test_config(low_memory=True)
    g = TxModel(tr, MaskedDataset(pr), cfg)
    pr2 = pr
    pr2.residuals = pr.raw_ratings.astype(np.float32) - np.float32(0.25)
    preds = g.gen_preds(pr2)
    base = g.predict_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    assert np.allclose(preds, base + 0.25, atol=1e-6)


@pytest.mark.parametrize("f", [16, 64, 256])
def test_stratified_epoch_matches_oracle_tsvdx4p(small, f):
    tr, pr = small
    cfg = lm_cfg(f=f, epochs=2)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED, nsvd_norm_exp=1.0)
    for e in (1, 2):
        o.fit_epoch(e, po.SCHED_P, nsvd_norm_exp=1.0, n_threads=1)
        g.fit_epoch(tr, pr, e)
    for n in PARAMS + ["ycache", "ycache_bias"]:
        a = np.asarray(g.get_param(n), np.float64).ravel()
        b = np.asarray(o.get_param(n), np.float64).ravel()
        assert np.max(np.abs(a - b)) < 2e-5, n
    assert abs(g.calc_rmse(pr) - o.calc_rmse(pr)) < 1e-5


def test_stratified_is_bitwise_reproducible(small):
    tr, pr = small
    cfg = lm_cfg(f=32, epochs=2)
    outs = []
    for _ in range(2):
        g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED)
        for e in (1, 2):
            g.fit_epoch(tr, pr, e)
        outs.append([g.get_param(n).copy() for n in ("ufeat", "ifeat", "yfeat", "ibias", "cu")])
    for a, b in zip(*outs):
        assert np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


@pytest.mark.parametrize("schedule", [SCHED_HOGWILD, SCHED_STRATIFIED])
def test_heldout_rmse_within_0p001_of_sequential_reference(schedule):
    """C1-shaped data (smaller user count for test time), lm preset, f=32."""
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=4000, n_items=1000, n_train=400000, seed=3)
    cfg = run_lm(32, 12, n_time_bins=30)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=schedule)
    for e in range(1, cfg.n_epochs + 1):
        o.fit_epoch(e)
        g.fit_epoch(tr, pr, e)
    ro, rg = o.calc_rmse(pr), g.calc_rmse(pr)
    print(f"oracle {ro:.6f} gpu {rg:.6f}")
    assert abs(rg - ro) <= 1e-3


def test_errors_surface_as_exceptions(tiny):
    tr, pr = tiny
    from netflix_prize_b200.native import TsvdError
    with pytest.raises(TsvdError, match="not user-sorted"):
        TxModel(pr, MaskedDataset(tr), regression_test_config(low_memory=True))
    g = TxModel(tr, MaskedDataset(pr), regression_test_config(low_memory=True))
    with pytest.raises(TsvdError, match="out of range"):
        g.predict_batch(np.array([99]), np.array([0]), np.array([1]))
    with pytest.raises(TsvdError, match="1-based"):
        g.fit_epoch(tr, pr, 0)
