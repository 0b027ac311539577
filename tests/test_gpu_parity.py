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


def test_initial_state_bitwise_12m_draws():
    """The device-side init at f=256 over ~12M normal draws (about 150k
    ziggurat wedge tests and a few thousand tail draws) equals the
    sequential host stream bit for bit."""
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=40000, n_items=400, n_train=200000, seed=5)
    cfg = lm_cfg(f=256, epochs=1)
    g = TxModel(tr, MaskedDataset(pr), cfg)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    for n in ["ufeat", "ifeat", "yfeat", "ifeat_freq"]:
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
    import copy
    pr2 = copy.copy(pr)  # the session fixture stays untouched
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


@pytest.mark.parametrize("f,heavy", [(16, 1024), (64, 1024), (256, 1024), (64, 40)])
def test_stratified_heavy_items_match_oracle_tsvdx4p(f, heavy):
    """Items with at least `heavy` ratings take the item stratum's whole-block
    path, whose serial chain runs 32 ratings per round from Gram-matrix
    lookahead; it must still follow the reference's per-rating item updates
    (heavy = 40: nearly every item, most of them ending in a partial round)."""
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=3000, n_items=80, n_train=90000, seed=13)
    assert np.bincount(tr.item_idxs, minlength=tr.n_items).max() >= 2048
    cfg = lm_cfg(f=f, epochs=2)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED, nsvd_norm_exp=1.0,
                heavy_item_ratings=heavy)
    for e in (1, 2):
        o.fit_epoch(e, po.SCHED_P, nsvd_norm_exp=1.0, n_threads=1)
        g.fit_epoch(tr, pr, e)
    for n in PARAMS + ["ycache", "ycache_bias"]:
        a = np.asarray(g.get_param(n), np.float64).ravel()
        b = np.asarray(o.get_param(n), np.float64).ravel()
        assert np.max(np.abs(a - b) - 1e-5 * np.abs(b)) < 2e-5, n
    assert abs(g.calc_rmse(pr) - o.calc_rmse(pr)) < 1e-5


def disjoint_sets(n_users=64, per_user=70, seed=5):
    """Users rate disjoint item blocks, so concurrent users never share an item
    row: Hogwild is then race-free and must equal the sequential reference.
    Several ratings per (user, day), in item order, exercise same-day updates
    at varying distances."""
    from netflix_prize_b200.data import Dataset
    rng = np.random.default_rng(seed)
    n_items = n_users * (per_user + 10)
    tu, ti, tr_, td, pu, pi, pd_ = [], [], [], [], [], [], []
    for u in range(n_users):
        items = u * (per_user + 10) + np.arange(per_user + 10)
        n_tr = int(rng.integers(per_user // 3, per_user))
        days = np.sort(rng.choice(np.arange(100, 2000), size=max(2, n_tr // 5), replace=False))
        d = rng.choice(days, size=n_tr)
        tu += [u] * n_tr
        ti += list(items[:n_tr])
        tr_ += list(rng.integers(1, 6, n_tr))
        td += list(d)
        k = int(rng.integers(1, 8))
        pu += [u] * k
        pi += list(items[per_user:per_user + k])
        pd_ += list(rng.choice(days, size=k))
    tr = Dataset.from_ratings(tu, ti, tr_, td, n_users, n_items, "disjoint_tr")
    o = np.lexsort((np.array(pu), np.array(pi)))
    pr = Dataset.from_ratings(np.array(pu)[o], np.array(pi)[o], rng.integers(1, 6, len(pu)), np.array(pd_)[o],
                              n_users, n_items, "disjoint_pr")
    return tr, pr


@pytest.mark.parametrize("f", [8, 64, 256])
def test_hogwild_equals_sequential_reference_without_races(f):
    tr, pr = disjoint_sets()
    cfg = lm_cfg(f=f, epochs=2)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_HOGWILD)
    for e in (1, 2):
        o.fit_epoch(e, po.SCHED_SEQ)
        g.fit_epoch(tr, pr, e)
    for n in PARAMS + ["ycache", "ycache_bias"]:
        a = np.asarray(g.get_param(n), np.float64).ravel()
        b = np.asarray(o.get_param(n), np.float64).ravel()
        assert np.max(np.abs(a - b)) < 2e-5, n
    assert abs(g.calc_rmse(pr) - o.calc_rmse(pr)) < 1e-5


def test_hogwild_ordinal_head_equals_sequential_without_races():
    """The ordinal head (src/lib.rs:500-609) as the tsvdx4 `o` jobs use it:
    lr_t = 0, thresholds sorted with a gap at each epoch end.  The initial
    thresholds are sorted but 2.5 -> 2.6 is closer than the 0.25 gap, so the
    epoch-end gap rule moves the third one.  (Unsorted thresholds make some
    P(Y=y) negative; the 1e-6 clamp then scales that rating's gradient by 1e6
    and the run measures exp() rounding rather than the schedule.)"""
    from netflix_prize_b200.config import OrdinalHeadConfig
    tr, pr = disjoint_sets(seed=9)
    cfg = lm_cfg(f=32, epochs=2, ordinal_head=OrdinalHeadConfig((1.5, 2.5, 2.6, 4.5), 0.25, 0.0, 0.0))
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_HOGWILD)
    for e in (1, 2):
        o.fit_epoch(e, po.SCHED_SEQ)
        g.fit_epoch(tr, pr, e)
    for n in PARAMS:
        a = np.asarray(g.get_param(n), np.float64).ravel()
        b = np.asarray(o.get_param(n), np.float64).ravel()
        assert np.max(np.abs(a - b) - 1e-6 * np.abs(b)) < 2e-5, n
    assert np.allclose(g.get_param("thresholds"), [1.5, 2.5, 2.75, 4.5], atol=1e-6, rtol=0)
    assert np.allclose(g.get_param("thresholds"), o.get_param("thresholds"), atol=0, rtol=0)
    want = o.predict_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    got = g.predict_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    assert np.max(np.abs(got - want)) < 1e-5
    assert abs(g.calc_rmse(pr) - o.calc_rmse(pr)) < 1e-5


@pytest.mark.parametrize("prec,rmse_tol,pred_tol", [(0, 2e-5, 2e-4), (1, 1e-3, 2e-2), (2, 1e-3, 2e-2)])
def test_precision_forms_against_fp64_oracle(prec, rmse_tol, pred_tol):
    """FP32 masters with FP32, BF16-item-table and BF16-everything read copies,
    each stated against the FP64 oracle running the same stratified schedule."""
    from netflix_prize_b200.abi import PREC_FP32
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=4000, n_items=1000, n_train=400000, seed=3)
    cfg = run_lm(64, 6, n_time_bins=30)
    o64 = po.OracleModel(tr, MaskedDataset(pr), cfg, fp64=True)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED, precision=prec)
    for e in range(1, cfg.n_epochs + 1):
        o64.fit_epoch(e, po.SCHED_P, nsvd_norm_exp=1.0, n_threads=1)
        g.fit_epoch(tr, pr, e)
    want = o64.predict_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    got = g.predict_batch(pr.user_idxs, pr.item_idxs, pr.dates).astype(np.float64)
    err = np.abs(got - want)
    r64, rg = o64.calc_rmse(pr), g.calc_rmse(pr)
    print(f"precision {prec}: max|pred - fp64| {err.max():.3e} mean {err.mean():.3e}; "
          f"rmse {rg:.6f} vs fp64 {r64:.6f} (diff {rg - r64:+.2e})")
    assert abs(rg - r64) < rmse_tol
    assert err.max() < pred_tol


def test_bf16_copies_need_stratified(small):
    from netflix_prize_b200.abi import PREC_BF16_READ
    from netflix_prize_b200.native import TsvdError
    tr, pr = small
    with pytest.raises(TsvdError, match="stratified"):
        TxModel(tr, MaskedDataset(pr), lm_cfg(), schedule=SCHED_HOGWILD, precision=PREC_BF16_READ)


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


def test_predict_batch_device_matches_host_and_flags_out_of_range_rows(small):
    """tsvd_predict_batch_device (device pointers, no host row checks) equals
    the host entry point on valid rows; a row whose user or item index is out
    of range reads no table and gets NaN."""
    import ctypes as C
    import torch
    from netflix_prize_b200 import native
    tr, pr = small
    g = TxModel(tr, MaskedDataset(pr), lm_cfg(f=40))
    g.fit_epoch(tr, pr, 1)
    want = g.predict_batch(pr.user_idxs, pr.item_idxs, pr.dates)
    u, i = pr.user_idxs.copy(), pr.item_idxs.copy()
    u[3], i[5], u[7] = pr.n_users + 10, pr.n_items, -4
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    du, di, dd = dev(u), dev(i), dev(pr.dates)
    out = torch.empty(pr.n_ratings, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = native.load().tsvd_predict_batch_device(g.h, C.c_void_p(du.data_ptr()), C.c_void_p(di.data_ptr()),
                                                 C.c_void_p(dd.data_ptr()), pr.n_ratings, C.c_void_p(out.data_ptr()))
    assert rc == 0
    g.synchronize()
    got = out.cpu().numpy()
    bad = np.zeros(pr.n_ratings, bool)
    bad[[3, 5, 7]] = True
    assert np.isnan(got[bad]).all()
    assert np.array_equal(got[~bad], want[~bad])
