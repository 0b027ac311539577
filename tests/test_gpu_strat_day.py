"""The deterministic stratified schedule on every tsvdx4 configuration, through
the C ABI: the per-day NSVD1 terms (low_memory = false), the ordinal head
(lr_t = 0) and Tsvdx4pConfig::seq_epochs, against the oracle.

Tolerances as in test_gpu_parity: one or two epochs from identical state
within 2e-5 of the oracle's Tsvdx4pModel epoch per parameter; the reference's
known answer within 1e-5; training runs within +-0.001 held-out RMSE of the
sequential reference.
"""
import numpy as np
import pytest

from netflix_prize_b200.abi import SCHED_STRATIFIED
from netflix_prize_b200.config import OrdinalHeadConfig, regression_test_config, run_lm
from netflix_prize_b200.data import MaskedDataset
from netflix_prize_b200.model import TxModel
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

PARAMS = ["ubias", "ibias", "ufeat", "ufeat2", "ifeat", "yfeat", "alpha_u", "but_bin", "bit_bin", "ybias",
          "ubias_day", "ibias_freq", "ifeat_freq", "cu", "cut"]
DAY_PARAMS = ["yfeat_day", "ufeat_day", "ycache_day"]


def test_default_schedule_is_stratified(tiny):
    """A NULL options pointer gives the stratified schedule: its epoch equals,
    bit for bit, that of a model created with the schedule named."""
    import ctypes as C
    from netflix_prize_b200 import native
    tr, pr = tiny
    L = native.load()
    cfg = regression_test_config()
    c = cfg.to_c()
    h = C.c_void_p()
    assert L.tsvd_create(C.byref(c), None, C.byref(tr.view()), C.byref(pr.view(masked=True)), C.byref(h)) == 0
    try:
        assert L.tsvd_fit_epoch(h, 1) == 0
        n = C.c_uint64()
        assert L.tsvd_param_nbytes(h, b"ifeat", C.byref(n)) == 0
        got = np.empty(n.value // 4, np.float32)
        assert L.tsvd_get_param(h, b"ifeat", got.ctypes.data_as(C.c_void_p), n.value) == 0
    finally:
        L.tsvd_destroy(h)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED)
    g.fit_epoch(tr, pr, 1)
    want = np.asarray(g.get_param("ifeat"), np.float32).ravel()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert TxModel.__init__.__defaults__[0] == SCHED_STRATIFIED


def test_stratified_reproduces_tsvdx4p_known_answer(tiny, golden):
    """tsvdx4p_probe_rmse_regression (tests/regressors_test.rs:157-175):
    low_memory = false, nsvd_norm_exp 0.5, reset_u_epoch 1, 3 epochs."""
    tr, pr = tiny
    cfg = regression_test_config(reset_u_epoch=1)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED, nsvd_norm_exp=0.5)
    for e in range(1, cfg.n_epochs + 1):
        g.fit_epoch(tr, pr, e)
    want = 1.02037806773939
    got = g.calc_rmse(pr)
    print(f"tsvdx4p known answer {want!r}, GPU stratified {got!r}")
    assert abs(got - want) < 1e-5


@pytest.mark.parametrize("f,has_ud", [(16, True), (60, True), (64, False), (160, True)])
def test_stratified_day_epochs_match_oracle_tsvdx4p(small, f, has_ud):
    """Two stratified epochs with the per-day terms against the oracle's
    Tsvdx4pModel (src/tsvdx4p.rs:390-805, !low_memory branches)."""
    tr, pr = small
    cfg = run_lm(f, 2, n_time_bins=30, low_memory=False)
    if not has_ud:
        cfg = cfg.replace(lr_ud=0.0)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED, nsvd_norm_exp=1.0)
    for e in (1, 2):
        o.fit_epoch(e, po.SCHED_P, nsvd_norm_exp=1.0, n_threads=1)
        g.fit_epoch(tr, pr, e)
    for n in PARAMS + DAY_PARAMS + ["ycache", "ycache_bias"]:
        a = np.asarray(g.get_param(n), np.float64).ravel()
        b = np.asarray(o.get_param(n), np.float64).ravel()
        assert np.max(np.abs(a - b)) < 2e-5, n
    assert abs(g.calc_rmse(pr) - o.calc_rmse(pr)) < 1e-5


def test_stratified_seq_epochs_follow_the_oracle():
    """seq_epochs = [1, 3]: epochs 1 and 3 are TxModel::fit_epoch, epoch 2 the
    parallel one (Tsvdx4pModel::fit_epoch, src/tsvdx4p.rs:815-822)."""
    from tests.test_gpu_parity import disjoint_sets
    tr, pr = disjoint_sets(seed=3)
    cfg = run_lm(32, 3, n_time_bins=30)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED, seq_epochs=(1, 3))
    for e, sch in ((1, po.SCHED_SEQ), (2, po.SCHED_P), (3, po.SCHED_SEQ)):
        o.fit_epoch(e, sch, nsvd_norm_exp=1.0, n_threads=1)
        g.fit_epoch(tr, pr, e)
    for n in PARAMS + ["ycache", "ycache_bias"]:
        a = np.asarray(g.get_param(n), np.float64).ravel()
        b = np.asarray(o.get_param(n), np.float64).ravel()
        assert np.max(np.abs(a - b)) < 2e-5, n


def test_seq_epochs_need_the_stratified_schedule(tiny):
    from netflix_prize_b200.abi import SCHED_HOGWILD
    from netflix_prize_b200.native import TsvdError
    tr, pr = tiny
    with pytest.raises(TsvdError, match="seq_epochs"):
        TxModel(tr, MaskedDataset(pr), regression_test_config(), schedule=SCHED_HOGWILD, seq_epochs=(1,))


@pytest.mark.parametrize("low_memory", [False, True])
def test_stratified_ordinal_head_tracks_sequential_reference(low_memory):
    """The `o` jobs' ordinal head (lr_t = 0, src/bin/tsvdx4-new.rs:163-200)
    on the stratified schedule: held-out RMSE within 0.001 of the sequential
    reference after 8 epochs."""
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=3000, n_items=800, n_train=250000, seed=21)
    cfg = run_lm(32, 8, n_time_bins=20, low_memory=low_memory).replace(
        ordinal_head=OrdinalHeadConfig((0.5, 1.25, 3.75, 5.5), 0.001, 0.0, 0.0), seed=64)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED)
    for e in range(1, cfg.n_epochs + 1):
        o.fit_epoch(e)
        g.fit_epoch(tr, pr, e)
    ro, rg = o.calc_rmse(pr), g.calc_rmse(pr)
    print(f"ordinal head, low_memory={low_memory}: oracle sequential {ro:.6f}, GPU stratified {rg:.6f}")
    assert abs(rg - ro) <= 1e-3


def test_stratified_day_heldout_tracks_sequential_reference():
    """tsvdx4-60-style run (low_memory = false) on C1-shaped data: held-out
    RMSE within 0.001 of the sequential reference after 10 epochs."""
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=4000, n_items=1000, n_train=400000, seed=3)
    cfg = run_lm(60, 10, n_time_bins=30, low_memory=False)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED)
    for e in range(1, cfg.n_epochs + 1):
        o.fit_epoch(e)
        g.fit_epoch(tr, pr, e)
    ro, rg = o.calc_rmse(pr), g.calc_rmse(pr)
    print(f"per-day terms: oracle sequential {ro:.6f}, GPU stratified {rg:.6f}")
    assert abs(rg - ro) <= 1e-3
