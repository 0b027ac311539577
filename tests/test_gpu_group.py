"""The batched form (several variants in one persistent launch per epoch).

On data where users rate disjoint items, Hogwild has no races, so every
variant trained inside the group must equal the sequential reference
(TxModel::fit_epoch) run on that variant alone, within FP32 rounding (2e-5),
whether the epoch is launched directly or replayed from the captured CUDA
graph. On shared-item data each variant's held-out RMSE must stay within
+-0.001 of its sequential reference.
"""
import numpy as np
import pytest

from netflix_prize_b200.abi import SCHED_HOGWILD, SCHED_STRATIFIED
from netflix_prize_b200.config import run_lm
from netflix_prize_b200.data import MaskedDataset
from netflix_prize_b200.model import TxGroup
from oracle import pyoracle as po
from tests.test_gpu_parity import PARAMS, disjoint_sets

pytestmark = pytest.mark.gpu


def variants():
    base = run_lm(8, 3, n_time_bins=30)
    return [base.replace(n_feat=8, lr_u=0.003, lr_i=0.003, seed=1),
            base.replace(n_feat=32, lr_u=0.007, lr_i=0.007, reg_u=0.015, reg_i=0.015, seed=2),
            base.replace(n_feat=64, lr_u=0.003, lr_i=0.003, reg_u=0.005, reg_i=0.005, seed=3),
            base.replace(n_feat=256, lr_u=0.007, lr_i=0.007, seed=4)]


@pytest.mark.parametrize("graphs", [True, False])
def test_group_variants_equal_sequential_reference_without_races(graphs):
    tr, pr = disjoint_sets()
    cfgs = variants()
    g = TxGroup(tr, MaskedDataset(pr), cfgs, schedule=SCHED_HOGWILD)
    g.set_graphs(graphs)
    oracles = [po.OracleModel(tr, MaskedDataset(pr), c) for c in cfgs]
    for e in (1, 2, 3):
        g.fit_epoch(e)
        for o in oracles:
            o.fit_epoch(e, po.SCHED_SEQ)
    for k, (m, o) in enumerate(zip(g.models, oracles)):
        for n in PARAMS + ["ycache", "ycache_bias"]:
            a = np.asarray(m.get_param(n), np.float64).ravel()
            b = np.asarray(o.get_param(n), np.float64).ravel()
            assert np.max(np.abs(a - b)) < 2e-5, (k, n)
        assert abs(m.calc_rmse(pr) - o.calc_rmse(pr)) < 1e-5
    assert g.last_epoch_ms() > 0


def test_group_heldout_rmse_matches_each_sequential_variant():
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=4000, n_items=1000, n_train=400000, seed=3)
    cfgs = [c.replace(n_epochs=8) for c in variants()[:3]]
    g = TxGroup(tr, MaskedDataset(pr), cfgs, schedule=SCHED_HOGWILD)
    oracles = [po.OracleModel(tr, MaskedDataset(pr), c) for c in cfgs]
    for e in range(1, 9):
        g.fit_epoch(e)
        for o in oracles:
            o.fit_epoch(e, po.SCHED_SEQ)
    for m, o in zip(g.models, oracles):
        rg, ro = m.calc_rmse(pr), o.calc_rmse(pr)
        print(f"f={m.cfg.n_feat}: group {rg:.6f} sequential {ro:.6f}")
        assert abs(rg - ro) <= 1e-3


def test_group_autotune_picks_a_depth_per_width_and_keeps_training_exact():
    tr, pr = disjoint_sets()
    cfgs = variants()
    g = TxGroup(tr, MaskedDataset(pr), cfgs, schedule=SCHED_HOGWILD)
    before = [m.get_param("ifeat").copy() for m in g.models]
    stages = g.autotune(sample_users=32)
    assert all(s in (2, 3, 4) for s in stages)
    for m, b in zip(g.models, before):  # tuning ran on throwaway copies
        assert np.array_equal(m.get_param("ifeat"), b)
    o = po.OracleModel(tr, MaskedDataset(pr), cfgs[3])
    g.fit_epoch(1)
    o.fit_epoch(1, po.SCHED_SEQ)
    a = np.asarray(g.models[3].get_param("ufeat"), np.float64).ravel()
    assert np.max(np.abs(a - np.asarray(o.get_param("ufeat")))) < 2e-5


@pytest.mark.parametrize("graphs", [True, False])
def test_stratified_group_variants_equal_their_single_models(graphs):
    """Stratified variants trained together (parallel streams, one captured
    graph per epoch from the second on) equal, bit for bit, the same variants
    trained one at a time: the schedule is deterministic."""
    from netflix_prize_b200.model import TxModel
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=3000, n_items=80, n_train=90000, seed=13)
    cfgs = [c.replace(reset_u_epoch=3, n_epochs=4) for c in variants()]
    g = TxGroup(tr, MaskedDataset(pr), cfgs, schedule=SCHED_STRATIFIED)
    g.set_graphs(graphs)
    singles = [TxModel(tr, MaskedDataset(pr), c, heavy_item_ratings=0) for c in cfgs]
    for e in (1, 2, 3, 4):
        g.fit_epoch(e)
        for m in singles:
            m.fit_epoch(tr, pr, e)
    for k, (gm, sm) in enumerate(zip(g.models, singles)):
        for n in PARAMS + ["ycache", "ycache_bias"]:
            a = np.asarray(gm.get_param(n), np.float32)
            b = np.asarray(sm.get_param(n), np.float32)
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (k, n)
    assert g.last_epoch_ms() > 0


def test_stratified_group_autotune_picks_thresholds_and_keeps_results():
    """The autotuner picks each variant's whole-CTA threshold on throwaway
    copies; the group's own parameters are untouched and training still
    follows the oracle's Tsvdx4pModel epoch."""
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=3000, n_items=80, n_train=90000, seed=13)
    cfgs = variants()
    g = TxGroup(tr, MaskedDataset(pr), cfgs, schedule=SCHED_STRATIFIED)
    before = [m.get_param("ifeat").copy() for m in g.models]
    thr = g.autotune()
    assert all(t in (0x7fffffff, 65536, 32768, 16384, 8192, 4096) for t in thr)
    for m, b in zip(g.models, before):
        assert np.array_equal(m.get_param("ifeat"), b)
    o = po.OracleModel(tr, MaskedDataset(pr), cfgs[2])
    g.fit_epoch(1)
    o.fit_epoch(1, po.SCHED_P, nsvd_norm_exp=1.0, n_threads=1)
    for n in PARAMS:
        a = np.asarray(g.models[2].get_param(n), np.float64).ravel()
        b = np.asarray(o.get_param(n), np.float64).ravel()
        assert np.max(np.abs(a - b) - 1e-5 * np.abs(b)) < 2e-5, n
