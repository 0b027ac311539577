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
    g = TxGroup(tr, MaskedDataset(pr), cfgs)
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
    g = TxGroup(tr, MaskedDataset(pr), cfgs)
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
    g = TxGroup(tr, MaskedDataset(pr), cfgs)
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
