"""The sharded stratified epoch's GPU steps (tsvd_shard_*, tsvd_copy_rows)
through the C ABI, on one GPU: P ranks emulated in one process, each with its
own model, their collectives served in lockstep (a sum of the ranks' tensors,
or the list of their blocks). Every parameter after two epochs must agree
within 2e-5 with the one-model stratified epochs (only the order of the NSVD1
delta additions differs), and every rank must hold the same model."""
import numpy as np
import pytest

from netflix_prize_b200.config import run_lm
from netflix_prize_b200.data import MaskedDataset
from netflix_prize_b200.model import TxModel
from netflix_prize_b200.shard import GpuEngine, Partition, ShardedEpochs

pytestmark = pytest.mark.gpu

PARAMS = ["ubias", "ibias", "ufeat", "ufeat2", "ifeat", "yfeat", "alpha_u", "but_bin", "bit_bin", "ybias",
          "ubias_day", "ibias_freq", "ifeat_freq", "cu", "cut", "ycache", "ycache_bias"]
DAY_PARAMS = ["yfeat_day", "ufeat_day", "ycache_day"]


def lockstep(shards, epoch):
    """Runs the ranks' steps, serving each collective across all of them."""
    gens = [s.steps(epoch) for s in shards]
    reqs = [next(g) for g in gens]
    while True:
        kind = reqs[0][0]
        assert all(r[0] == kind for r in reqs)
        if kind == "sum":
            total = reqs[0][1].clone()
            for r in reqs[1:]:
                total += r[1]
            res = [total.clone() for _ in reqs]
        else:
            parts = [r[1] for r in reqs]
            res = [parts for _ in reqs]
        nxt, done = [], 0
        for g, x in zip(gens, res):
            try:
                nxt.append(g.send(x))
            except StopIteration:
                done += 1
        if done:
            assert done == len(gens)
            return
        reqs = nxt


@pytest.mark.parametrize("f,low_memory,ranks,heavy", [(16, True, 2, 0), (64, False, 2, 0), (32, True, 3, 40),
                                                      (400, True, 2, 0)])
def test_emulated_ranks_equal_one_model(f, low_memory, ranks, heavy):
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=3000, n_items=80, n_train=90000, seed=13) if heavy else small_sets()
    cfg = run_lm(f, 2, n_time_bins=30, low_memory=low_memory).replace(reset_u_epoch=2)
    one = TxModel(tr, MaskedDataset(pr), cfg, heavy_item_ratings=heavy)
    models = [TxModel(tr, MaskedDataset(pr), cfg, heavy_item_ratings=heavy) for _ in range(ranks)]
    part = Partition.for_data(tr, ranks)
    shards = [ShardedEpochs(GpuEngine(m), r, part) for r, m in enumerate(models)]
    for e in (1, 2):
        one.fit_epoch(tr, pr, e)
        lockstep(shards, e)
    names = PARAMS + ([] if low_memory else DAY_PARAMS)
    for n in names:
        want = np.asarray(one.get_param(n), np.float64).ravel()
        for m in models:
            got = np.asarray(m.get_param(n), np.float64).ravel()
            assert np.max(np.abs(got - want) - 1e-5 * np.abs(want)) < 2e-5, (n, float(np.max(np.abs(got - want))))
        a0 = np.asarray(models[0].get_param(n), np.float32)
        for m in models[1:]:
            assert np.array_equal(a0, np.asarray(m.get_param(n), np.float32)), n
    assert abs(models[0].calc_rmse(pr) - one.calc_rmse(pr)) < 1e-5
