"""The sharded stratified epoch (netflix_prize_b200/shard.py) on CPU: two gloo
ranks, each with the oracle as its engine, against the oracle's one-process
Tsvdx4pModel epochs (src/tsvdx4p.rs:815-822). Only the order of the NSVD1
delta additions differs, so every parameter must agree within 2e-5 after two
epochs, with and without the per-day terms."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

PARAMS = ["ubias", "ibias", "ufeat", "ufeat2", "ifeat", "yfeat", "alpha_u", "but_bin", "bit_bin", "ybias",
          "ubias_day", "ibias_freq", "ifeat_freq", "cu", "cut", "ycache", "ycache_bias"]
DAY_PARAMS = ["yfeat_day", "ufeat_day", "ycache_day"]


class OracleEngine:
    """The sharded steps over the CPU oracle (test only)."""

    def __init__(self, o, tr, pr, cfg):
        self.o, self.cfg = o, cfg
        self.per_day = not cfg.low_memory
        self.n_freq_bins = cfg.n_freq_bins
        # SparseUD (src/tx.rs:21-84): a user's distinct days over train and pr
        u = np.concatenate([tr.user_idxs, pr.user_idxs]).astype(np.int64)
        d = np.concatenate([tr.dates, pr.dates]).astype(np.int64)
        pairs = np.unique(u * 65536 + d)
        cnt = np.bincount(pairs // 65536, minlength=tr.n_users)
        self.ud_start = np.concatenate([[0], np.cumsum(cnt)])

    def cols(self, name):
        c = self.cfg
        return {"ufeat": c.n_feat, "ufeat2": c.n_feat, "ufeat_day": c.n_feat, "ifeat": c.n_feat,
                "ifeat_freq": c.n_feat, "but_bin": c.n_time_bins, "bit_bin": c.n_time_bins,
                "ibias_freq": c.n_freq_bins}.get(name, 1)

    def user_day_range(self, lo, hi):
        return int(self.ud_start[lo]), int(self.ud_start[hi])

    def user_block(self, epoch, lo, hi):
        import torch
        d = self.o.user_block_p(epoch, lo, hi)
        return {k: torch.from_numpy(np.ascontiguousarray(v)) for k, v in d.items() if v is not None}

    def apply_deltas(self, d):
        self.o.apply_deltas_p({k: d[k].numpy() if k in d else None for k in ("dy", "dyb", "dyd", "nc")}, 1.0)

    def item_block(self, lo, hi):
        self.o.item_block_p(lo, hi)

    def get_rows(self, name, lo, hi):
        import torch
        c = self.cols(name)
        return torch.from_numpy(self.o.get_param(name).reshape(-1, c)[lo:hi].ravel().copy())

    def set_rows(self, name, lo, hi, t):
        c = self.cols(name)
        full = self.o.get_param(name).reshape(-1, c)
        full[lo:hi] = t.numpy().reshape(hi - lo, c)
        self.o.set_param(name, full)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _data():
    from tests.conftest import small_sets
    return small_sets(n_users=500, n_items=120, n_train=25000, seed=23)


def _cfg(low_memory):
    from netflix_prize_b200.config import run_lm
    return run_lm(16, 2, n_time_bins=30, low_memory=low_memory).replace(reset_u_epoch=2)


def _rank(rank, world, port, low_memory, out):
    import datetime

    import torch

    from netflix_prize_b200.data import MaskedDataset
    from netflix_prize_b200.shard import Partition, ShardedEpochs, TorchComm
    from oracle import pyoracle as po
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=120))
    tr, pr = _data()
    cfg = _cfg(low_memory)
    o = po.OracleModel(tr, MaskedDataset(pr), cfg)
    sh = ShardedEpochs(OracleEngine(o, tr, pr, cfg), rank, Partition.for_data(tr, world), TorchComm(world, rank))
    for e in (1, 2):
        sh.fit_epoch(e)
    names = PARAMS + (DAY_PARAMS if not low_memory else [])
    out[rank] = {n: o.get_param(n) for n in names}
    torch.distributed.destroy_process_group()


@pytest.mark.parametrize("low_memory", [True, False])
def test_two_rank_sharded_epochs_equal_one_process_epochs(low_memory):
    from netflix_prize_b200.data import MaskedDataset
    from oracle import pyoracle as po
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, low_memory, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        got = dict(out)
    tr, pr = _data()
    cfg = _cfg(low_memory)
    ref = po.OracleModel(tr, MaskedDataset(pr), cfg)
    for e in (1, 2):
        ref.fit_epoch(e, po.SCHED_P, nsvd_norm_exp=1.0, n_threads=1)
    for n, a in got[0].items():
        b = ref.get_param(n)
        assert np.array_equal(a, got[1][n]), n                 # every rank holds the same model
        assert np.max(np.abs(a - b)) < 2e-5, (n, float(np.max(np.abs(a - b))))


def test_balanced_blocks_cover_every_id_once():
    from netflix_prize_b200.shard import balanced_blocks
    counts = np.random.default_rng(1).integers(0, 100, 1000)
    for parts in (1, 2, 3, 8):
        b = balanced_blocks(counts, parts)
        assert b[0][0] == 0 and b[-1][1] == 1000
        assert all(b[k][1] == b[k + 1][0] for k in range(parts - 1))
        sums = [counts[lo:hi].sum() for lo, hi in b]
        assert max(sums) - min(sums) <= 2 * counts.max()
