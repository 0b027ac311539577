"""Sharded stratified epochs: one process per GPU, one model per process.

The reference's parallel schedule (Tsvdx4pModel::fit_epoch,
src/tsvdx4p.rs:815-822) split over P processes:

  user stratum   process r trains the users of user block r (item tables
                 frozen and replicated, src/tsvdx4p.rs:390-639) and sums its
                 users' NSVD1 deltas per item (NsvdDelta, :63-80);
  all-reduce     the per-item delta sums (the one collective of the path's
                 math: :346-355 add the threads' buffers);
  all-gather     the user blocks' rows, so every process holds every user;
  apply          apply_nsvd_deltas (:341-385) and the cache rebuild, the same
                 on every process;
  item stratum   process r trains the items of item block r (:644-762);
  all-gather     the item blocks' rows, so every process holds the model.

Blocks are contiguous id ranges balanced by rating count. The results equal
the one-process stratified epoch up to the order of the delta additions.

`ShardedEpochs` is written against two small interfaces so the same
orchestration runs on GPUs (`GpuEngine` over the C ABI, `TorchComm` over
torch.distributed with NCCL) and in CPU tests (an oracle-backed engine over
gloo).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

# user-side tables a user block owns, and their row space ("user" or "ud")
USER_TABLES = [("ufeat", "user"), ("ufeat2", "user"), ("ubias", "user"), ("alpha_u", "user"), ("cu", "user"),
               ("but_bin", "user"), ("ubias_day", "ud")]
USER_DAY_TABLES = [("ufeat_day", "ud")]
# item-side tables an item block owns ("item" rows, or n_freq_bins rows per item)
ITEM_TABLES = [("ifeat", "item"), ("ifeat_freq", "item_freq"), ("ibias", "item"), ("bit_bin", "item"),
               ("ibias_freq", "item")]


def balanced_blocks(counts: np.ndarray, parts: int) -> list[tuple[int, int]]:
    """Contiguous id ranges [lo, hi) with about equal sums of `counts`."""
    counts = np.asarray(counts, np.int64)
    n = len(counts)
    cum = np.concatenate([[0], np.cumsum(counts)])
    total = int(cum[-1])
    cuts = [0]
    for r in range(1, parts):
        c = int(np.searchsorted(cum, total * r / parts, side="left"))
        cuts.append(min(max(c, cuts[-1]), n))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(parts)]


@dataclass
class Partition:
    users: list      # [(u_lo, u_hi)] per rank
    items: list      # [(i_lo, i_hi)] per rank

    @staticmethod
    def for_data(tr, parts: int) -> "Partition":
        return Partition(balanced_blocks(tr.user_cnts, parts), balanced_blocks(tr.item_cnts, parts))


class TorchComm:
    """Collectives of the sharded epoch over torch.distributed (NCCL on GPUs,
    gloo on CPU). Uneven blocks travel padded to the longest one."""

    def __init__(self, world: int, rank: int):
        self.world, self.rank = world, rank

    def all_reduce_sum(self, t):
        import torch.distributed as dist
        dist.all_reduce(t)
        return t

    def all_gather_rows(self, mine, lengths: list):
        """Each rank's flat `mine` (its block's length) -> list of every rank's."""
        import torch
        import torch.distributed as dist
        n = max(lengths)
        buf = torch.zeros(n, dtype=mine.dtype, device=mine.device)
        buf[:mine.numel()] = mine.reshape(-1)
        out = [torch.empty_like(buf) for _ in range(self.world)]
        dist.all_gather(out, buf)
        return [out[r][:lengths[r]] for r in range(self.world)]


class ShardedEpochs:
    """The steps of a sharded stratified epoch for one rank's engine.

    `steps(epoch)` is a generator that yields at each collective, ("sum", t)
    or ("gather", mine, lengths), and is sent the result; `fit_epoch` serves
    those requests with a TorchComm. A single process can drive several
    ranks' generators in lockstep instead (one GPU emulating P ranks)."""

    def __init__(self, engine, rank: int, part: Partition, comm=None):
        self.e, self.rank, self.part, self.comm = engine, rank, part, comm

    def _rows(self, space: str, lo: int, hi: int) -> tuple[int, int]:
        if space == "ud":
            return self.e.user_day_range(lo, hi)
        if space == "item_freq":
            nf = self.e.n_freq_bins
            return lo * nf, hi * nf
        return lo, hi

    def _exchange(self, tables, blocks):
        for name, space in tables:
            ranges = [self._rows(space, lo, hi) for lo, hi in blocks]
            cols = self.e.cols(name)
            lengths = [(b - a) * cols for a, b in ranges]
            if max(lengths) == 0:  # n_feat = 0 tables, or no days
                continue
            mine = self.e.get_rows(name, *ranges[self.rank])
            parts = yield ("gather", mine, lengths)
            for r, (a, b) in enumerate(ranges):
                if r != self.rank and b > a:
                    self.e.set_rows(name, a, b, parts[r])

    def steps(self, epoch: int):
        u_lo, u_hi = self.part.users[self.rank]
        deltas = self.e.user_block(epoch, u_lo, u_hi)
        for k in sorted(deltas):
            deltas[k] = yield ("sum", deltas[k])
        tables = USER_TABLES + (USER_DAY_TABLES if self.e.per_day else [])
        yield from self._exchange(tables, self.part.users)
        self.e.apply_deltas(deltas)
        self.e.item_block(*self.part.items[self.rank])
        yield from self._exchange(ITEM_TABLES, self.part.items)

    def fit_epoch(self, epoch: int):
        g = self.steps(epoch)
        try:
            req = next(g)
            while True:
                if req[0] == "sum":
                    res = self.comm.all_reduce_sum(req[1])
                else:
                    res = self.comm.all_gather_rows(req[1], req[2])
                req = g.send(res)
        except StopIteration:
            pass


class GpuEngine:
    """The sharded steps of one TxModel (stratified, FP32) over the C ABI;
    buffers are torch tensors on the model's device."""

    def __init__(self, model):
        import torch
        self.m, self.L = model, model._L
        self.device = torch.device("cuda", model.device)
        w = C.c_uint32()
        model._check(self.L.tsvd_row_width(model.h, C.byref(w)))
        self.Fs = w.value
        self.per_day = not model.cfg.low_memory
        self.n_freq_bins = model.cfg.n_freq_bins
        self.n_items = model.n_items

    def cols(self, name: str) -> int:
        c = self.m.cfg
        return {"ufeat": c.n_feat, "ufeat2": c.n_feat, "ufeat_day": c.n_feat, "ifeat": c.n_feat,
                "ifeat_freq": c.n_feat, "but_bin": c.n_time_bins, "bit_bin": c.n_time_bins,
                "ibias_freq": c.n_freq_bins}.get(name, 1)

    def user_day_range(self, u_lo, u_hi):
        a, b = C.c_uint64(), C.c_uint64()
        self.m._check(self.L.tsvd_user_day_range(self.m.h, u_lo, u_hi, C.byref(a), C.byref(b)))
        return a.value, b.value

    def user_block(self, epoch, u_lo, u_hi):
        import torch
        d = {"sums": torch.empty((self.n_items, self.Fs), dtype=torch.float32, device=self.device),
             "sums_e": torch.empty(self.n_items, dtype=torch.float32, device=self.device)}
        if self.per_day:
            d["dyd"] = torch.empty((self.n_items, self.Fs), dtype=torch.int64, device=self.device)
        torch.cuda.synchronize(self.device)
        self.m._check(self.L.tsvd_shard_user_block(self.m.h, epoch, u_lo, u_hi, C.c_void_p(d["sums"].data_ptr()),
                                                   C.c_void_p(d["sums_e"].data_ptr()),
                                                   C.c_void_p(d["dyd"].data_ptr()) if self.per_day else None))
        return d

    def apply_deltas(self, d):
        import torch
        torch.cuda.synchronize(self.device)
        self.m._check(self.L.tsvd_shard_apply(self.m.h, C.c_void_p(d["sums"].data_ptr()),
                                              C.c_void_p(d["sums_e"].data_ptr()),
                                              C.c_void_p(d["dyd"].data_ptr()) if self.per_day else None))

    def item_block(self, i_lo, i_hi):
        self.m._check(self.L.tsvd_shard_item_block(self.m.h, i_lo, i_hi))

    def get_rows(self, name, lo, hi):
        import torch
        t = torch.empty((hi - lo) * self.cols(name), dtype=torch.float32, device=self.device)
        if hi > lo:
            self.m._check(self.L.tsvd_copy_rows(self.m.h, name.encode(), lo, hi, C.c_void_p(t.data_ptr()), 0))
        return t

    def set_rows(self, name, lo, hi, t):
        import torch
        t = t.contiguous()
        torch.cuda.synchronize(self.device)
        self.m._check(self.L.tsvd_copy_rows(self.m.h, name.encode(), lo, hi, C.c_void_p(t.data_ptr()), 1))
