"""The replica path's collectives (bench.py --gpus N) on CPU: two gloo ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch

    from netflix_prize_b200 import dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    torch.distributed.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    w, r, lr = dist.world_rank_local()
    assert (w, r, lr) == (world, rank, rank)
    dist.barrier(world, device="cpu")
    out[rank] = dist.max_over_ranks(10.0 + rank, world, device="cpu")
    torch.distributed.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert dict(out) == {0: 11.0, 1: 11.0}


def test_single_process_needs_no_group():
    from netflix_prize_b200 import dist
    assert dist.max_over_ranks(3.5, 1, device="cpu") == 3.5
    dist.barrier(1, device="cpu")
