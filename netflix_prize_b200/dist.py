"""Process-group helpers for multi-GPU runs (bench.py --gpus N): the timing
barrier and the max-over-ranks of a timed duration. The epoch's own
collectives are in shard.py. `device` is "cuda" on GPUs and "cpu" under the
gloo backend (tests)."""
from __future__ import annotations

import os


def world_rank_local() -> tuple[int, int, int]:
    """WORLD_SIZE, RANK, LOCAL_RANK from the launcher's environment (1, 0, 0 without one)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def barrier(world: int, device: str = "cuda") -> None:
    import torch
    if world > 1:
        torch.distributed.barrier()
    if device == "cuda":
        torch.cuda.synchronize()


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The slowest rank's value: multi-GPU numbers are timed as the max over ranks."""
    if world == 1:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())
