"""Multi-GPU plumbing of the batched multiply: one process per GPU, each an
independent replica over its own ciphertext pairs (no data-path collective:
pairs are independent), timed as the maximum over ranks.

Backends: "nccl" on GPUs, "gloo" for CPU runs of the same logic (tests)."""
from __future__ import annotations

import datetime
import os

ENC_ID_STRIDE = 1_000_000  # encryption ids of rank r start at r * ENC_ID_STRIDE


def world_from_env():
    """(world, rank, local_rank) as torchrun exports them (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0):
    """Join the process group if WORLD_SIZE > 1; returns (world, rank, local)."""
    world, rank, local = world_from_env()
    if world > 1:
        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, **kw)
    return world, rank, local


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world: int, value: float) -> float:
    """The slowest rank's time: the job's time."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def enc_id_base(rank: int) -> int:
    """first encryption id of this rank's inputs (ranks never share ids)"""
    return rank * ENC_ID_STRIDE


def job_rate(world: int, units_per_rank: int, ms_max: float) -> float:
    """whole-job throughput: units on all ranks over the slowest rank's time"""
    return world * units_per_rank / (ms_max / 1e3)


def finish(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
