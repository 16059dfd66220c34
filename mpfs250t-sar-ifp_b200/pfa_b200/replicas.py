"""Replica parallelism over independent frames (one process per GPU, torch.distributed).

PFA frames are independent, so N GPUs run N replicas: frames are dealt round-robin to ranks, every rank
forms its own frames with no data-path collective, and only the timing (max over ranks) and, when
asked, the per-frame results (gathered to rank 0) cross processes.  Works with any torch.distributed
backend: NCCL on GPUs, gloo on CPU (the tests).
"""
from __future__ import annotations


def world():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def shard(n_frames: int, rank: int, world_size: int) -> list:
    """Frame indices owned by `rank` (round robin, so uneven frame lists stay balanced)."""
    return list(range(rank, n_frames, world_size))


def _tensor_device():
    import torch
    import torch.distributed as dist
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x: float) -> float:
    ws, _ = world()
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_tensor_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    ws, _ = world()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def gather_results(local: dict) -> dict | None:
    """{frame index: result} from every rank, merged on rank 0 (None elsewhere)."""
    ws, rank = world()
    if ws == 1:
        return dict(local)
    import torch.distributed as dist
    parts = [None] * ws if rank == 0 else None
    dist.gather_object(local, parts, dst=0)
    if rank != 0:
        return None
    merged = {}
    for p in parts:
        merged.update(p)
    return merged


def ms_per_frame(elapsed_ms_this_rank: float, frames_total: int) -> float:
    """Whole-job time per frame: the slowest rank's elapsed time over all frames of all ranks."""
    return max_over_ranks(elapsed_ms_this_rank) / max(frames_total, 1)
