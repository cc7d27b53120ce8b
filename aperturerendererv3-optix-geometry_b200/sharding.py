"""Split of one offline render over several GPUs (one process per GPU).

Camera paths are independent (the reference traces one path per pixel and
sample, core/scene.cu:201-255, and only sums them), so the render shards with
no exchange during tracing: every rank traces the whole image with its own
sample streams -- frame indices [rank * spp, (rank + 1) * spp) of the
reference's per-frame seeding curand_init(seed, pixel, frame * 2^32) -- and the
per-pixel FP64 sums are added once per image with one reduce.  N ranks thus
trace N * spp samples per pixel (weak scaling).  Job time is the slowest rank's
device time; counts add over ranks.

The functions take the torch.distributed module so that the same code runs
over NCCL on GPUs and over gloo on CPU tensors.
"""
from __future__ import annotations


def rank_frame_offset(rank: int, spp: int, base: int = 0) -> int:
    """First frame index (TOTAL_FRAME_INDEX) of this rank's samples."""
    if rank < 0 or spp <= 0:
        raise ValueError("rank must be >= 0 and spp > 0")
    return base + rank * spp


def reduce_accumulators(accum, dist, dst: int = 0) -> None:
    """Sum the FP64 per-pixel accumulators of all ranks into rank dst."""
    dist.reduce(accum, dst=dst, op=dist.ReduceOp.SUM)


def job_totals(local_ms: float, counts, dist, device) -> tuple[float, list[float]]:
    """(max device time over ranks, per-counter sums over ranks)."""
    import torch
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    c = torch.tensor([float(x) for x in counts], dtype=torch.float64, device=device)
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), [float(x) for x in c.tolist()]
