"""Split of one offline render over several GPUs (one process per GPU).

Camera paths are independent (the reference traces one path per pixel and
sample, core/scene.cu:201-255, and only sums them), so the render shards with
no exchange during tracing: every rank traces the whole image with its own
sample streams -- frame indices [rank * spp, (rank + 1) * spp) of the
reference's per-frame seeding curand_init(seed, pixel, frame * 2^32) -- and the
per-pixel FP64 sums are added once per image with one reduce.  N ranks thus
trace N * spp samples per pixel (weak scaling).  Job time is the slowest rank's
device time; counts add over ranks.

A batch of independent render jobs (ar_render_batch) shards by job instead:
partition_jobs assigns whole jobs to ranks by the longest-processing-time
rule, each rank renders its own jobs into its own outputs, and no collective
touches the data path.

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


def job_cost(width: int, height: int, spp: int, triangles: int = 1, spectral: int = 0, cache: bool = False) -> float:
    """Estimated device time of one render job, in arbitrary units: camera
    paths (width * height * spp) times a traversal factor that grows with the
    logarithm of the scene size, 1.25x for spectral jobs (lookup-table work in
    shading) and 1.5x for jobs with a radiance cache (inference and training
    per frame)."""
    import math
    paths = float(width) * float(height) * float(max(spp, 1))
    trav = 1.0 + 0.1 * math.log2(max(int(triangles), 2))
    return paths * trav * (1.25 if spectral else 1.0) * (1.5 if cache else 1.0)


def partition_jobs(costs, world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of jobs to `world` ranks: jobs
    in order of decreasing cost, each to the rank with the least assigned cost
    so far (ties to the lower rank; equal costs keep job order).  Returns, per
    rank, its job indices in ascending order.  The makespan is at most 4/3 of
    the optimum (Graham 1969)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda j: (-float(costs[j]), j))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for j in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(j)
        load[r] += float(costs[j])
    return [sorted(p) for p in parts]
