"""Host-side logic that needs no GPU: the XORWOW frame jump table, and the
multi-GPU split of a render run as two gloo ranks on CPU tensors with the
oracle standing in for each rank's GPU render.
"""
import os
import shutil
import socket
import subprocess

import numpy as np
import pytest

import sharding

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_xorwow_frame_jump_table(tmp_path):
    """A^(2^16) against explicit steps, A^(2^32) against 2^16 jumps of 2^16,
    A^(2^33) and A^(2^67) (the subsequence jump of the per-pixel
    initialisation) against two jumps of half the distance."""
    exe = tmp_path / "xorwow_jump_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe),
                    os.path.join(HERE, "native", "xorwow_jump_check.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "OK", out.stdout


def test_rank_frame_offsets_are_disjoint():
    spp = 5
    frames = [set(range(sharding.rank_frame_offset(r, spp), sharding.rank_frame_offset(r, spp) + spp))
              for r in range(8)]
    assert set().union(*frames) == set(range(8 * spp))
    assert sum(len(f) for f in frames) == 8 * spp
    with pytest.raises(ValueError):
        sharding.rank_frame_offset(0, 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, spp, out_path):
    import sys
    sys.path[:0] = [os.path.join(os.path.dirname(HERE), "aperturerendererv3-optix-geometry_b200"),
                    os.path.join(os.path.dirname(HERE), "oracle")]
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    import oracle
    import scenes
    from aperture_b200 import make_params
    from sharding import job_totals, rank_frame_offset, reduce_accumulators

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        cam = scenes.box_camera(12, 10)
        p = make_params(spp=spp, max_depth=6, frame_offset=rank_frame_offset(rank, spp))
        acc, e, s = oracle.OracleScene(scenes.box_scene()).render_image(cam, p, threads=1)
        accum = torch.from_numpy(acc.reshape(-1).copy())
        reduce_accumulators(accum, dist)
        t, (rays,) = job_totals(10.0 + rank, [e + s], dist, torch.device("cpu"))
        if rank == 0:
            np.save(out_path, accum.numpy())
            with open(out_path + ".txt", "w") as f:
                f.write(f"{t} {rays}\n")
    finally:
        dist.destroy_process_group()


def test_two_rank_render_sums_to_single_render(tmp_path):
    """Two ranks with frame offsets 0 and spp, reduced, equal one render of 2*spp."""
    import torch.multiprocessing as mp

    import oracle
    import scenes
    from aperture_b200 import make_params

    spp, world = 2, 2
    out = str(tmp_path / "acc.npy")
    mp.start_processes(_rank_main, args=(world, _free_port(), spp, out), nprocs=world, start_method="spawn",
                       join=True)
    got = np.load(out)
    cam = scenes.box_camera(12, 10)
    acc, e, s = oracle.OracleScene(scenes.box_scene()).render_image(cam, make_params(spp=world * spp, max_depth=6),
                                                                    threads=1)
    np.testing.assert_allclose(got, acc.reshape(-1), rtol=1e-12, atol=1e-12)
    t, rays = open(out + ".txt").read().split()
    assert float(t) == 11.0                    # slowest rank
    assert float(rays) == float(e + s)         # queries add over ranks


def test_partition_jobs_is_lpt():
    from sharding import partition_jobs
    costs = [7, 5, 4, 4, 3, 3, 2, 1]
    parts = partition_jobs(costs, 3)
    assert sorted(j for p in parts for j in p) == list(range(len(costs)))
    loads = [sum(costs[j] for j in p) for p in parts]
    assert max(loads) == 10 and min(loads) == 9          # LPT on this instance: 10, 10, 9 or better
    assert partition_jobs(costs, 1) == [list(range(len(costs)))]
    assert partition_jobs([], 4) == [[], [], [], []]
    # Graham's bound on random instances, against the trivial lower bound
    rng = np.random.default_rng(3)
    for _ in range(50):
        c = rng.exponential(1.0, int(rng.integers(1, 40))).tolist()
        w = int(rng.integers(1, 9))
        p = partition_jobs(c, w)
        mk = max(sum(c[j] for j in q) for q in p)
        assert mk <= (4.0 / 3.0) * max(sum(c) / w, max(c)) + 1e-9


def _batch_rank_main(rank, world, port, out_dir):
    import os
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    import oracle
    import scenes
    from aperture_b200 import make_params
    from sharding import job_cost, job_totals, partition_jobs

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        jobs = _batch_jobs()
        parts = partition_jobs([job_cost(w, h, spp) for (w, h, spp, _) in jobs], world)
        rays = 0
        for j in parts[rank]:
            w, h, spp, seed = jobs[j]
            acc, e, s = oracle.OracleScene(scenes.box_scene(seed=seed)).render_image(
                scenes.box_camera(w, h), make_params(spp=spp, max_depth=5), threads=1)
            rays += e + s
            np.save(os.path.join(out_dir, f"job{j}_rank{rank}.npy"), acc)
        t, (total,) = job_totals(float(len(parts[rank])), [rays], dist, torch.device("cpu"))
        if rank == 0:
            with open(os.path.join(out_dir, "totals.txt"), "w") as f:
                f.write(f"{t} {total}\n")
    finally:
        dist.destroy_process_group()


def _batch_jobs():
    return [(8, 6, 2, 0xA11CE + 11), (5, 5, 4, 0xA11CE + 12), (12, 4, 1, 0xA11CE + 13), (6, 6, 3, 0xA11CE + 14),
            (4, 4, 1, 0xA11CE + 15)]


def test_two_rank_batch_partition_renders_every_job_once(tmp_path):
    """Jobs split by partition_jobs over two gloo ranks: every job rendered by
    exactly one rank, its image equal to a single-process render, no
    collective on the data path (only the job-time max and ray count sum)."""
    import os

    import torch.multiprocessing as mp

    import oracle
    import scenes
    from aperture_b200 import make_params

    world = 2
    mp.start_processes(_batch_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    jobs = _batch_jobs()
    files = sorted(os.listdir(tmp_path))
    for j, (w, h, spp, seed) in enumerate(jobs):
        mine = [f for f in files if f.startswith(f"job{j}_")]
        assert len(mine) == 1, (j, mine)
        got = np.load(os.path.join(tmp_path, mine[0]))
        acc, _, _ = oracle.OracleScene(scenes.box_scene(seed=seed)).render_image(
            scenes.box_camera(w, h), make_params(spp=spp, max_depth=5), threads=1)
        np.testing.assert_array_equal(got, acc)
    ranks = {f.split("_rank")[1].split(".")[0] for f in files if f.startswith("job")}
    assert ranks == {"0", "1"}
