"""ar_trace_rays_static -- ray queries for callers that cannot allocate.

Some callers of this library may not call cudaMalloc when they query rays (a
host with a fixed device-memory budget, a real-time thread, a process where
another thread may be capturing a CUDA graph).  ar_trace_rays_static keeps its
scratch in a file-scope device array instead of a library allocation.  These
tests call it through the C ABI with caller-owned device buffers, twice in a
row (the second call reuses the shared scratch left by the first), and require
the same hit ids and distances, bit for bit, as the allocating ar_trace_rays.
The file runs last so that a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

import scenes
from aperture_b200 import Scene

from test_gpu_trace import camera_rays, random_rays


def _static_twice(scene, rays, any_hit):
    import torch
    dev = torch.device("cuda", 0)
    r = torch.from_numpy(np.ascontiguousarray(rays, np.float32)).to(dev)
    n = rays.shape[0]
    results = []
    for _ in range(2):
        obj = torch.full((n,), -7, dtype=torch.int32, device=dev)
        t = torch.full((n,), -7.0, dtype=torch.float32, device=dev)
        scene.trace_rays_static(r.data_ptr(), n, any_hit, obj.data_ptr(), t.data_ptr(),
                                torch.cuda.current_stream(dev).cuda_stream)
        torch.cuda.synchronize(dev)
        results.append((obj.cpu().numpy(), t.cpu().numpy()))
    return results


@pytest.mark.gpu
@pytest.mark.parametrize("any_hit", [False, True])
def test_static_matches_allocating_box(box_objects, any_hit):
    scene = Scene(box_objects)
    rays = random_rays(150_000, -0.7, 0.7, 21)
    if any_hit:
        rays[:, 7] = np.random.default_rng(22).uniform(0.05, 1.5, len(rays))
    ref_obj, ref_t = scene.trace_rays(rays, any_hit=any_hit)
    for obj, t in _static_twice(scene, rays, any_hit):
        if any_hit:
            assert np.array_equal(obj >= 0, ref_obj >= 0)
        else:
            assert np.array_equal(obj, ref_obj)
            hit = ref_obj >= 0
            assert np.array_equal(t[hit].view(np.uint32), ref_t[hit].view(np.uint32))


@pytest.mark.gpu
def test_static_matches_allocating_spheres(small_spheres_objects):
    scene = Scene(small_spheres_objects)
    cam = scenes.spheres_camera(96, 54)
    cam.position.z = -45.0
    rays = np.concatenate([camera_rays(cam), random_rays(60_000, -25, 25, 23)])
    ref_obj, ref_t = scene.trace_rays(rays)
    for obj, t in _static_twice(scene, rays, False):
        assert np.array_equal(obj, ref_obj)
        assert np.array_equal(t.view(np.uint32), ref_t.view(np.uint32))


@pytest.mark.gpu
def test_static_rejects_unaligned_rays(box_objects):
    import torch
    scene = Scene(box_objects)
    buf = torch.zeros(8 * 4 + 1, dtype=torch.float32, device="cuda")
    out = torch.zeros(4, dtype=torch.int32, device="cuda")
    from aperture_b200 import ArError
    with pytest.raises(ArError):
        scene.trace_rays_static(buf.data_ptr() + 4, 4, False, out.data_ptr(), None)
