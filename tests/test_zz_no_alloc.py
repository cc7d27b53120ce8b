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


def _static_once(scene, rays, any_hit, with_t):
    import torch
    dev = torch.device("cuda", 0)
    r = torch.from_numpy(np.ascontiguousarray(rays, np.float32)).to(dev)
    n = rays.shape[0]
    obj = torch.full((n,), -7, dtype=torch.int32, device=dev)
    t = torch.full((n,), -7.0, dtype=torch.float32, device=dev) if with_t else None
    scene.trace_rays_static(r.data_ptr(), n, any_hit, obj.data_ptr(), t.data_ptr() if with_t else None,
                            torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize(dev)
    return obj.cpu().numpy(), (t.cpu().numpy() if with_t else None)


@pytest.mark.gpu
@pytest.mark.parametrize("any_hit", [False, True])
def test_static_matches_allocating_sdf(any_hit):
    """Scenes with signed-distance objects run the SDF instantiations of the
    static kernel (sphere tracing after the BVH walk); a second call passes no
    distance buffer."""
    objs, vols = scenes.sdf_box_scene(precision=16)
    scene = Scene(objs, volumes=vols)
    rays = random_rays(80_000, -0.6, 0.6, 24)
    if any_hit:
        rays[:, 7] = np.random.default_rng(25).uniform(0.05, 1.2, len(rays))
    ref_obj, ref_t = scene.trace_rays(rays, any_hit=any_hit)
    n = len(objs)
    assert np.isin(ref_obj, [n - 2, n - 1]).sum() > 300 or any_hit
    obj, t = _static_once(scene, rays, any_hit, True)
    obj2, _ = _static_once(scene, rays, any_hit, False)
    if any_hit:
        assert np.array_equal(obj >= 0, ref_obj >= 0)
        assert np.array_equal(obj2 >= 0, ref_obj >= 0)
    else:
        assert np.array_equal(obj, ref_obj)
        assert np.array_equal(obj2, ref_obj)
        hit = ref_obj >= 0
        assert np.array_equal(t[hit].view(np.uint32), ref_t[hit].view(np.uint32))
