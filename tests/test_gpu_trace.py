"""Ray-query parity of the sm_100a traversal with the CPU oracle.

The oracle restates TraverseBVH + IntersectTriangleObject / IntersectAABBObject /
IntersectSphereObject (core/render/intersection.cuh:15-370, core/object/*.cuh);
hit object indices and distances must agree bit for bit (ties in t go to the
lowest object index in both)."""
import numpy as np
import pytest

import oracle
import scenes
from aperture_b200 import Scene


def random_rays(n, lo, hi, seed, tmin=1e-4):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmin
    r[:, 4:7] = d
    r[:, 7] = np.inf
    return r


def camera_rays(cam, jitter_seed=0):
    rng = np.random.default_rng(jitter_seed)
    w, h = cam.width, cam.height
    jit = rng.random((w * h, 2)).astype(np.float32)
    return np.stack([oracle.camera_ray(cam, k % w, k // w, jit[k, 0], jit[k, 1]) for k in range(w * h)])


def check(objects, rays, any_hit=False):
    gs = Scene(objects)
    os_ = oracle.OracleScene(objects)
    g_obj, g_t = gs.trace_rays(rays, any_hit=any_hit)
    o_obj, o_t = os_.trace(rays, any_hit=any_hit)
    if any_hit:
        assert np.array_equal(g_obj >= 0, o_obj >= 0), f"{(g_obj >= 0) != (o_obj >= 0)}"
    else:
        bad = np.nonzero(g_obj != o_obj)[0]
        assert bad.size == 0, f"{bad.size} hit-id mismatches, first {bad[:5]} gpu {g_obj[bad[:5]]} cpu {o_obj[bad[:5]]}"
        hit = o_obj >= 0
        assert np.array_equal(g_t[hit].view(np.uint32), o_t[hit].view(np.uint32)), "hit distances differ"
    return g_obj


@pytest.mark.gpu
def test_box_scene_random_rays(box_objects):
    rays = random_rays(200_000, -0.7, 0.7, 1)
    obj = check(box_objects, rays)
    assert (obj >= 0).mean() > 0.3


@pytest.mark.gpu
def test_box_scene_any_hit(box_objects):
    rays = random_rays(100_000, -0.7, 0.7, 2)
    rays[:, 7] = np.random.default_rng(3).uniform(0.05, 1.5, len(rays))
    check(box_objects, rays, any_hit=True)


@pytest.mark.gpu
def test_box_scene_camera_rays(box_objects):
    check(box_objects, camera_rays(scenes.box_camera(128, 128)))


@pytest.mark.gpu
def test_spheres_scene_rays(small_spheres_objects):
    cam = scenes.spheres_camera(160, 90)
    cam.position.z = -45.0
    cam.position.y = 8.0
    check(small_spheres_objects, camera_rays(cam))
    check(small_spheres_objects, random_rays(100_000, -25, 25, 4))
    rays = random_rays(100_000, -25, 25, 5)
    rays[:, 7] = 10.0
    check(small_spheres_objects, rays, any_hit=True)


@pytest.mark.gpu
def test_empty_and_degenerate(box_objects):
    # empty scene: everything misses
    empty = Scene(box_objects[:0])
    obj, t = empty.trace_rays(random_rays(1000, -1, 1, 6))
    assert (obj == -1).all()
    # zero direction components, tmin > tmax, rays starting on a wall
    r = random_rays(64, -0.4, 0.4, 7)
    r[:16, 4:7] = [0.0, -1.0, 0.0]
    r[16:32, 4:7] = [0.0, 0.0, -1.0]
    r[32:40, 3] = 5.0
    r[40:48, 0:3] = [0.0, -0.5, 0.0]
    check(box_objects, r)
