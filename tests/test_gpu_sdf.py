"""Signed-distance objects on the GPU (an analytic torus and a torus sampled
on a 64^3 grid, float or half): ray queries against the oracle, bit for bit,
and per-path parity of whole paths that hit, refract through and shadow with
them.  The oracle's SDF intersector is pinned to the reference's
(tests/test_cpu_reference_pin.py::test_sdf_objects_match_reference)."""
import numpy as np
import pytest

import oracle
import scenes
from aperture_b200 import Scene, make_params, rng_tape

from test_gpu_trace import random_rays


def _u32(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [32, 16])
def test_sdf_ray_queries_equal_oracle(precision):
    objs, vols = scenes.sdf_box_scene(precision=precision)
    gs = Scene(objs, volumes=vols)
    osc = oracle.OracleScene(objs, volumes=vols)
    rays = random_rays(100_000, -0.6, 0.6, 31)
    g_obj, g_t = gs.trace_rays(rays)
    o_obj, o_t = osc.trace(rays)
    assert np.array_equal(g_obj, o_obj)
    hit = o_obj >= 0
    assert np.array_equal(_u32(g_t[hit]), _u32(o_t[hit]))
    n = len(objs)
    assert (o_obj == n - 2).sum() > 300 and (o_obj == n - 1).sum() > 300
    rays[:, 7] = np.random.default_rng(32).uniform(0.05, 1.2, len(rays))
    g_any, _ = gs.trace_rays(rays, any_hit=True)
    o_any, _ = osc.trace(rays, any_hit=True)
    assert np.array_equal(g_any >= 0, o_any >= 0)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [32, 16])
def test_sdf_paths_equal_oracle(precision):
    objs, vols = scenes.sdf_box_scene(precision=precision)
    cam = scenes.box_camera(40, 40)
    params = make_params(spp=2, max_depth=8)
    g = Scene(objs, volumes=vols).debug_paths(cam, params)
    tape = rng_tape(cam, params, 512)
    o, overflow = oracle.OracleScene(objs, volumes=vols).render_paths(cam, params, tape)
    assert overflow == 0
    for f in ("segments", "uniforms", "nee_rays", "nee_depth_mask"):
        assert np.array_equal(g[f], o[f]), f
    assert np.array_equal(g["hit_object"], o["hit_object"])
    err = np.abs(g["radiance"] - o["radiance"]) / np.maximum(np.abs(o["radiance"]), 1e-30)
    err[(g["radiance"] == 0) & (o["radiance"] == 0)] = 0
    assert err.max() <= 1e-5
    n = len(objs)
    assert np.isin(g["hit_object"], [n - 2, n - 1]).sum() > 100


@pytest.mark.gpu
def test_camera_inside_sdf():
    """A camera inside the glass torus starts its paths inside the medium
    (intersection::Overlap at the path start)."""
    objs, vols = scenes.sdf_box_scene()
    c = objs[len(objs) - 2]
    # a point on the torus core circle: unit-box (R, 0, 0) -> world
    cam = scenes.box_camera(8, 8)
    import math
    ang = math.radians(float(c["rotation_deg"]["y"]))
    # rotation Rz*(Ry*Rx) with x = 20 deg about X first: the core point lies in the
    # local XZ plane; take the local point (2*extent*R, 0, 0)
    ex = float(c["extent"]["x"])
    lx = 2.0 * ex * 0.3
    cam.position.x = float(c["center"]["x"]) + lx * math.cos(ang)
    cam.position.y = float(c["center"]["y"])
    cam.position.z = float(c["center"]["z"]) - lx * math.sin(ang)
    osc = oracle.OracleScene(objs, volumes=vols)
    assert osc.overlap(np.array([[cam.position.x, cam.position.y, cam.position.z]], np.float32))[0] == len(objs) - 2
    params = make_params(spp=1, max_depth=6)
    g = Scene(objs, volumes=vols).debug_paths(cam, params)
    o, _ = osc.render_paths(cam, params, rng_tape(cam, params, 512))
    assert np.array_equal(g["hit_object"], o["hit_object"])
    assert np.array_equal(g["segments"], o["segments"])
