"""Parity on the benchmark's own scenes at full size.

Config 2 as benchmarked -- 800 icospheres x 1280 triangles, the ground quad and
16 emissive spheres (1,024,018 objects), a deep 8-wide BVH whose traversal
stacks spill from shared into global memory -- and config 3's scene -- the box
with a glass torus, a GGX torus sampled on a 256^3 half-precision grid and a
128^3 half-precision fBm medium -- checked against the oracle:

* 247,456 closest-hit queries (a 512 x 288 camera and 100,000 random rays in
  the scene's box): hit object and distance bit for bit;
* 200,000 any-hit segments: occlusion flags equal;
* 2,304 whole paths of config 2 at depth 12 and 2,304 paths of config 3 at
  depth 16 in single-wavelength spectral mode with the medium: hit object per
  segment, segments, uniforms, shadow rays equal, radiance within 1e-5.
"""
import numpy as np
import pytest

import oracle
import scenes
import spectral_tables
from aperture_b200 import Scene, make_params, rng_tape

from test_gpu_trace import camera_rays, random_rays

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def config2(config2_objects):
    return Scene(config2_objects), oracle.OracleScene(config2_objects)


def test_config2_closest_hits(config2):
    gs, osc = config2
    cam = scenes.spheres_camera(512, 288)
    rays = np.concatenate([camera_rays(cam, 11), random_rays(100_000, -100.0, 100.0, 12)])
    assert len(rays) == 247_456
    g_obj, g_t = gs.trace_rays(rays)
    o_obj, o_t = osc.trace(rays)
    bad = np.nonzero(g_obj != o_obj)[0]
    assert bad.size == 0, f"{bad.size} hit-id mismatches, first {bad[:5]}"
    hit = o_obj >= 0
    assert np.array_equal(g_t[hit].view(np.uint32), o_t[hit].view(np.uint32))
    assert hit.sum() > 50_000


def test_config2_any_hits(config2):
    gs, osc = config2
    rays = random_rays(200_000, -100.0, 100.0, 13)
    rays[:, 7] = np.random.default_rng(14).uniform(1.0, 120.0, len(rays))
    g_obj, _ = gs.trace_rays(rays, any_hit=True)
    o_obj, _ = osc.trace(rays, any_hit=True)
    assert np.array_equal(g_obj >= 0, o_obj >= 0)
    assert (o_obj >= 0).sum() > 5_000


def _compare_paths(g, o):
    for f in ("segments", "uniforms", "nee_rays", "nee_depth_mask"):
        bad = np.nonzero(g[f] != o[f])[0]
        assert bad.size == 0, f"{f}: {bad.size} paths differ, first {bad[:5]}"
    assert np.array_equal(g["hit_object"], o["hit_object"])
    err = np.abs(g["radiance"] - o["radiance"]) / np.maximum(np.abs(o["radiance"]), 1e-30)
    err[(g["radiance"] == 0) & (o["radiance"] == 0)] = 0
    assert err.max() <= 1e-5, err.max()


def test_config2_paths(config2):
    gs, osc = config2
    cam = scenes.spheres_camera(64, 36)
    params = make_params(spp=1, max_depth=12)
    g = gs.debug_paths(cam, params)
    o, overflow = osc.render_paths(cam, params, rng_tape(cam, params, 768))
    assert overflow == 0
    _compare_paths(g, o)
    assert len(g) == 2304 and g["nee_rays"].sum() > 300


@pytest.mark.skipif(not spectral_tables.available(), reason="spectral tables not built")
def test_config3_scene_paths():
    objs, vols, med = scenes.medium_box_scene(precision=16, grid=256, medium_grid=128)
    tables = spectral_tables.load()[0]
    cam = scenes.box_camera(64, 36)
    params = make_params(spp=1, max_depth=16, spectral=1)
    gs = Scene(objs, volumes=vols)
    gs.set_medium(**med)
    gs.set_spectral(64, tables)
    g = gs.debug_paths(cam, params)
    osc = oracle.OracleScene(objs, volumes=vols)
    osc.set_medium(**med)
    osc.set_spectral(tables, 64)
    o, overflow = osc.render_paths(cam, params, rng_tape(cam, params, 1024))
    assert overflow == 0
    _compare_paths(g, o)
    n = len(objs)
    assert (g["hit_object"] == -2).sum() > 100                 # medium collisions
    assert np.isin(g["hit_object"], [n - 2, n - 1]).sum() > 50  # the two tori
