"""Per-path parity of the wavefront path tracer with the CPU oracle.

The GPU renders with curand XORWOW seeded as core/random.cuh:31-39 and records
every path (ar_render_debug_paths).  The oracle (a restatement of
CalculateRadiance, core/render/render.cuh:460-999) replays the same paths from
a tape of the same random streams (ar_rng_tape).  Closest-hit object ids per
segment, segment counts, shadow-ray counts and the number of uniforms each path
consumed must be identical; radiance must agree to 1e-5 relative (FP32).
"""
import numpy as np
import pytest

import oracle
import scenes
from aperture_b200 import Scene, make_params, rng_tape

RTOL = 1e-5


def compare(objects, cam, params, per_path=512):
    g = Scene(objects).debug_paths(cam, params)
    tape = rng_tape(cam, params, per_path)
    o, overflow = oracle.OracleScene(objects).render_paths(cam, params, tape)
    assert overflow == 0, "tape too short"
    for f in ("segments", "uniforms", "nee_rays", "nee_depth_mask"):
        bad = np.nonzero(g[f] != o[f])[0]
        assert bad.size == 0, f"{f}: {bad.size} paths differ, first {bad[:5]} gpu {g[f][bad[:5]]} cpu {o[f][bad[:5]]}"
    assert np.array_equal(g["hit_object"], o["hit_object"]), "closest-hit ids differ"
    gr, orad = g["radiance"], o["radiance"]
    err = np.abs(gr - orad) / np.maximum(np.abs(orad), 1e-30)
    err[(gr == 0) & (orad == 0)] = 0
    assert err.max() <= RTOL, f"max rel radiance error {err.max()}"
    return g, o


@pytest.mark.gpu
def test_box_paths(box_objects):
    g, o = compare(box_objects, scenes.box_camera(48, 48), make_params(spp=2, max_depth=8))
    assert (g["segments"] > 2).mean() > 0.3
    assert g["nee_rays"].sum() > 0


@pytest.mark.gpu
def test_box_paths_no_sky_no_nee(box_objects):
    compare(box_objects, scenes.box_camera(32, 32), make_params(spp=2, max_depth=8, sky=0, use_nee=0))


@pytest.mark.gpu
def test_spheres_paths(small_spheres_objects):
    cam = scenes.spheres_camera(64, 36)
    cam.position.z = -45.0
    cam.position.y = 8.0
    compare(small_spheres_objects, cam, make_params(spp=2, max_depth=12))


@pytest.mark.gpu
def test_render_equals_path_mean(box_objects):
    cam = scenes.box_camera(40, 24)
    p = make_params(spp=3, max_depth=8, frame_offset=5)
    s = Scene(box_objects)
    rec = s.debug_paths(cam, p)
    img, stats = s.render(cam, p)
    mean = rec["radiance"].astype(np.float64).reshape(3, cam.height, cam.width, 3).sum(0) / 3.0
    # per-pixel FP64 sums are added with atomics in any order: equal to FP32 rounding
    np.testing.assert_allclose(img, mean.astype(np.float32), rtol=1e-6, atol=0)
    assert stats.paths == cam.width * cam.height * 3
    assert stats.extension_rays == rec["segments"].sum()


@pytest.mark.gpu
def test_many_samples_frame_jump(box_objects):
    """Samples 1..6 of each pixel start from the per-pixel state jumped ahead by
    2^32 draws per frame; the oracle replays curand_init(seed, pixel, f * 2^32)."""
    compare(box_objects, scenes.box_camera(16, 12), make_params(spp=7, max_depth=8, frame_offset=11))
