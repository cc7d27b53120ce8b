"""GPU parity of the extensions beyond the reference (same per-path contract
as tests/test_gpu_paths.py): triangle-light NEE on config 1 with its emissive
quad as two triangles."""
import numpy as np
import pytest

import oracle
import scenes
from aperture_b200 import Scene, make_params, rng_tape


def _compare(objects, cam, params, per_path=600):
    g = Scene(objects).debug_paths(cam, params)
    o, overflow = oracle.OracleScene(objects).render_paths(cam, params, rng_tape(cam, params, per_path))
    assert overflow == 0
    for f in ("segments", "uniforms", "nee_rays", "nee_depth_mask"):
        assert np.array_equal(g[f], o[f]), f
    assert np.array_equal(g["hit_object"], o["hit_object"])
    err = np.abs(g["radiance"] - o["radiance"]) / np.maximum(np.abs(o["radiance"]), 1e-30)
    err[(g["radiance"] == 0) & (o["radiance"] == 0)] = 0
    assert err.max() <= 1e-5, err.max()
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("spectral", [0])
def test_triangle_light_nee_paths(spectral):
    objs = scenes.box_scene(light_as="triangles")
    g = _compare(objs, scenes.box_camera(40, 40), make_params(spp=2, max_depth=8, tri_light_nee=1))
    assert g["nee_rays"].sum() > 1000
