"""Participating medium on the GPU (extension: delta tracking in the extension
stage, Henyey-Greenstein scattering with NEE, ratio-tracking transmittance on
shadow rays): whole paths against the oracle's restatement -- the same
collisions (hit_object -2), vertex counts and uniforms, radiance within 1e-5
-- with the grid in float and half, and the converged image of a homogeneous
absorbing slab against Beer-Lambert."""
import numpy as np
import pytest

import oracle
import scenes
import spectral_tables
from aperture_b200 import ArError, Scene, make_params, rng_tape

from test_cpu_medium import beer_lambert_scene, expected_beer_lambert


def _compare(g, o, min_medium=100):
    for f in ("segments", "uniforms", "nee_rays", "nee_depth_mask"):
        assert np.array_equal(g[f], o[f]), f
    assert np.array_equal(g["hit_object"], o["hit_object"])
    err = np.abs(g["radiance"] - o["radiance"]) / np.maximum(np.abs(o["radiance"]), 1e-30)
    err[(g["radiance"] == 0) & (o["radiance"] == 0)] = 0
    assert err.max() <= 1e-5
    assert (g["hit_object"] == -2).sum() > min_medium


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [32, 16])
def test_medium_paths_equal_oracle(precision):
    objs, vols, med = scenes.medium_box_scene(precision=precision, grid=32, medium_grid=32)
    cam = scenes.box_camera(40, 40)
    params = make_params(spp=2, max_depth=10)
    gs = Scene(objs, volumes=vols)
    gs.set_medium(**med)
    g = gs.debug_paths(cam, params)
    tape = rng_tape(cam, params, 768)
    osc = oracle.OracleScene(objs, volumes=vols)
    osc.set_medium(**med)
    o, overflow = osc.render_paths(cam, params, tape)
    assert overflow == 0
    _compare(g, o)


@pytest.mark.gpu
@pytest.mark.skipif(not spectral_tables.available(), reason="spectral tables not built")
def test_medium_spectral_paths_equal_oracle():
    objs, vols, med = scenes.medium_box_scene(precision=16, grid=32, medium_grid=32)
    tables = spectral_tables.load()[0]
    cam = scenes.box_camera(24, 24)
    params = make_params(spp=2, max_depth=10, spectral=1)
    gs = Scene(objs, volumes=vols)
    gs.set_medium(**med)
    gs.set_spectral(16, tables)
    g = gs.debug_paths(cam, params)
    tape = rng_tape(cam, params, 768)
    osc = oracle.OracleScene(objs, volumes=vols)
    osc.set_medium(**med)
    osc.set_spectral(tables, 16)
    o, overflow = osc.render_paths(cam, params, tape)
    assert overflow == 0
    _compare(g, o, min_medium=30)


@pytest.mark.gpu
def test_medium_beer_lambert_image():
    objs, medium, cam = beer_lambert_scene()
    gs = Scene(objs)
    gs.set_medium(**medium)
    spp = 512
    img, _ = gs.render(cam, make_params(spp=spp, max_depth=4, sky=0))
    want = expected_beer_lambert(cam)
    got = img[..., 0]
    assert abs(got.mean() - want.mean()) < 0.01 * want.mean(), (got.mean(), want.mean())
    # removing the medium gives the unattenuated light
    gs.set_medium(None)
    img, _ = gs.render(cam, make_params(spp=4, max_depth=4, sky=0))
    assert np.allclose(img, 1.0, rtol=1e-6)


@pytest.mark.gpu
def test_set_medium_rejects_bad_descriptions():
    objs, medium, _ = beer_lambert_scene()
    gs = Scene(objs)
    for key, bad in (("g", 1.0), ("sigma_t_max", -1.0), ("albedo", (1.5, 0.0, 0.0)),
                     ("bounds_max", (-5.0, 4.0, 0.5))):
        m = dict(medium)
        m[key] = bad
        with pytest.raises(ArError):
            gs.set_medium(**m)
    m = dict(medium)
    m["density"] = -np.ones((2, 2, 2), np.float32)
    with pytest.raises(ArError):
        gs.set_medium(**m)
