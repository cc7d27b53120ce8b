"""Four wavelengths per path (extension; the reference traces one hero
wavelength): the hero and its rotations by 105 nm, one estimate per rotation
set.  The XYZ image must converge to the single-wavelength image (both are
unbiased estimators of the same integral over wavelength) with less colour
noise per sample, including through dispersive glass (the path continues with
the hero alone) and the participating medium."""
import numpy as np
import pytest

import scenes
import spectral_tables
from aperture_b200 import Scene, make_params

pytestmark = pytest.mark.skipif(not spectral_tables.available(), reason="spectral tables not built")


def _pair(scene, cam, spp, mode, base):
    a, _ = scene.render(cam, make_params(spp=spp, max_depth=10, spectral=mode, frame_offset=base))
    b, _ = scene.render(cam, make_params(spp=spp, max_depth=10, spectral=mode, frame_offset=base + 100000))
    return a, b


def _check(scene, cam, spp, tol):
    a1, b1 = _pair(scene, cam, spp, 1, 0)
    a4, b4 = _pair(scene, cam, spp, 4, 500000)
    m1 = 0.5 * (a1 + b1)
    m4 = 0.5 * (a4 + b4)
    for c in range(3):   # channel means agree
        assert abs(m4[..., c].mean() - m1[..., c].mean()) <= tol * m1[..., c].mean(), (c, m4[..., c].mean(), m1[..., c].mean())
    # noise: spread between two independent renders of each mode
    n1 = np.mean((a1 - b1) ** 2)
    n4 = np.mean((a4 - b4) ** 2)
    return n1, n4


@pytest.mark.gpu
def test_four_wavelengths_converge_to_single_wavelength_box():
    sc = Scene(scenes.box_scene())
    sc.set_spectral(32)
    n1, n4 = _check(sc, scenes.box_camera(48, 48), 256, 0.02)
    assert n4 < 0.8 * n1, (n1, n4)


@pytest.mark.gpu
def test_four_wavelengths_dispersive_glass_and_medium():
    objs, vols, med = scenes.medium_box_scene(precision=16, grid=32, medium_grid=32)
    sc = Scene(objs, volumes=vols)
    sc.set_medium(**med)
    sc.set_spectral(32)
    _check(sc, scenes.box_camera(40, 40), 256, 0.04)
