"""Progressive rendering: renders that continue one another (frame_offset =
previous offset + spp, same seed and image) reuse the per-pixel generator
states the previous render left instead of re-initialising them; the sums
must equal one render of all the samples."""
import numpy as np
import pytest

import scenes
from aperture_b200 import Scene, make_params


@pytest.mark.gpu
def test_continued_renders_equal_one_render():
    sc = Scene(scenes.box_scene())
    cam = scenes.box_camera(48, 40)
    one = np.zeros(48 * 40 * 3)
    sc.render(cam, make_params(spp=8, max_depth=8, frame_offset=5), accum=one)
    parts = np.zeros_like(one)
    for k in range(8):   # 1 spp each, frames 5..12
        sc.render(cam, make_params(spp=1, max_depth=8, frame_offset=5 + k), accum=parts)
    assert np.allclose(parts, one, rtol=1e-12, atol=1e-12)
    # a jump back re-initialises the states
    again = np.zeros_like(one)
    sc.render(cam, make_params(spp=8, max_depth=8, frame_offset=5), accum=again)
    assert np.allclose(again, one, rtol=1e-12, atol=1e-12)
