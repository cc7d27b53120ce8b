"""Extensions beyond the reference, checked for unbiasedness on the CPU oracle.

Triangle-light NEE (ar_render_params.tri_light_nee): the reference's NEE
samples only cube and sphere lights (nee.cuh:362-369), so a scene lit by an
emissive triangle quad (config 1 as specified) converges only through BSDF
sampling.  With the extension, NEE also samples the triangles (uniform area
density, MIS with BSDF hits): the converged image must be the same and its
noise lower."""
import numpy as np

import oracle
import scenes
from aperture_b200 import make_params


def _render(osc, cam, spp, tri, frame):
    acc, _, _ = osc.render_image(cam, make_params(spp=spp, max_depth=8, frame_offset=frame, tri_light_nee=tri))
    return acc / spp


def test_triangle_light_nee_is_unbiased_and_less_noisy():
    objs = scenes.box_scene(light_as="triangles")
    osc = oracle.OracleScene(objs)
    cam = scenes.box_camera(24, 24)
    a = np.stack([_render(osc, cam, 16, 0, 1000 * k) for k in range(4)])
    b = np.stack([_render(osc, cam, 16, 1, 1000 * k + 500) for k in range(4)])
    ma, mb = a.mean(0).mean(), b.mean(0).mean()
    # image means agree within the BSDF-only estimate's noise
    assert abs(ma - mb) / ma < 0.05, (ma, mb)
    # per-pixel spread across independent runs: NEE on triangles lowers it
    assert b.std(0).mean() < 0.7 * a.std(0).mean()
