"""Path guiding on the GPU (interactive frames): probes are created and
filled from the frames' paths, their mip chains are averages and their
density (oracle/guiding_oracle.py) is normalised, and guided frames, whose
directions partly come from the probes with the mixture pdf in the weights
and in MIS, converge to the plain tracer's image (no bias)."""
import math

import numpy as np
import pytest

import guiding_oracle as G
import scenes
from aperture_b200 import PathGuide, Scene, make_params


@pytest.mark.gpu
def test_guided_frames_fill_probes_and_converge():
    import torch
    sc = Scene(scenes.box_scene())
    cam = scenes.box_camera(64, 64)
    ref, _ = sc.render(cam, make_params(spp=2048, max_depth=8, frame_offset=900000))
    guide = PathGuide(sc)
    n = 64 * 64 * 3
    acc = torch.zeros(n, dtype=torch.float64, device="cuda")
    frames = 384
    for f in range(frames):
        guide.render_frame(cam, make_params(spp=1, max_depth=8, frame_offset=f), None, acc.data_ptr())
    torch.cuda.synchronize()
    st = guide.stats()
    assert st.frames == frames and st.probes > 200 and st.samples > 1000
    assert abs(st.alpha - 0.5) < 1e-6
    img = (acc / frames).cpu().numpy().reshape(64, 64, 3)
    for c in range(3):
        assert abs(img[..., c].mean() - ref[..., c].mean()) < 0.02 * ref[..., c].mean(), c
    plain, _ = sc.render(cam, make_params(spp=frames, max_depth=8, frame_offset=500000))
    rel_g = ((img - ref) ** 2 / (ref ** 2 + 1e-2)).mean()
    rel_p = ((plain - ref) ** 2 / (ref ** 2 + 1e-2)).mean()
    print("relMSE guided", rel_g, "plain", rel_p)
    assert rel_g < 1.5 * rel_p
    # probes: leaves clamped, mips are averages, density normalised
    # texel centres: the density is constant per texel and texels have equal area
    c = (np.arange(8) + 0.5) / 8
    cu, cv = np.meshgrid(c, c)
    w = G.uv_to_dir(cu.reshape(-1), cv.reshape(-1))
    for idx in (0, st.probes // 2, st.probes - 1):
        t = guide.probe(int(idx))[:, :3].astype(np.float64)
        assert np.all(t[:64] >= 1e-5 * (1 - 1e-6))
        assert np.allclose(t[84], t[:64].mean(0), rtol=1e-4)
        assert np.allclose(t[80:84].mean(0), t[84], rtol=1e-4)
        q = np.array([0.3, 0.4, 0.3])
        assert abs(np.sum(G.pdf(t[:85], w, q)) * 4 * math.pi / 64 - 1.0) < 1e-4


@pytest.mark.gpu
def test_device_probe_math_matches_reference():
    """csrc/guiding.cuh on the GPU (ar_guide_probe_eval) against the
    reference's Octahedron and grid run on the host
    (tests/golden/reference_guiding.npz, 8,000 queries over 8 probes): the
    (voxel, face) key of every point and direction equal -- the face in the
    reference's numbering --, hemisphere sample directions within 2e-6,
    sample pdfs and pdfs of given directions within 2e-5 relative (the two
    codes write the equal-area map and the mirror with different float
    operations)."""
    import os

    from aperture_b200 import guide_probe_eval
    fx = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_guiding.npz"))
    d, p, e, k = guide_probe_eval(fx["texels"], fx["probe_of"], fx["normal"], fx["query"], fx["u5"], fx["eval_dir"],
                                  fx["pos"])
    m = (1 << 19) - 1
    vox = np.stack([(k >> s) & m for s in (0, 19, 38)], 1).astype(np.int64)
    vox = np.where(vox >= (1 << 18), vox - (1 << 19), vox)
    face = (k >> 57).astype(np.int64)
    ref = fx["voxel"].astype(np.int64)
    assert np.array_equal(vox, ref[:, :3])
    assert np.array_equal(face, ref[:, 3])
    assert np.abs(d - fx["dir"]).max() < 2e-6
    assert np.max(np.abs(p - fx["pdf"]) / fx["pdf"]) < 2e-5
    ep = fx["epdf"]
    assert np.array_equal(e == 0, ep == 0)
    nz = ep > 0
    assert np.max(np.abs(e[nz] - ep[nz]) / ep[nz]) < 2e-5
