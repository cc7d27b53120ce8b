"""Batched jobs (ar_render_batch): uneven resolutions, spp, scenes (a shared
scene among them), RGB and spectral jobs in one CUDA graph replayed until all
are done.  Each job's image equals a separate ar_render of the same job:
paths draw the same random streams whatever pool they share (per-pixel FP64
sums, added in another order: equal to FP32 rounding)."""
import numpy as np
import pytest

import scenes
import spectral_tables
from aperture_b200 import Scene, make_params, render_batch


@pytest.mark.gpu
def test_batch_equals_separate_renders(box_objects, small_spheres_objects):
    import torch
    box = Scene(box_objects)
    sph = Scene(small_spheres_objects)
    spectral = spectral_tables.available()
    if spectral:
        box.set_spectral(32)
    cam_s = scenes.spheres_camera(72, 40)
    cam_s.position.z = -45.0
    specs = [
        (box, scenes.box_camera(64, 48), make_params(spp=4, max_depth=8)),
        (box, scenes.box_camera(33, 17), make_params(spp=16, max_depth=6, frame_offset=3)),
        (sph, cam_s, make_params(spp=2, max_depth=10)),
        (box, scenes.box_camera(20, 20), make_params(spp=8, max_depth=8, spectral=1 if spectral else 0)),
        (sph, scenes.spheres_camera(16, 9), make_params(spp=1, max_depth=12, use_nee=0)),
    ]
    outs, jobs = [], []
    for scene, cam, p in specs:
        o = torch.zeros(cam.width * cam.height * 3, dtype=torch.float32, device="cuda")
        outs.append(o)
        jobs.append((scene, cam, p, o.data_ptr(), None))
    st = render_batch(jobs, iterations_per_graph=6, path_budget=1 << 16)
    torch.cuda.synchronize()
    # one graph launch; the device-side loop ran its passes
    assert st.graph_launches == 1 and st.loop_passes >= 1 and st.graph_nodes > 5 * 10 * 6
    assert st.paths == sum(c.width * c.height * p.spp for _, c, p in specs)
    for (scene, cam, p), o in zip(specs, outs):
        ref, _ = scene.render(cam, p)
        np.testing.assert_allclose(o.cpu().numpy().reshape(cam.height, cam.width, 3), ref, rtol=1e-6, atol=1e-7)


@pytest.mark.gpu
def test_batch_rejects_bad_jobs(box_objects):
    from aperture_b200 import ArError
    s = Scene(box_objects)
    with pytest.raises(ArError):
        render_batch([(s, scenes.box_camera(8, 8), make_params(spp=1), None, None)])


@pytest.mark.gpu
def test_batch_autotune(box_objects, small_spheres_objects):
    """The autotuner times its probe on scratch outputs (the jobs' buffers keep
    their contents) over graph lengths x path budgets and then the per-job
    kernel grids, returns one of its candidates, the fastest, and the next
    default render_batch of the same batch shape uses it (grids included) with
    unchanged results."""
    import torch
    from aperture_b200 import autotune_batch
    box = Scene(box_objects)
    sph = Scene(small_spheres_objects)
    cam_s = scenes.spheres_camera(48, 32)
    cam_s.position.z = -45.0
    specs = [(box, scenes.box_camera(40, 30), make_params(spp=8, max_depth=8)),
             (sph, cam_s, make_params(spp=4, max_depth=10)),
             (box, scenes.box_camera(17, 23), make_params(spp=16, max_depth=6, frame_offset=9))]
    outs, jobs = [], []
    for scene, cam, p in specs:
        o = torch.full((cam.width * cam.height * 3,), -1.0, dtype=torch.float32, device="cuda")
        outs.append(o)
        jobs.append((scene, cam, p, o.data_ptr(), None))
    t = autotune_batch(jobs, probe_spp=2)
    torch.cuda.synchronize()
    assert all(bool((o == -1.0).all()) for o in outs)
    assert t.candidates == 24
    assert t.iterations_per_graph in (4, 8, 16, 32)
    assert t.path_budget in (1 << 20, 1 << 21, 1 << 22, 1 << 23)
    assert t.trace_blocks_per_sm in (0, 4, 2)
    assert t.shade_blocks_per_sm in (4, 2, 1)
    assert 0 < t.best_ms <= t.default_ms * 1.0001
    st = render_batch(jobs)
    torch.cuda.synchronize()
    assert st.iterations_per_graph == t.iterations_per_graph + (t.iterations_per_graph & 1)
    for (scene, cam, p), o in zip(specs, outs):
        ref, _ = scene.render(cam, p)
        np.testing.assert_allclose(o.cpu().numpy().reshape(cam.height, cam.width, 3), ref, rtol=1e-6, atol=1e-7)
