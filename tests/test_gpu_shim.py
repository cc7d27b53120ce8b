"""The C++ shim of the reference's API on the GPU: a caller written against
SceneRenderer / Camera (tests/native/shim_render.cpp) gets the same image as
the C ABI gives for the same objects, its BMP holds the tone-mapped image,
and three interactive frames give the running mean of frames 0..2."""
import numpy as np
import pytest

import shim_build
from aperture_b200 import OBJECT_DTYPE, Scene, make_camera, make_params, tonemap

W, H, SPP = 48, 32, 4


@pytest.mark.gpu
@pytest.mark.skipif(not shim_build.available(), reason="needs g++ and CUDA headers")
def test_shim_matches_c_abi(tmp_path):
    out = shim_build.run(str(tmp_path), W, H, SPP)
    assert "ERROR" not in out, out
    objs = np.fromfile(tmp_path / "objects.bin", OBJECT_DTYPE)
    scene = Scene(objs)
    cam = make_camera((0.0, 0.0, 1.9), (0.0, 0.0, -1.0), 60.0, W, H)
    ref, _ = scene.render(cam, make_params(spp=SPP, max_depth=1000, rr_depth=3))
    img = np.fromfile(tmp_path / "image.f32", np.float32).reshape(H, W, 3)
    assert img.max() > 0
    np.testing.assert_allclose(img, ref, rtol=1e-6, atol=1e-7)

    w, h, rgba = shim_build.read_bmp(str(tmp_path / "shot.bmp"))
    assert (w, h) == (W, H)
    packed = tonemap(img.reshape(-1, 3), 2, 1.3).reshape(H, W)
    want = np.stack([(packed >> 16) & 255, (packed >> 8) & 255, packed & 255], -1).astype(np.int32)
    assert np.abs(rgba[..., :3].astype(np.int32) - want).max() <= 1
    _, _, custom = shim_build.read_bmp(str(tmp_path / "custom.bmp"))
    c = img / (np.float32(1.0) + img)
    want_c = (np.float32(255.0) * np.clip(c, 0, 1)).astype(np.int32)
    assert np.abs(custom[..., :3].astype(np.int32) - want_c).max() <= 1

    frames = np.fromfile(tmp_path / "frames.f32", np.float32)
    hdr = frames[:W * H * 3].reshape(H, W, 3)
    ldr = frames[W * H * 3:].view(np.uint32)
    three, _ = scene.render(cam, make_params(spp=3, max_depth=1000, rr_depth=3))
    np.testing.assert_allclose(hdr, three, rtol=1e-6, atol=1e-7)
    assert np.array_equal(ldr, tonemap(hdr.reshape(-1, 3), 2, 1.0))
