"""The C++ shim of the reference's API (include/aperture_b200_renderer.hpp)
without a GPU: a caller written against SceneObject / Material /
SceneRenderer / Camera compiles and runs, every failing call prints the
library's message (the reference prints its CUDA errors and carries on), the
BMP writer produces a valid file, the objects reach the C ABI with the
factories' values, and the host tone curves (Gamma, ACES) match the
reference's quantised output."""
import ctypes

import numpy as np
import pytest

import shim_build
from aperture_b200 import OBJECT_DTYPE, load_library


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


pytestmark = pytest.mark.skipif(not shim_build.available(), reason="needs g++ and CUDA headers")


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device behaviour")
def test_shim_without_device(tmp_path):
    out = shim_build.run(str(tmp_path), 20, 12, 2)
    assert "aperture_b200 ERROR: no CUDA device available" in out and "shim done" in out
    img = np.fromfile(tmp_path / "image.f32", np.float32)
    assert img.shape == (20 * 12 * 3,) and not img.any()
    w, h, rgba = shim_build.read_bmp(str(tmp_path / "shot.bmp"))
    assert (w, h) == (20, 12)
    assert np.all(rgba[..., 3] == 255) and np.all(rgba[..., :3] == 0)


def test_shim_objects_reach_the_abi(tmp_path):
    shim_build.run(str(tmp_path), 8, 8, 1)
    objs = np.fromfile(tmp_path / "objects.bin", OBJECT_DTYPE)
    assert len(objs) == 13
    assert np.all(objs["type"][:10] == 3)
    cube, sphere, light = objs[10], objs[11], objs[12]
    assert cube["type"] == 0 and cube["material"]["shading_model"] == 3
    assert cube["rotation_deg"]["y"] == np.float32(25.0)
    assert cube["material"]["roughness"] == np.float32(0.3) and cube["material"]["metallic"] == 1.0
    assert sphere["type"] == 1 and sphere["material"]["shading_model"] == 2
    assert sphere["material"]["ior"] == np.float32(1.5) and sphere["material"]["sigma_a"] == np.float32(0.5)
    assert light["material"]["shading_model"] == 1 and light["material"]["emissive"]["x"] == 17.0
    assert np.all(objs["visible"] == 1)


@pytest.mark.parametrize("tone", [1, 2])
def test_host_tone_curve_matches_reference(tone):
    """ar_tone_curve (behind the shim's Gamma / ACES) quantised like the
    Tonemap kernel equals the reference's output up to 1 LSB on a few pixels."""
    import os
    fx = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_queries.npz"))
    hdr = fx["tonemap_hdr"] * np.float32(1.7)
    lib = load_library()
    got = np.empty(len(hdr), np.uint32)
    out = np.zeros(3, np.float32)
    for i, v in enumerate(hdr):
        v = np.ascontiguousarray(v, np.float32)
        assert lib.ar_tone_curve(v.ctypes.data, tone, out.ctypes.data) == 0
        q = [int(np.float32(255.0) * np.float32(min(max(float(c), 0.0), 1.0))) for c in out]
        got[i] = 0xFF000000 | (q[0] << 16) | (q[1] << 8) | q[2]
    ref = fx[f"tonemap_t{tone}_x0"]
    assert (got != ref).mean() <= 5e-4
    assert lib.ar_tone_curve(None, 1, out.ctypes.data) == 1
    assert lib.ar_tone_curve(hdr[0].ctypes.data, 7, out.ctypes.data) == 1
