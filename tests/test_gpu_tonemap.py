"""ar_tonemap (the output epilogue kernel) against the oracle's restatement of
the reference's Tonemap kernel, on HDR values spanning 1e-4 .. 1e3 and on a
rendered image, host and device buffers."""
import ctypes

import numpy as np
import pytest

import oracle
import scenes
from aperture_b200 import MEM_DEVICE, Scene, load_library, make_params, tonemap


def _hdr(n, seed):
    rng = np.random.default_rng(seed)
    h = np.exp(rng.normal(-1.0, 2.0, (n, 3))).astype(np.float32)
    h[:64] = 0.0
    return h


@pytest.mark.gpu
@pytest.mark.parametrize("tone", [0, 1, 2])
@pytest.mark.parametrize("xyz", [False, True])
def test_tonemap_equals_oracle(tone, xyz):
    hdr = _hdr(300_000, 5 + tone)
    assert np.array_equal(tonemap(hdr, tone, 1.3, xyz), oracle.tonemap(hdr, tone, 1.3, xyz))


@pytest.mark.gpu
def test_tonemap_device_buffers_of_a_render(box_objects):
    import torch
    scene = Scene(box_objects)
    cam = scenes.box_camera(64, 48)
    img, _ = scene.render(cam, make_params(spp=4, max_depth=8))
    dev = torch.from_numpy(np.ascontiguousarray(img, np.float32).reshape(-1)).cuda()
    out = torch.zeros(64 * 48, dtype=torch.int32, device="cuda")
    lib = load_library()
    st = lib.ar_tonemap(ctypes.c_void_p(dev.data_ptr()), 64 * 48, 2, 1.0, 0, ctypes.c_void_p(out.data_ptr()),
                        MEM_DEVICE, None)
    torch.cuda.synchronize()
    assert st == 0
    got = out.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, oracle.tonemap(img.reshape(-1, 3), 2, 1.0))
    assert np.all((got >> 24) == 0xFF)
