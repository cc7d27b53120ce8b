"""Denoiser on the GPU against the oracle: frame recording bit for bit (from
caller-supplied hits and inside interactive frames), and the bilateral filter
over ragged image sizes with pixels that never hit a surface."""
import os

import numpy as np
import pytest

import aperture_b200 as ab
import oracle
import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TQ = np.load(os.path.join(ROOT, "tests", "golden", "t_quantile_005_ref.npy"))


def to_dev(a: np.ndarray):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()


def from_dev(t, dtype) -> np.ndarray:
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy().view(dtype)


def random_frame(rng, n, p_hit=0.8):
    hits = np.zeros((n, 12), np.float32)
    hits[:, 0:3] = rng.random((n, 3))
    hits[:, 3:6] = rng.normal(size=(n, 3))
    hits[:, 6] = rng.random(n)
    hits[:, 7] = rng.random(n)
    hits[:, 8] = rng.uniform(0.5, 80.0, n)
    hits[:, 9] = rng.integers(0, 4, n)
    hits[:, 10] = rng.random(n) < p_hit
    samples = (rng.gamma(0.8, 1.5, (n, 3)) * (rng.random((n, 1)) < 0.9)).astype(np.float32)
    samples[:5] = [0.0, 0.0, 0.0]
    return hits, samples


@pytest.mark.gpu
def test_record_equals_oracle():
    rng = np.random.default_rng(11)
    n = 5000
    g_ref = np.zeros(n, ab.GBUFFER_DTYPE)
    s_ref = np.zeros(n, ab.STATS_DTYPE)
    g_dev, s_dev = to_dev(g_ref), to_dev(s_ref)
    for _ in range(7):
        hits, samples = random_frame(rng, n)
        oracle.dn_record(hits, samples, g_ref, s_ref)
        ab.denoise_record(to_dev(hits), to_dev(samples), n, g_dev, s_dev)
    assert from_dev(g_dev, np.uint8).tobytes() == g_ref.view(np.uint8).tobytes()
    assert from_dev(s_dev, np.uint8).tobytes() == s_ref.view(np.uint8).tobytes()


def filter_inputs(w, h, frames, seed):
    rng = np.random.default_rng(seed)
    n = w * h
    g = np.zeros(n, ab.GBUFFER_DTYPE)
    s = np.zeros(n, ab.STATS_DTYPE)
    ys, xs = np.meshgrid(np.arange(h), np.arange(w), indexing="ij")
    region = ((xs * 3 // w) + 3 * (ys * 2 // h)).reshape(-1)
    for f in range(frames):
        hits, samples = random_frame(rng, n, p_hit=1.0)
        hits[:, 0:3] = 0.15 * region[:, None] % 1.0 + 0.05 * hits[:, 0:3]
        hits[:, 3:6] = np.stack([np.cos(region), np.sin(region), 0.2 + 0 * region], 1) + 0.05 * hits[:, 3:6]
        hits[:, 8] = 2.0 + region + 0.1 * hits[:, 8] / 80.0
        hits[:, 9] = region % 4
        hits[:, 10] = (ys.reshape(-1) >= 3) | (f % 2 == 0)  # top rows: half the frames miss
        hits[(xs.reshape(-1) == 0) & (ys.reshape(-1) < 2), 10] = 0.0  # never hit: zero normal
        samples *= (1.0 + region[:, None]) / 4.0
        if f >= frames - 1:
            samples[::7] = 0.0
        oracle.dn_record(hits, samples, g, s)
    s[::53] = np.zeros(1, ab.STATS_DTYPE)  # no samples recorded
    img = (rng.gamma(2.0, 0.5, (n, 3)) * (1.0 + region[:, None]) / 3.0).astype(np.float32)
    img[::97] = 0.0
    return img, g, s


@pytest.mark.gpu
@pytest.mark.parametrize("w,h", [(70, 45), (32, 8), (5, 3), (129, 17)])
def test_bilateral_equals_oracle(w, h):
    import torch
    img, g, s = filter_inputs(w, h, 12, w * 1000 + h)
    ref = oracle.dn_bilateral(img, g, s, w, h, TQ)
    out = torch.full((w * h * 3,), float("nan"), dtype=torch.float32, device="cuda")
    ab.denoise_bilateral(torch.from_numpy(img.reshape(-1)).cuda(), out, to_dev(g), to_dev(s), w, h)
    got = out.cpu().numpy()
    assert np.all(np.isfinite(got))
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), np.abs(got - ref).max()
    # the filter changes the image where neighbours pass the test
    assert np.mean(got != img.reshape(-1)) > 0.2


@pytest.mark.gpu
def test_bilateral_rejects_bad_arguments():
    import torch
    buf = torch.zeros(48 * 4, dtype=torch.uint8, device="cuda")
    hdr = torch.zeros(12, dtype=torch.float32, device="cuda")
    with pytest.raises(ab.ArError):
        ab.denoise_bilateral(hdr, hdr, buf, buf, 2, 2)
    with pytest.raises(ab.ArError):
        ab.denoise_bilateral(hdr, torch.zeros_like(hdr), buf, buf, 0, 2)


@pytest.mark.gpu
def test_interactive_frames_record_the_paths():
    """Frames of ar_render_frame_denoise record each frame's sample (equal to
    the per-path radiance of ar_render_debug_paths for the same frame) and the
    primary hit's material, bit for bit against the oracle fed with those."""
    import torch
    objs = scenes.box_scene()
    sc = ab.Scene(objs)
    w, h = 24, 20
    cam = scenes.box_camera(w, h)
    n = w * h
    g_dev = torch.zeros(n * 48, dtype=torch.uint8, device="cuda")
    s_dev = torch.zeros(n * 48, dtype=torch.uint8, device="cuda")
    acc = torch.zeros(n * 3, dtype=torch.float64, device="cuda")
    g_ref = np.zeros(n, ab.GBUFFER_DTYPE)
    s_ref = np.zeros(n, ab.STATS_DTYPE)
    mats = objs["material"]
    frames = 6
    for f in range(frames):
        p = ab.make_params(spp=1, max_depth=8, frame_offset=f)
        ab.render_frame_denoise(sc, cam, p, None, acc, g_dev, s_dev)
        rec = sc.debug_paths(cam, p)
        obj = rec["hit_object"][:, 0]
        hits = np.zeros((n, 12), np.float32)
        hit = obj >= 0
        m = mats[np.where(hit, obj, 0)]
        hits[:, 0:3] = np.stack([m["albedo"]["x"], m["albedo"]["y"], m["albedo"]["z"]], 1)
        hits[:, 6] = m["metallic"]
        hits[:, 7] = m["roughness"]
        hits[:, 9] = m["shading_model"]
        hits[:, 10] = hit
        oracle.dn_record(hits, rec["radiance"].astype(np.float32), g_ref, s_ref)
    g = from_dev(g_dev, ab.GBUFFER_DTYPE)
    s = from_dev(s_dev, ab.STATS_DTYPE)
    assert s.tobytes() == s_ref.tobytes()
    for k in ("albedo", "metallic", "roughness", "valid_frames", "frames", "shading_model"):
        assert np.array_equal(g[k], g_ref[k]), k
    valid = g["valid_frames"] > 0
    assert valid.mean() > 0.5
    nrm = np.linalg.norm(g["normal"].view(np.float16).astype(np.float32), axis=1)
    assert np.all(g["depth"][valid] > 0) and np.all(nrm[valid] < 1.01)
    # the accumulated image is the sum of the recorded samples' frames
    img = (acc.cpu().numpy() / frames).reshape(n, 3)
    assert np.all(np.isfinite(img)) and img.mean() > 0
