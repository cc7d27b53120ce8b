"""Denoiser on the CPU: the t-quantile table against the reference's table, and
the oracle's recording and bilateral filter against closed-form expectations."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "aperturerendererv3-optix-geometry_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import aperture_b200 as ab  # noqa: E402
import oracle  # noqa: E402

TABLE_H = os.path.join(PKG, "csrc", "t_quantile_table.h")
FIXTURE = os.path.join(ROOT, "tests", "golden", "t_quantile_005_ref.npy")


def t_table() -> np.ndarray:
    body = open(TABLE_H).read().split("kTQuantiles] = {", 1)[1].split("}", 1)[0]
    return np.array([float.fromhex(v.strip().rstrip("f")) for v in body.split(",") if v.strip()], np.float32)


def test_t_quantile_table_equals_reference_table():
    ours, ref = t_table(), np.load(FIXTURE)
    assert ours.shape == (1024,) and np.array_equal(ours.view(np.uint32), ref.view(np.uint32))


def test_t_quantile_table_is_regenerated_by_its_script():
    pytest.importorskip("scipy")
    import make_t_quantiles
    assert np.array_equal(make_t_quantiles.table().view(np.uint32), t_table().view(np.uint32))


def boxcox(x):
    return (np.sqrt(np.maximum(x, 0.0)) - 1.0) * 2.0


def test_recorded_moments_match_float64_moments():
    rng = np.random.default_rng(5)
    n, frames = 64, 40
    st = np.zeros(n, ab.STATS_DTYPE)
    xs = rng.gamma(0.7, 2.0, size=(frames, n, 3)).astype(np.float32)
    xs[:, :4] = 0.0  # constant pixels: zero variance
    for f in range(frames):
        oracle.dn_record(None, xs[f], None, st)
    bc = boxcox(xs.astype(np.float64))
    mean = bc.mean(0)
    m2 = ((bc - mean) ** 2).mean(0)
    m3 = ((bc - mean) ** 3).mean(0)
    assert np.all(st["num"] == frames)
    assert np.allclose(st["mean"], mean, rtol=1e-5, atol=1e-5)
    assert np.allclose(st["m2_div_n"], m2, rtol=1e-4, atol=1e-6)
    assert np.allclose(st["m3_div_n"], m3, rtol=1e-3, atol=1e-5)
    assert np.all(st["m2_div_n"][:4] == 0.0)


def test_recorded_gbuffer_is_the_running_mean():
    rng = np.random.default_rng(6)
    n, frames = 32, 24
    g = np.zeros(n, ab.GBUFFER_DTYPE)
    hit = rng.random((frames, n)) < 0.75
    hit[:, 0] = False  # never hit
    hits = np.zeros((frames, n, 12), np.float32)
    hits[..., 0:3] = rng.random((frames, n, 3))
    hits[..., 3:6] = rng.normal(size=(frames, n, 3))
    hits[..., 6] = rng.random((frames, n))
    hits[..., 7] = rng.random((frames, n))
    hits[..., 8] = rng.uniform(1, 50, (frames, n))
    hits[..., 9] = rng.integers(0, 4, (frames, n))
    hits[..., 10] = hit
    for f in range(frames):
        oracle.dn_record(hits[f], None, g, None)
    assert np.all(g["frames"] == frames)
    assert np.array_equal(g["valid_frames"], hit.sum(0))
    h2f = lambda a: a.view(np.float16).astype(np.float64)  # noqa: E731
    for i in range(1, n):
        sel = hits[hit[:, i], i]
        assert np.allclose(h2f(g["albedo"][i]), sel[:, 0:3].mean(0), atol=4e-3)
        assert np.isclose(g["depth"][i], sel[:, 8].mean(), rtol=1e-4)
        share = np.array([(sel[:, 9] == m).sum() for m in range(4)] + [frames - len(sel)]) / frames
        assert np.allclose(h2f(g["shading_model"][i][:5]), share, atol=4e-3)
    assert h2f(g["shading_model"][0][4]) == 1.0 and g["valid_frames"][0] == 0


def recorded_buffers(w, h, frames, seed, image=None):
    """Guide buffers of a synthetic scene: two flat regions with their own
    albedo, normal and depth; a band of pixels that never hit a surface."""
    rng = np.random.default_rng(seed)
    n = w * h
    g = np.zeros(n, ab.GBUFFER_DTYPE)
    st = np.zeros(n, ab.STATS_DTYPE)
    xs, ys = np.meshgrid(np.arange(w), np.arange(h))
    left = (xs < w // 2).reshape(-1)
    sky = (ys < 2).reshape(-1)
    for _ in range(frames):
        hits = np.zeros((n, 12), np.float32)
        hits[:, 0:3] = np.where(left[:, None], [0.7, 0.2, 0.2], [0.2, 0.6, 0.3])
        hits[:, 3:6] = np.where(left[:, None], [0.0, 1.0, 0.0], [1.0, 0.0, 0.0])
        hits[:, 8] = np.where(left, 3.0, 9.0)
        hits[:, 9] = np.where(left, 0, 3)
        hits[:, 10] = ~sky
        base = np.where(left[:, None], [0.8, 0.5, 0.3], [0.2, 0.3, 0.9]) if image is None else image
        samples = (base * rng.gamma(4.0, 0.25, size=(n, 3))).astype(np.float32)
        oracle.dn_record(hits, samples, g, st)
    return g, st


def test_bilateral_keeps_flat_regions_and_isolated_pixels():
    w, h = 24, 12
    g, st = recorded_buffers(w, h, 16, 7)
    img = np.zeros((h, w, 3), np.float32)
    img[:, : w // 2] = [0.8, 0.5, 0.3]
    img[:, w // 2:] = [0.2, 0.3, 0.9]
    out = oracle.dn_bilateral(img, g, st, w, h, np.load(FIXTURE)).reshape(h, w, 3)
    # a constant region filters to itself; sky pixels (zero normal) keep their value
    assert np.allclose(out[4:, 2:8], img[4:, 2:8], rtol=2e-5)
    assert np.allclose(out[:2], img[:2], rtol=2e-5)
    assert np.all(np.isfinite(out))
    # no samples recorded: every t-test fails and each pixel is its own output
    out0 = oracle.dn_bilateral(img, g, np.zeros_like(st), w, h, np.load(FIXTURE)).reshape(h, w, 3)
    assert np.allclose(out0, img, rtol=2e-5)


def test_bilateral_lowers_noise_within_a_region():
    w, h = 32, 16
    g, st = recorded_buffers(w, h, 32, 8)
    rng = np.random.default_rng(9)
    clean = np.full((h, w, 3), 0.5, np.float32)
    noisy = (clean * rng.gamma(8.0, 1 / 8.0, size=clean.shape)).astype(np.float32)
    out = oracle.dn_bilateral(noisy, g, st, w, h, np.load(FIXTURE)).reshape(h, w, 3)
    region = (slice(4, h), slice(0, w // 2 - 4))
    assert np.std(out[region]) < 0.5 * np.std(noisy[region])


def test_sqrt_thresholds_decide_the_t_test_exactly():
    """The filter compares x < threshold instead of sqrtf(x) < quantile."""
    body = open(TABLE_H).read()
    b = body.split("kTQuantileSqrtThreshold[kTQuantiles] = {", 1)[1].split("}", 1)[0]
    thr = np.array([float.fromhex(v.strip().rstrip("f")) for v in b.split(",") if v.strip()], np.float32)
    q = t_table()
    assert np.all(np.sqrt(thr) >= q) and np.all(np.sqrt(np.nextafter(thr, np.float32(0))) < q)
    rng = np.random.default_rng(1)
    for k in range(0, 1024, 31):
        xs = (thr[k] * (1 + rng.uniform(-1e-5, 1e-5, 4000))).astype(np.float32)
        xs = np.concatenate([xs, np.float32([0.0, -0.0, -1e-30, np.inf, np.nan])])
        with np.errstate(invalid="ignore"):
            assert np.array_equal(np.sqrt(xs) < q[k], ~(xs < 0) & (xs < thr[k]))
