"""Learned radiance cache on the GPU: inference and gradients of the CUDA
kernels (bf16 mma.sync MLP, hash-grid encoding and its backward) against the
numpy restatement (oracle/nrc_oracle.py, itself checked against finite
differences), training on a known field, and whole frames of the
cache-terminated tracer converging to the plain tracer's image."""
import numpy as np
import pytest

import nrc_oracle as N
import scenes
from aperture_b200 import RadianceCache, Scene, make_params, nrc_config

BOUNDS = ((-0.6, -0.6, -0.6), (0.6, 0.6, 0.6))


def _cache(**kw):
    cfg = nrc_config(bounds=BOUNDS, **kw)
    sc = Scene(scenes.box_scene())
    return sc, RadianceCache(sc, cfg), cfg


def _vertices(n, seed):
    rng = np.random.default_rng(seed)
    v = np.zeros((n, 16), np.float32)
    v[:, 0:3] = rng.uniform(-0.55, 0.55, (n, 3))
    d = rng.normal(size=(n, 3))
    v[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    v[:, 7] = rng.uniform(0, 1, n)
    nr = rng.normal(size=(n, 3))
    v[:, 8:11] = nr / np.linalg.norm(nr, axis=1, keepdims=True)
    v[:, 12:15] = rng.uniform(0, 1, (n, 3))
    return v


def _random_params(c, seed, tscale=0.5, wscale=0.25):
    rng = np.random.default_rng(seed)
    t = rng.uniform(-tscale, tscale, c.table_floats).astype(np.float32)
    w = rng.uniform(-wscale, wscale, N.PARAMS).astype(np.float32)
    c.set_params(t, w)
    return t.astype(np.float16).astype(np.float32).reshape(-1, 2), w


def _geo(cfg):
    return N.Geometry(cfg.levels, cfg.log2_entries, cfg.base_resolution, cfg.max_resolution, BOUNDS[0], BOUNDS[1])


@pytest.mark.gpu
def test_nrc_inference_equals_oracle():
    _, c, cfg = _cache(log2_entries=15)
    table, w = _random_params(c, 1)
    v = _vertices(5000, 2)
    g = c.infer(v)
    o = N.predict(_geo(cfg), v, table, w)
    rel = np.abs(g - o) / np.maximum(np.abs(o), 1e-6)
    assert np.median(rel) < 1e-3 and np.mean(rel) < 5e-3, (np.median(rel), np.mean(rel), rel.max())
    assert np.percentile(rel, 99) < 0.05


@pytest.mark.gpu
def test_nrc_gradients_equal_oracle():
    _, c, cfg = _cache(log2_entries=15, train_batch=2048)
    table, w = _random_params(c, 3, 0.3, 0.2)
    s = _vertices(2000, 4)
    s[:, [3, 11, 15]] = np.random.default_rng(5).uniform(0.05, 3.0, (2000, 3))
    tg, wg, loss = c.gradients(s)
    lo, dT, dW = N.loss_and_gradients(_geo(cfg), s, table, w)
    assert abs(loss - lo) <= 1e-3 * abs(lo)
    assert np.linalg.norm(wg - dW) <= 2e-2 * np.linalg.norm(dW)
    dT = dT.reshape(-1)
    assert np.linalg.norm(tg - dT) <= 2e-2 * np.linalg.norm(dT)
    assert np.count_nonzero(dT) > 10000


@pytest.mark.gpu
def test_nrc_training_fits_a_smooth_field():
    _, c, cfg = _cache(log2_entries=16, train_batch=4096)
    s = _vertices(4096 * 50, 6)
    p, d = s[:, 0:3], s[:, 4:7]
    field = np.stack([1.0 + np.sin(4 * p[:, 0]) * 0.5 + 0.3 * d[:, 1],
                      0.5 + 0.4 * np.cos(3 * p[:, 1] + p[:, 2]),
                      0.2 + np.exp(-4 * (p ** 2).sum(1)) + 0.2 * (d[:, 2] > 0)], 1)
    s[:, [3, 11, 15]] = field
    losses = c.train(s, 50)
    losses2 = np.concatenate([c.train(s, 50) for _ in range(3)])
    assert losses2[-10:].mean() < 0.1 * losses[:3].mean(), (losses[:3], losses2[-10:])
    test = _vertices(4000, 7)
    pt, dt = test[:, 0:3], test[:, 4:7]
    want = np.stack([1.0 + np.sin(4 * pt[:, 0]) * 0.5 + 0.3 * dt[:, 1],
                     0.5 + 0.4 * np.cos(3 * pt[:, 1] + pt[:, 2]),
                     0.2 + np.exp(-4 * (pt ** 2).sum(1)) + 0.2 * (dt[:, 2] > 0)], 1)
    got = c.infer(test)
    assert np.mean(np.abs(got - want) / want) < 0.1


@pytest.mark.gpu
def test_nrc_frames_converge_to_plain_image():
    import torch
    objs = scenes.box_scene()
    sc = Scene(objs)
    cam = scenes.box_camera(64, 64)
    ref, _ = sc.render(cam, make_params(spp=1024, max_depth=8))
    cfg = nrc_config(bounds=BOUNDS, log2_entries=16, train_paths=1024, train_batch=2048, train_steps=2)
    c = RadianceCache(sc, cfg)
    n = 64 * 64 * 3
    acc = torch.zeros(n, dtype=torch.float64, device="cuda")
    frames = 256
    queries = 0
    for f in range(frames):
        st = c.render_frame(cam, make_params(spp=1, max_depth=8, frame_offset=f), None, acc.data_ptr(),
                            train=True, stats=(f % 64 == 63))
        if st is not None:
            queries = st.queries
            assert st.train_samples > 500
    img = (acc / frames).cpu().numpy().reshape(64, 64, 3)
    rel = ((img - ref) ** 2 / (ref ** 2 + 1e-2)).mean()
    assert queries > 1000
    assert rel < 0.02, rel
    # what the trained network gains: the plain tracer at the same number of
    # samples, and the same frames with a cache that is never trained
    plain, _ = sc.render(cam, make_params(spp=frames, max_depth=8, frame_offset=100000))
    rel_plain = ((plain - ref) ** 2 / (ref ** 2 + 1e-2)).mean()
    c0 = RadianceCache(sc, cfg)
    acc0 = torch.zeros(n, dtype=torch.float64, device="cuda")
    for f in range(frames):
        c0.render_frame(cam, make_params(spp=1, max_depth=8, frame_offset=f), None, acc0.data_ptr(), train=False)
    img0 = (acc0 / frames).cpu().numpy().reshape(64, 64, 3)
    rel_untrained = ((img0 - ref) ** 2 / (ref ** 2 + 1e-2)).mean()
    print("relMSE cache", rel, "plain", rel_plain, "untrained cache", rel_untrained)
    assert rel < rel_plain, (rel, rel_plain)
    assert rel < 0.5 * rel_untrained, (rel, rel_untrained)


@pytest.mark.gpu
def test_nrc_tcgen05_inference_equals_mma_sync():
    """The tcgen05 inference kernel (128-row tiles, tensor-memory accumulators)
    and the mma.sync kernel compute the same bf16 network with fp32 sums in
    the same order per output: identical predictions."""
    _, c, cfg = _cache(log2_entries=15)
    table, w = _random_params(c, 11)
    v = _vertices(70_000, 12)      # several tiles per CTA, a ragged last tile
    c.set_tensor_path(False)
    a = c.infer(v)
    c.set_tensor_path(True)
    b = c.infer(v)
    assert np.array_equal(a, b)
    o = N.predict(_geo(cfg), v, table, w)
    rel = np.abs(b - o) / np.maximum(np.abs(o), 1e-6)
    assert np.median(rel) < 1e-3 and np.mean(rel) < 5e-3


@pytest.mark.gpu
def test_nrc_frames_of_several_samples():
    """A cache frame of k samples per pixel: every sample may end in the cache,
    sample 0 of the training pixels trains, out_rgb is the mean over the k
    samples and accum gets their sums.  With the cache frozen (train off),
    k-sample frames and k times as many one-sample frames estimate the same
    image."""
    import torch
    objs = scenes.box_scene()
    sc = Scene(objs)
    cam = scenes.box_camera(48, 48)
    cfg = nrc_config(bounds=BOUNDS, log2_entries=15, train_paths=1024, train_batch=1024, train_steps=2)
    c = RadianceCache(sc, cfg)
    n = 48 * 48 * 3
    acc = torch.zeros(n, dtype=torch.float64, device="cuda")
    for f in range(16):   # train a little with 4-sample frames
        st = c.render_frame(cam, make_params(spp=4, max_depth=8, frame_offset=4 * f), None, acc.data_ptr(),
                            train=True, stats=(f == 15))
    assert st.queries > 4 * 500 and 500 < st.train_samples
    out = torch.empty(n, dtype=torch.float32, device="cuda")
    acc_k = torch.zeros(n, dtype=torch.float64, device="cuda")
    acc_1 = torch.zeros(n, dtype=torch.float64, device="cuda")
    k, frames = 8, 32
    for f in range(frames):
        c.render_frame(cam, make_params(spp=k, max_depth=8, frame_offset=1000 + k * f), out.data_ptr(),
                       acc_k.data_ptr(), train=False)
    for f in range(frames * k):
        c.render_frame(cam, make_params(spp=1, max_depth=8, frame_offset=100000 + f), None, acc_1.data_ptr(),
                       train=False)
    a = (acc_k / (frames * k)).cpu().numpy()
    b = (acc_1 / (frames * k)).cpu().numpy()
    assert np.isfinite(a).all() and abs(a.mean() - b.mean()) < 0.02 * b.mean()
    last = out.cpu().numpy()
    assert abs(last.mean() - a.mean()) < 0.1 * a.mean()    # out_rgb is the k-sample mean, not the sum


def _spectral_cache(**kw):
    import spectral_tables
    if not spectral_tables.available():
        pytest.skip("spectral tables not built")
    cfg = nrc_config(bounds=BOUNDS, **kw)
    sc = Scene(scenes.box_scene())
    sc.set_spectral(32)
    c = RadianceCache(sc, cfg)
    c.set_spectral(4)
    return sc, c, cfg


@pytest.mark.gpu
def test_nrc_spectral_inference_equals_oracle():
    """Four-wavelength cache: the 16 exp'd spectral bins of the tcgen05 and
    mma.sync kernels are identical and agree with the numpy restatement."""
    _, c, cfg = _spectral_cache(log2_entries=15)
    table, w = _random_params(c, 21)
    v = _vertices(6000, 22)
    c.set_tensor_path(True)
    a = c.infer(v)
    c.set_tensor_path(False)
    b = c.infer(v)
    assert a.shape == (6000, 16) and np.array_equal(a, b)
    o = N.predict_bins(_geo(cfg), v, table, w)
    rel = np.abs(a - o) / np.maximum(np.abs(o), 1e-6)
    assert np.median(rel) < 1e-3 and np.mean(rel) < 5e-3


@pytest.mark.gpu
def test_nrc_spectral_gradients_equal_oracle():
    """Four-wavelength loss (per-wavelength relative L2 of the interpolated
    bins, negative targets left out) and its gradients against the numpy
    restatement."""
    _, c, cfg = _spectral_cache(log2_entries=15, train_batch=2048)
    table, w = _random_params(c, 23, 0.3, 0.2)
    rng = np.random.default_rng(24)
    s = np.zeros((2000, 20), np.float32)
    s[:, :16] = _vertices(2000, 25)
    s[:, [3, 11, 15, 16]] = rng.uniform(0.05, 3.0, (2000, 4))
    s[rng.random(2000) < 0.1, 16] = -1.0            # wavelength 3 without throughput
    s[:, 17] = rng.uniform(360.0, 780.0, 2000)       # hero wavelength
    tg, wg, loss = c.gradients(s)
    lo, dT, dW = N.loss_and_gradients_spectral(_geo(cfg), s, table, w)
    assert abs(loss - lo) <= 2e-3 * abs(lo)
    assert np.linalg.norm(wg - dW) <= 2e-2 * np.linalg.norm(dW)
    dT = dT.reshape(-1)
    assert np.linalg.norm(tg - dT) <= 2e-2 * np.linalg.norm(dT)


@pytest.mark.gpu
def test_nrc_spectral_frames_converge_to_plain_image():
    """Frames of four wavelengths per path with the four-wavelength cache: after
    32 frames of online training the XYZ image of the next 96 frames agrees
    with the plain four-wavelength tracer's within 10 % per channel mean (the
    cache's bias), with paths ending in the cache and a finite training loss."""
    import torch
    sc, c, cfg = _spectral_cache(log2_entries=16, train_paths=2048, train_batch=2048, train_steps=2)
    cam = scenes.box_camera(48, 48)
    ref, _ = sc.render(cam, make_params(spp=1024, max_depth=8, spectral=4))
    warm = torch.zeros(48 * 48 * 3, dtype=torch.float64, device="cuda")
    for f in range(32):
        c.render_frame(cam, make_params(spp=2, max_depth=8, spectral=4, frame_offset=2 * f), None, warm.data_ptr(),
                       train=True)
    acc = torch.zeros(48 * 48 * 3, dtype=torch.float64, device="cuda")
    frames = 96
    st = None
    for f in range(frames):
        st = c.render_frame(cam, make_params(spp=2, max_depth=8, spectral=4, frame_offset=1000 + 2 * f), None,
                            acc.data_ptr(), train=True, stats=(f == frames - 1))
    assert st.queries > 500 and st.train_samples > 500 and np.isfinite(st.loss)
    img = (acc / (2 * frames)).cpu().numpy().reshape(48, 48, 3)
    assert np.isfinite(img).all()
    m, r = img.mean(axis=(0, 1)), ref.reshape(48, 48, 3).mean(axis=(0, 1))
    assert np.all(np.abs(m - r) < 0.10 * r), (m, r)
    with pytest.raises(Exception):   # a frame of another mode than the cache's
        c.render_frame(cam, make_params(spp=1, max_depth=8), None, acc.data_ptr(), train=False)


@pytest.mark.gpu
@pytest.mark.parametrize("spectral", [0, 4])
def test_nrc_tcgen05_training_equals_mma_sync(spectral):
    """Training forward and backward on the tcgen05 tensor cores (128-row
    tiles, tensor-memory accumulators, the transposed weights for the
    backward chain) against the warp-level mma.sync kernels and the numpy
    restatement: losses equal to 1e-4, gradients within 1e-2 (bf16 rounding of
    the layer gradients after a different fp32 summation order) of each other
    and within 2e-2 of the oracle."""
    if spectral:
        _, c, cfg = _spectral_cache(log2_entries=15, train_batch=2048)
    else:
        _, c, cfg = _cache(log2_entries=15, train_batch=2048)
    table, w = _random_params(c, 31, 0.3, 0.2)
    rng = np.random.default_rng(32)
    s = np.zeros((2000, 20), np.float32)
    s[:, :16] = _vertices(2000, 33)
    s[:, [3, 11, 15, 16]] = rng.uniform(0.05, 3.0, (2000, 4))
    s[:, 17] = rng.uniform(360.0, 780.0, 2000)
    c.set_tensor_path(False)
    tg0, wg0, l0 = c.gradients(s)
    c.set_tensor_path(True)
    tg1, wg1, l1 = c.gradients(s)
    assert abs(l1 - l0) <= 1e-4 * abs(l0)
    assert np.linalg.norm(wg1 - wg0) <= 1e-2 * np.linalg.norm(wg0)
    assert np.linalg.norm(tg1 - tg0) <= 1e-2 * np.linalg.norm(tg0)
    lo, dT, dW = (N.loss_and_gradients_spectral(_geo(cfg), s, table, w) if spectral
                  else N.loss_and_gradients(_geo(cfg), s[:, :16], table, w))
    assert np.linalg.norm(wg1 - dW) <= 2e-2 * np.linalg.norm(dW)
    assert np.linalg.norm(tg1 - dT.reshape(-1)) <= 2e-2 * np.linalg.norm(dT)
