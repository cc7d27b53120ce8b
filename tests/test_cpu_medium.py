"""Participating medium (extension: delta tracking, ratio tracking,
Henyey-Greenstein) on the CPU oracle: the sampling routines against their
closed forms, and a Beer-Lambert image.  The reference has no volumetric
media (its Henyey-Greenstein helpers, core/render/sample.cuh:110-145, have no
call site), so the checks are statistical against the analytic answers."""
import math

import numpy as np

import oracle
import scenes
from aperture_b200 import make_params


def test_hg_phase_is_normalised_and_sampled_exactly():
    g = 0.3
    mu = np.linspace(-1.0, 1.0, 20001)
    ph = np.array([oracle.hg_phase(g, float(m)) for m in mu[::10]])
    integral = np.trapezoid(ph * 2.0 * math.pi, mu[::10])
    assert abs(integral - 1.0) < 1e-3
    rng = np.random.default_rng(5)
    n = 200_000
    d = np.array([0.3, -0.5, 0.8], np.float32)
    d /= np.linalg.norm(d)
    dirs = oracle.hg_sample(d, g, rng.random((n, 2), dtype=np.float32))
    assert np.allclose(np.linalg.norm(dirs, axis=1), 1.0, atol=1e-5)
    cos = dirs @ d
    assert abs(cos.mean() - g) < 0.005          # E[cos] = g for Henyey-Greenstein
    # histogram of cos against the closed-form CDF
    edges = np.linspace(-1.0, 1.0, 21)
    cdf = (1 - g * g) / (2 * g) * ((1 + g * g - 2 * g * edges) ** -0.5 - 1 / (1 + g))
    expect = np.diff(cdf) * n
    got, _ = np.histogram(cos, edges)
    assert np.all(np.abs(got - expect) < 5 * np.sqrt(expect) + 5)
    # azimuth uniform about d
    t = np.cross([0.0, 0.0, 1.0], d); t /= np.linalg.norm(t)
    b = np.cross(d, t)
    phi = np.arctan2(dirs @ b, dirs @ t)
    hist, _ = np.histogram(phi, np.linspace(-math.pi, math.pi, 9))
    assert np.all(np.abs(hist - n / 8) < 5 * math.sqrt(n / 8))


def _two_voxel_scene():
    osc = oracle.OracleScene(scenes.box_scene())
    grid = np.array([1.0, 0.25], np.float32).reshape(1, 1, 2)
    osc.set_medium(grid, (-0.5, -0.5, -0.5), (0.5, 0.5, 0.5), 2.0, (0.8, 0.8, 0.8), 0.3)
    return osc


def test_medium_density_is_trilinear_between_voxel_centres():
    osc = _two_voxel_scene()
    # voxel centres at x = -0.25 (1.0) and x = 0.25 (0.25), clamped outside
    for x, want in ((-0.5, 1.0), (-0.25, 1.0), (0.0, 0.625), (0.125, 0.4375), (0.25, 0.25), (0.49, 0.25)):
        assert abs(osc.medium_density([x, 0.1, -0.2]) - want) < 1e-6


def test_delta_and_ratio_tracking_match_beer_lambert():
    osc = _two_voxel_scene()
    xs = np.linspace(-0.5, 0.5, 4001)
    dens = np.array([osc.medium_density([x, 0.0, 0.0]) for x in xs])
    tau = 2.0 * np.trapezoid(dens, xs)
    T = math.exp(-tau)
    n = 40_000
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0] = -0.8
    rays[:, 4] = 1.0
    rays[:, 7] = 10.0
    seeds = (np.arange(n, dtype=np.uint64) * 2654435761 % (1 << 32)).astype(np.uint32)
    tc = osc.medium_track(rays, seeds)
    free = (tc < 0).mean()
    sd = math.sqrt(T * (1 - T) / n)
    assert abs(free - T) < 4 * sd, (free, T)
    hit = tc[tc >= 0]
    assert hit.min() >= 0.3 - 1e-6 and hit.max() < 1.3   # collisions only inside the box
    tr = osc.medium_track(rays, seeds ^ np.uint32(0x5bd1e995), ratio=True)
    assert np.all((tr >= 0) & (tr <= 1))
    assert abs(tr.mean() - T) < 4 * tr.std() / math.sqrt(n) + 1e-4, (tr.mean(), T)
    # a segment that ends before the box sees no medium
    short = rays.copy()
    short[:, 7] = 0.25
    assert np.all(osc.medium_track(short[:100], seeds[:100], ratio=True) == 1.0)
    assert np.all(osc.medium_track(short[:100], seeds[:100]) < 0)


def test_fbm_density_is_seeded_and_in_range():
    a = scenes.fbm_density(7, n=32)
    b = scenes.fbm_density(7, n=32)
    c = scenes.fbm_density(8, n=32)
    assert a.shape == (32, 32, 32) and a.dtype == np.float32
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a.min() >= 0.0 and a.max() <= 1.0
    assert 0.2 < (a > 0).mean() < 0.95


def beer_lambert_scene():
    """An emissive slab (radiance 1) at z = -1 seen through a homogeneous
    absorbing slab z in [-0.5, 0.5] (sigma_t 1.5, albedo 0)."""
    L = scenes.cube_object((0.0, 0.0, -1.0), (4.0, 4.0, 0.01))
    scenes.light(L, (1.0, 1.0, 1.0))
    medium = dict(density=np.ones((1, 1, 1), np.float32), bounds_min=(-4.0, -4.0, -0.5), bounds_max=(4.0, 4.0, 0.5),
                  sigma_t_max=1.5, albedo=(0.0, 0.0, 0.0), g=0.0)
    cam = scenes.make_camera((0.0, 0.0, 2.0), (0.0, 0.0, -1.0), 10.0, 12, 12)
    return L, medium, cam


def expected_beer_lambert(cam):
    w, h = cam.width, cam.height
    t = math.tan(math.radians(cam.fov_y_deg) / 2)
    i, j = np.meshgrid(np.arange(w) + 0.5, np.arange(h) + 0.5)
    x = (2 * i / w - 1) * t
    y = (1 - 2 * j / h) * t
    cz = 1.0 / np.sqrt(1 + x * x + y * y)
    return np.exp(-1.5 / cz)


def test_oracle_beer_lambert_image():
    objs, medium, cam = beer_lambert_scene()
    osc = oracle.OracleScene(objs)
    osc.set_medium(**medium)
    spp = 256
    acc, _, _ = osc.render_image(cam, make_params(spp=spp, max_depth=4, sky=0))
    img = acc.reshape(cam.height, cam.width, 3)[..., 0] / spp
    want = expected_beer_lambert(cam)
    assert abs(img.mean() - want.mean()) < 0.02 * want.mean(), (img.mean(), want.mean())
