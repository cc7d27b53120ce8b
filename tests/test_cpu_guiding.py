"""Path-guiding probe math on the CPU (oracle/guiding_oracle.py): the
equal-area octahedral map, the probe density and its mip-descent sampler."""
import math

import numpy as np

import guiding_oracle as G


def test_equal_area_map_round_trip_and_uniformity():
    rng = np.random.default_rng(1)
    su, sv = rng.random(200_000), rng.random(200_000)
    w = G.uv_to_dir(su, sv)
    assert np.allclose(np.linalg.norm(w, axis=1), 1.0, atol=1e-12)
    u2, v2 = G.dir_to_uv(w)
    assert np.allclose(u2, su, atol=1e-9) and np.allclose(v2, sv, atol=1e-9)
    # equal area: z uniform in [-1, 1], azimuth uniform
    hz, _ = np.histogram(w[:, 2], np.linspace(-1, 1, 21))
    assert np.all(np.abs(hz - 10_000) < 5 * math.sqrt(10_000))
    ha, _ = np.histogram(np.arctan2(w[:, 1], w[:, 0]), np.linspace(-math.pi, math.pi, 17))
    assert np.all(np.abs(ha - 12_500) < 5 * math.sqrt(12_500))


def test_probe_density_is_normalised_and_matches_sampler():
    rng = np.random.default_rng(2)
    tex = G.build_mips(rng.gamma(0.5, 1.0, (64, 3)))
    q = np.array([0.2, 0.5, 0.3])
    # density integrates to 1 over the sphere (equal-area uniform samples)
    w = G.uv_to_dir(rng.random(400_000), rng.random(400_000))
    assert abs(np.mean(G.pdf(tex, w, q)) * 4 * math.pi - 1.0) < 0.01
    # the hemisphere density integrates to 1 over the hemisphere
    n = np.array([0.3, -0.4, 0.866])
    n /= np.linalg.norm(n)
    assert abs(np.mean(G.hemi_pdf(tex, w, n, q)) * 4 * math.pi - 1.0) < 0.01
    # mip descent picks leaf texels with probability w_leaf / sum w
    wl = tex[:64] @ q
    want = wl / wl.sum()
    counts = np.zeros(64)
    for u in rng.random((40_000, 3)):
        x, y, p = G.sample_leaf(tex, q, u)
        counts[y * 8 + x] += 1
        assert abs(p - want[y * 8 + x]) < 1e-9
    assert np.all(np.abs(counts / 40_000 - want) < 5 * np.sqrt(want / 40_000) + 1e-4)


def test_mips_are_averages():
    rng = np.random.default_rng(3)
    leaves = rng.random((64, 3))
    tex = G.build_mips(leaves)
    assert np.allclose(tex[84], leaves.mean(0))
    assert np.allclose(tex[80:84].mean(0), tex[84])


def test_probe_math_matches_reference():
    """The numpy restatement against the reference's own Octahedron and grid,
    run on the host (tests/golden/reference_guiding.npz): the 20 face normals
    in the reference's numbering, the (voxel, face) grid of points and
    directions exactly; hemisphere sample directions within 2e-6 and pdfs
    within 2e-5 relative (float against float64 arithmetic)."""
    import os
    fx = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_guiding.npz"))
    assert np.array_equal(G.face_normals(), fx["faces"])
    assert np.array_equal(G.voxel_grid(fx["pos"], fx["eval_dir"]), fx["voxel"])
    tex = fx["texels"][:, :, :3].astype(np.float64)
    n = 2000
    dirs, pdfs, epdfs = [], [], []
    for i in range(n):
        t = tex[fx["probe_of"][i]]
        w, p = G.sample_hemi(t, fx["normal"][i], fx["query"][i], fx["u5"][i].astype(np.float64))
        dirs.append(w)
        pdfs.append(p)
        epdfs.append(float(G.hemi_pdf(t, fx["eval_dir"][i][None].astype(np.float64), fx["normal"][i].astype(np.float64),
                                      fx["query"][i])[0]))
    assert np.abs(np.array(dirs) - fx["dir"][:n]).max() < 2e-6
    assert np.max(np.abs(np.array(pdfs) - fx["pdf"][:n]) / fx["pdf"][:n]) < 2e-5
    e = fx["epdf"][:n]
    assert np.array_equal(np.array(epdfs) == 0, e == 0)
    nz = e > 0
    assert np.max(np.abs(np.array(epdfs)[nz] - e[nz]) / e[nz]) < 2e-5
