"""Learned radiance cache, CPU side: the numpy restatement (oracle/nrc_oracle.py)
checked against the closed forms it restates -- spherical harmonics against
their orthonormality, hash-grid indices against the instant-ngp rule, the
backward pass against central finite differences in float64 -- and the bf16
rounding helper against exact halfway cases.  The CUDA kernels are compared
with this restatement in tests/test_gpu_nrc.py."""
import math

import numpy as np

import nrc_oracle as N


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e-20], np.float32)
    r = N.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # halfway, rounds to even mantissa
    assert r[2] == np.float32(1.0 + 4 * 2 ** -8)
    assert r[3] == 1.0
    assert r[4] == -2.5
    assert abs(r[5] - 3.0e-20) / 3.0e-20 < 2 ** -8


def test_sh16_is_orthonormal():
    rng = np.random.default_rng(3)
    d = rng.normal(size=(400_000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    Y = N.sh16(d.astype(np.float32)).astype(np.float64)
    G = Y.T @ Y * (4 * math.pi / len(d))
    assert np.allclose(G, np.eye(16), atol=0.02)


def test_grid_geometry_and_hash():
    g = N.Geometry(16, 19, 16, 2048)
    assert g.res[0] == 16 and g.res[-1] == 2048
    assert all(g.res[i] < g.res[i + 1] for i in range(15))
    assert g.dense[0] and not g.dense[-1]
    u = np.array([[0.5, 0.25, 0.75]], np.float32)
    idx, w = g.corners(u, 15)
    r = g.res[15]
    x, y, z = int(0.5 * r), int(0.25 * r), int(0.75 * r)
    h = (x ^ ((y * 2654435761) & 0xFFFFFFFF) ^ ((z * 805459861) & 0xFFFFFFFF)) & g.mask
    assert idx[0, 0] == h + 15 * g.entries
    assert abs(w.sum() - 1.0) < 1e-6
    idx0, _ = g.corners(u, 0)
    s = g.res[0] + 1
    assert idx0[0, 0] == int(0.5 * 16) + int(0.25 * 16) * s + int(0.75 * 16) * s * s


def _tiny():
    rng = np.random.default_rng(11)
    geo = N.Geometry(3, 8, 2, 8, (-1, -1, -1), (1, 1, 1))
    table = rng.uniform(-0.5, 0.5, (geo.levels * geo.entries, 2))
    W = rng.uniform(-0.3, 0.3, N.PARAMS)
    n = 6
    s = np.zeros((n, 16), np.float64)
    s[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    d = rng.normal(size=(n, 3))
    s[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    s[:, 7] = rng.uniform(0, 1, n)
    nr = rng.normal(size=(n, 3))
    s[:, 8:11] = nr / np.linalg.norm(nr, axis=1, keepdims=True)
    s[:, 12:15] = rng.uniform(0, 1, (n, 3))
    s[:, [3, 11, 15]] = rng.uniform(0.1, 2.0, (n, 3))
    return geo, table, W, s


def test_backward_matches_finite_differences():
    geo, table, W, s = _tiny()
    loss, dT, dW = N.loss_and_gradients(geo, s, table, W, exact=True)
    # denominator held at its unperturbed value, as the loss's gradient holds it
    X, _ = N.encode(geo, s, table, exact=True)
    raw, _ = N.forward(X, N.layer_weights(W, exact=True), exact=True)
    pred = np.exp(np.minimum(raw[:, :3], 15.0))
    den = pred * pred + 0.01
    h = 1e-6
    rng = np.random.default_rng(2)
    for k in rng.choice(N.PARAMS, 25, replace=False).tolist() + [0, 5 * 64 * 64 + 1]:
        Wp, Wm = W.copy(), W.copy()
        Wp[k] += h
        Wm[k] -= h
        lp = N.loss_and_gradients(geo, s, table, Wp, exact=True, den_fixed=den)[0]
        lm = N.loss_and_gradients(geo, s, table, Wm, exact=True, den_fixed=den)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - dW[k]) <= 1e-6 + 1e-4 * abs(fd), (k, fd, dW[k])
    touched = np.argwhere(np.abs(dT) > 0)
    assert len(touched) > 20
    for e, f in touched[rng.choice(len(touched), 20, replace=False)]:
        tp, tm = table.copy(), table.copy()
        tp[e, f] += h
        tm[e, f] -= h
        lp = N.loss_and_gradients(geo, s, tp, W, exact=True, den_fixed=den)[0]
        lm = N.loss_and_gradients(geo, s, tm, W, exact=True, den_fixed=den)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - dT[e, f]) <= 1e-6 + 1e-4 * abs(fd), (e, f, fd, dT[e, f])
