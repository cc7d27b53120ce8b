"""CPU restatement of the learned radiance cache -- TEST INFRASTRUCTURE ONLY.

Only tests/ (and nothing on the product path) import this module; it is the
checker of the CUDA cache kernels (aperturerendererv3-optix-geometry_b200/csrc/nrc.cu),
never the thing measured or shipped.

The reference renderer has no radiance cache, so nothing of the reference pins
this restatement ("parity unpinned" for the reference); it is pinned instead
to the published method it restates and to itself:
  * the hash-grid encoding of Mueller et al. 2022 (instant-ngp): levels with
    resolutions base * b^l, b = (max / base)^(1 / (levels - 1)); a level is
    indexed densely when (res + 1)^3 fits its table, else by the spatial hash
    x * 1 ^ y * 2654435761 ^ z * 805459861 (Teschner et al. 2003) modulo the
    table size; trilinear interpolation of 2 features;
  * real spherical harmonics of degree 0-3 (16 coefficients) of the outgoing
    direction; roughness, albedo, normal * 0.5 + 0.5 and a constant 1;
  * an MLP of 5 hidden ReLU layers of width 64 and a 16-wide output whose
    first 3 columns pass through exp (Mueller et al. 2021); bf16 weights and
    activations (round to nearest even), fp32 sums;
  * the relative L2 loss (pred - target)^2 / (pred^2 + 0.01) with the
    denominator held constant, averaged over samples and channels;
  * backward propagation, checked against central finite differences in
    float64 (tests/test_cpu_nrc.py).
The float32 arithmetic of the encoding follows the device code operation by
operation, so indices and weights agree exactly and features to rounding.
"""
from __future__ import annotations

import math

import numpy as np

IN, HID, OUT, LAYERS = 64, 64, 16, 6
PARAMS = 5 * HID * IN + OUT * HID
SH_C = (0.28209479177387814, 0.48860251190291987, 1.0925484305920792, 0.94617469575755997, 0.31539156525251999,
        0.54627421529603959, 0.59004358992664352, 2.8906114426405538, 0.45704579946446572, 0.3731763325901154,
        1.4453057213202769)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).reshape(a.shape)


class Geometry:
    """Hash-grid geometry of ar_nrc_create."""

    def __init__(self, levels=16, log2_entries=19, base=16, maxres=2048, bmin=(0, 0, 0), bmax=(1, 1, 1)):
        self.levels = levels
        self.entries = 1 << log2_entries
        self.mask = self.entries - 1
        b = math.exp((math.log(maxres) - math.log(base)) / (levels - 1)) if levels > 1 else 1.0
        self.res = [int(math.floor(base * b ** l + 1e-6)) for l in range(levels)]
        self.dense = [(r + 1) ** 3 <= self.entries for r in self.res]
        self.bmin = np.asarray(bmin, np.float32)
        self.inv_ext = (np.float32(1.0) / (np.asarray(bmax, np.float32) - self.bmin)).astype(np.float32)

    def unit(self, p: np.ndarray) -> np.ndarray:
        u = (p.astype(np.float32) - self.bmin) * self.inv_ext
        return np.clip(u, 0.0, 1.0).astype(np.float32)

    def corners(self, u: np.ndarray, l: int):
        """(n, 8) table entry indices and float32 trilinear weights of level l."""
        r = self.res[l]
        f = (u * np.float32(r)).astype(np.float32)
        i = np.clip(np.floor(f).astype(np.int64), 0, r - 1)
        t = np.clip(f - i.astype(np.float32), 0.0, 1.0).astype(np.float32)
        stride = np.uint64(r + 1)
        idx = np.empty((len(u), 8), np.int64)
        w = np.empty((len(u), 8), np.float32)
        one = np.float32(1.0)
        for c in range(8):
            bits = ((c & 1), (c >> 1) & 1, (c >> 2) & 1)
            cx, cy, cz = [(i[:, a] + bits[a]).astype(np.uint64) for a in range(3)]
            if self.dense[l]:
                h = (cx + cy * stride + cz * stride * stride) & np.uint64(0xFFFFFFFF)
            else:
                h = ((cx * np.uint64(1)) ^ (cy * np.uint64(2654435761)) ^ (cz * np.uint64(805459861))) & np.uint64(0xFFFFFFFF)
            idx[:, c] = (h & np.uint64(self.mask)).astype(np.int64) + l * self.entries
            wx = t[:, 0] if bits[0] else one - t[:, 0]
            wy = t[:, 1] if bits[1] else one - t[:, 1]
            wz = t[:, 2] if bits[2] else one - t[:, 2]
            w[:, c] = (wx * wy).astype(np.float32) * wz
        return idx, w


def sh16(d: np.ndarray) -> np.ndarray:
    x, y, z = (d[:, k].astype(np.float32) for k in range(3))
    xx, yy, zz = x * x, y * y, z * z
    c = [np.float32(v) for v in SH_C]
    o = np.empty((len(d), 16), np.float32)
    o[:, 0] = c[0]
    o[:, 1] = -c[1] * y
    o[:, 2] = c[1] * z
    o[:, 3] = -c[1] * x
    o[:, 4] = c[2] * x * y
    o[:, 5] = -c[2] * y * z
    o[:, 6] = c[3] * zz - c[4]
    o[:, 7] = -c[2] * x * z
    o[:, 8] = c[5] * (xx - yy)
    o[:, 9] = c[6] * y * (np.float32(-3.0) * xx + yy)
    o[:, 10] = c[7] * x * y * z
    o[:, 11] = c[8] * y * (np.float32(1.0) - np.float32(5.0) * zz)
    o[:, 12] = c[9] * z * (np.float32(5.0) * zz - np.float32(3.0))
    o[:, 13] = c[8] * x * (np.float32(1.0) - np.float32(5.0) * zz)
    o[:, 14] = c[10] * z * (xx - yy)
    o[:, 15] = c[6] * x * (-xx + np.float32(3.0) * yy)
    return o


def encode(geo: Geometry, v: np.ndarray, table: np.ndarray, exact: bool = False):
    """Network inputs (n, 64) of vertices v (n, 16) with table values
    (levels * entries, 2) as the device reads them (half -> float).  Returns
    (inputs, per-level corner (idx, w) for the backward pass)."""
    n = len(v)
    dt = np.float64 if exact else np.float32
    X = np.zeros((n, IN), dt)
    u = geo.unit(v[:, 0:3])
    cw = []
    for l in range(geo.levels):
        idx, w = geo.corners(u, l)
        cw.append((idx, w))
        f = np.zeros((n, 2), dt)
        for c in range(8):
            f = f + w[:, c:c + 1].astype(dt) * table[idx[:, c]].astype(dt)
        X[:, 2 * l:2 * l + 2] = f
    X[:, 32:48] = sh16(v[:, 4:7])
    X[:, 48] = v[:, 7]
    X[:, 49:52] = v[:, 12:15]
    X[:, 52:55] = v[:, 8:11] * np.float32(0.5) + np.float32(0.5)
    X[:, 55] = 1.0
    return (X if exact else bf16(X)), cw


def layer_weights(W: np.ndarray, exact: bool = False):
    out = []
    for l in range(LAYERS):
        rows = OUT if l == LAYERS - 1 else HID
        m = W[l * HID * IN: l * HID * IN + rows * IN].reshape(rows, IN)
        out.append(m.astype(np.float64) if exact else bf16(m))
    return out


def forward(X: np.ndarray, Ws, exact: bool = False):
    """Raw outputs (n, 16) and the stored activations [X, H1..H5]."""
    acts = [X]
    h = X
    for l in range(LAYERS - 1):
        z = h @ Ws[l].T
        h = np.maximum(z, 0.0)
        if not exact:
            h = bf16(h.astype(np.float32))
        acts.append(h)
    return h @ Ws[LAYERS - 1].T, acts


def predict(geo: Geometry, v: np.ndarray, table: np.ndarray, W: np.ndarray) -> np.ndarray:
    X, _ = encode(geo, v, table)
    raw, _ = forward(X, layer_weights(W))
    return np.exp(np.minimum(raw[:, :3], 15.0)).astype(np.float32)


# Four-wavelength cache: 16 spectral bins of 26.25 nm over [360, 780] nm,
# linear interpolation between bin centres (csrc/nrc.cuh, nrc_bin_weights),
# the path's wavelengths the hero and its rotations by 105 nm in [360, 780].
BINS, LAMBDA0, BIN_WIDTH = 16, 360.0, 26.25


def rotate_lambda(h, i):
    """csrc/spectral.cuh rotate_lambda, in float32"""
    x = (np.asarray(h, np.float32) - np.float32(360.0)) + np.float32(105.0) * np.float32(i)
    x = np.where(x >= np.float32(420.0), x - np.float32(420.0), x).astype(np.float32)
    return (np.float32(360.0) + x).astype(np.float32)


def bin_weights(lam):
    x = (np.asarray(lam, np.float32) - np.float32(LAMBDA0)) / np.float32(BIN_WIDTH) - np.float32(0.5)
    x = np.clip(x, 0.0, BINS - 1).astype(np.float32)
    b = np.minimum(np.floor(x).astype(np.int64), BINS - 2)
    return b, (x - b.astype(np.float32)).astype(np.float32)


def predict_bins(geo: Geometry, v: np.ndarray, table: np.ndarray, W: np.ndarray) -> np.ndarray:
    X, _ = encode(geo, v, table)
    raw, _ = forward(X, layer_weights(W))
    return np.exp(np.minimum(raw, 15.0)).astype(np.float32)


def loss_and_gradients_spectral(geo: Geometry, s: np.ndarray, table: np.ndarray, W: np.ndarray):
    """The four-wavelength loss over samples s (n, 20; targets of wavelengths
    0-2 at 3, 11, 15, of wavelength 3 at 16, hero wavelength at 17; negative
    targets left out): relative L2 of the interpolated bins per wavelength,
    normalised by 4 n, and its gradients (bf16 roundings as the GPU's)."""
    n = len(s)
    X, cw = encode(geo, s[:, :16], table)
    Ws = layer_weights(W)
    raw, acts = forward(X, Ws)
    e = np.exp(np.minimum(raw, 15.0))
    tg = s[:, [3, 11, 15, 16]].astype(np.float32)
    norm = 1.0 / (4.0 * n)
    d = np.zeros((n, OUT))
    loss = 0.0
    for w in range(4):
        b, f = bin_weights(rotate_lambda(s[:, 17], w))
        rows = np.arange(n)
        pred = (1.0 - f) * e[rows, b] + f * e[rows, b + 1]
        ok = tg[:, w] >= 0
        den = pred * pred + 0.01
        diff = pred - tg[:, w]
        loss += float(np.sum(np.where(ok, diff * diff / den, 0.0)) * norm)
        g = np.where(ok, 2.0 * diff / den * norm, 0.0)
        np.add.at(d, (rows, b), g * (1.0 - f) * e[rows, b])
        np.add.at(d, (rows, b + 1), g * f * e[rows, b + 1])
    g = bf16(d.astype(np.float32))
    grads = [None] * LAYERS
    for l in range(LAYERS - 1, -1, -1):
        grads[l] = g.T @ acts[l]
        dIn = g @ Ws[l]
        if l == 0:
            dX = dIn
            break
        g = bf16(np.where(acts[l] > 0, dIn, 0.0).astype(np.float32))
    dW = np.concatenate([gr.reshape(-1) for gr in grads])
    dT = np.zeros((geo.levels * geo.entries, 2), np.float64)
    for l, (idx, w) in enumerate(cw):
        for c in range(8):
            np.add.at(dT, idx[:, c], w[:, c:c + 1].astype(np.float64) * dX[:, 2 * l:2 * l + 2])
    return loss, dT, dW


def loss_and_gradients(geo: Geometry, s: np.ndarray, table: np.ndarray, W: np.ndarray, exact: bool = False,
                       den_fixed: np.ndarray | None = None):
    """Mean relative L2 loss over samples s (n, 16; targets at 3, 11, 15) and its
    gradients w.r.t. the table values (levels * entries, 2) and the packed
    weights.  exact=True: float64 throughout, no bf16 rounding; den_fixed
    replaces the loss denominator (for finite differences of the loss with the
    denominator held constant)."""
    n = len(s)
    X, cw = encode(geo, s, table, exact)
    Ws = layer_weights(W, exact)
    raw, acts = forward(X, Ws, exact)
    tgt = s[:, [3, 11, 15]].astype(np.float64 if exact else np.float32)
    pred = np.exp(np.minimum(raw[:, :3], 15.0))
    den = pred * pred + 0.01 if den_fixed is None else den_fixed
    norm = 1.0 / (3.0 * n)
    loss = float(np.sum((pred - tgt) ** 2 / den) * norm)
    d = 2.0 * (pred - tgt) / den * norm * pred          # d loss / d raw (denominator held)
    dO = np.zeros((n, OUT), d.dtype)
    dO[:, :3] = d if exact else bf16(d.astype(np.float32))
    grads = [None] * LAYERS
    g = dO
    for l in range(LAYERS - 1, -1, -1):
        grads[l] = g.T @ acts[l]
        dIn = g @ Ws[l]
        if l == 0:
            dX = dIn
            break
        g = np.where(acts[l] > 0, dIn, 0.0)
        if not exact:
            g = bf16(g.astype(np.float32))
    dW = np.concatenate([gr.reshape(-1) for gr in grads])
    dT = np.zeros((geo.levels * geo.entries, 2), np.float64)
    for l, (idx, w) in enumerate(cw):
        for c in range(8):
            np.add.at(dT, idx[:, c], w[:, c:c + 1].astype(np.float64) * dX[:, 2 * l:2 * l + 2])
    return loss, dT, dW
