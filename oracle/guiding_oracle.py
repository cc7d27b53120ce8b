"""CPU restatement of the path-guiding probe math -- TEST INFRASTRUCTURE ONLY.

Only tests/ import this module; it checks the CUDA probes of
aperturerendererv3-optix-geometry_b200/csrc/guiding.cuh and is never on the
product path.  It restates, in numpy:
  * the equal-area octahedral map of the unit square onto the sphere and its
    inverse (Clarberg, "Fast equal-area mapping of the (hemi)sphere using
    SIMD", JGT 2008), the map the reference's probes use
    (core/guiding/octahedron.cuh, PATH_GUIDING_CLARBERG);
  * a probe's mip chain (8x8 -> 4x4 -> 2x2 -> 1x1 averages, leaves clamped to
    1e-5), its density pdf(w) = (w_leaf / w_avg) / (4 pi) with texel weights
    dot(rgb, query), the hemisphere density pdf(w) + pdf(mirror(w)), and the
    mip-descent sampler (children in (x, y) order (0,0) (0,1) (1,0) (1,1)).
Pinned to the mathematics it restates: equal area (uniform square samples are
uniform on the sphere), the round trip, and sampler = density
(tests/test_cpu_guiding.py); the GPU's probes are compared with this file in
tests/test_gpu_guiding.py.
"""
from __future__ import annotations

import math

import numpy as np

RES = 8
OFFSETS = (0, 64, 80, 84)


def uv_to_dir(su, sv):
    u = 2.0 * np.asarray(su, np.float64) - 1.0
    v = 2.0 * np.asarray(sv, np.float64) - 1.0
    au, av = np.abs(u), np.abs(v)
    d = 1.0 - (au + av)
    r = 1.0 - np.abs(d)
    with np.errstate(divide="ignore", invalid="ignore"):
        phi = np.where(r > 0, ((av - au) / np.where(r > 0, r, 1.0) + 1.0) * (math.pi / 4), 0.0)
    z = np.copysign(1.0 - r * r, d)
    s = r * np.sqrt(np.maximum(0.0, 2.0 - r * r))
    return np.stack([np.copysign(np.cos(phi) * s, u), np.copysign(np.sin(phi) * s, v), z], -1)


def dir_to_uv(w):
    w = np.asarray(w, np.float64)
    r = np.sqrt(np.maximum(0.0, 1.0 - np.abs(w[..., 2])))
    psi = np.arctan2(np.abs(w[..., 1]), np.abs(w[..., 0])) * (2.0 / math.pi)
    v = psi * r
    u = r - v
    neg = w[..., 2] < 0
    u, v = np.where(neg, 1.0 - v, u), np.where(neg, 1.0 - u, v)
    u = np.copysign(u, w[..., 0])
    v = np.copysign(v, w[..., 1])
    return np.clip(0.5 * (u + 1.0), 0, 1), np.clip(0.5 * (v + 1.0), 0, 1)


def build_mips(leaves_rgb: np.ndarray) -> np.ndarray:
    """(64, 3) leaf radiance -> (85, 3) texels: clamped leaves then mips."""
    t = np.zeros((85, 3))
    t[:64] = np.maximum(leaves_rgb.reshape(64, 3), 1e-5)
    src, res = t[:64].reshape(RES, RES, 3), RES
    for level in range(1, 4):
        res //= 2
        m = 0.25 * (src[0::2, 0::2] + src[0::2, 1::2] + src[1::2, 0::2] + src[1::2, 1::2])
        t[OFFSETS[level]:OFFSETS[level] + res * res] = m.reshape(-1, 3)
        src = m
    return t


def pdf(texels: np.ndarray, w: np.ndarray, q) -> np.ndarray:
    su, sv = dir_to_uv(w)
    ix = np.clip(np.floor(su * RES).astype(int), 0, RES - 1)
    iy = np.clip(np.floor(sv * RES).astype(int), 0, RES - 1)
    q = np.asarray(q, np.float64)
    wl = texels[iy * RES + ix] @ q
    wa = texels[84] @ q
    return np.maximum(wl / wa / (4 * math.pi), 1e-12)


def mirror(w, n):
    return w - 2.0 * (w @ n)[..., None] * n


def hemi_pdf(texels, w, n, q):
    p = pdf(texels, w, q) + pdf(texels, mirror(w, n), q)
    return np.where(w @ n > 0, p, 0.0)


def sample_leaf(texels: np.ndarray, q, u3) -> tuple[int, int, float]:
    """Mip descent with three uniforms: leaf (x, y) and its probability."""
    q = np.asarray(q, np.float64)
    cx = cy = 0
    pt = 1.0
    for level in (3, 2, 1):
        res = RES >> level
        total = 4.0 * (texels[OFFSETS[level] + cy * res + cx] @ q)
        nx, ny = cx * 2, cy * 2
        cres = RES >> (level - 1)
        r = u3[3 - level]
        cdf = 0.0
        for c in range(4):
            ox, oy = c >> 1, c & 1
            wc = (texels[OFFSETS[level - 1] + (ny + oy) * cres + nx + ox] @ q) / total
            cdf += wc
            if r <= cdf or c == 3:
                cx, cy = nx + ox, ny + oy
                pt *= wc
                break
    return cx, cy, pt


# The reference's face numbering (FaceNormal20FromIndex, core/guiding/
# guiding_bin.cuh:40-66) as the signs of each face normal's x, y, z: three
# non-zero signs are a cube-diagonal face (+-1, +-1, +-1) / sqrt 3; a zero at
# axis k puts phi^2 / sqrt(1 + phi^4) on axis (k + 1) % 3 and 1 / sqrt(1 + phi^4)
# on axis (k + 2) % 3 (the table of csrc/guiding.cu, pg_face_normals).
FACE_SIGNS = ((-1, 1, 1), (0, 1, 1), (0, 1, -1), (-1, 1, -1), (-1, 1, 0), (1, 1, 1), (-1, 0, 1), (-1, -1, 0),
              (-1, 0, -1), (1, 1, -1), (1, -1, 1), (0, -1, 1), (0, -1, -1), (1, -1, -1), (1, -1, 0), (1, 0, 1),
              (-1, -1, 1), (-1, -1, -1), (1, 0, -1), (1, 1, 0))


def face_normals() -> np.ndarray:
    phi = (1.0 + math.sqrt(5.0)) / 2.0
    ln = math.sqrt(1.0 + phi ** 4)
    out = np.zeros((20, 3))
    for f, s in enumerate(FACE_SIGNS):
        if 0 not in s:
            out[f] = np.array(s) / math.sqrt(3.0)
        else:
            k = s.index(0)
            out[f, (k + 1) % 3] = s[(k + 1) % 3] * phi * phi / ln
            out[f, (k + 2) % 3] = s[(k + 2) % 3] / ln
    return out.astype(np.float32)


def voxel_grid(pos, dirs) -> np.ndarray:
    """(voxel x, y, z of 0.05 units, face whose normal is nearest the direction)"""
    p = np.asarray(pos, np.float32)
    d = np.asarray(dirs, np.float64)
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    face = np.argmax(d @ face_normals().astype(np.float64).T, axis=1)
    g = np.floor(p * np.float32(20.0)).astype(np.int64)
    return np.concatenate([g, face[:, None]], axis=1)


def sample_hemi(texels: np.ndarray, n, q, u5):
    """SampleOctahedronHemisphere: mip descent with u5[0:3], the point in the
    leaf texel from 1 - u5[3:5], the mirror about the normal for directions
    below it; pdf = leaf pdf + pdf of the mirror direction."""
    n = np.asarray(n, np.float64)
    cx, cy, pt = sample_leaf(texels, q, u5[:3])
    su = min(max((cx + (1.0 - u5[3])) / RES, 0.0), 1.0)
    sv = min(max((cy + (1.0 - u5[4])) / RES, 0.0), 1.0)
    w = uv_to_dir(su, sv)
    p = max(pt * RES * RES / (4 * math.pi), 1e-12)
    m = mirror(w, n)
    p += float(pdf(texels, m[None], q)[0])
    if w @ n < 0:
        w = m
    return w, p
