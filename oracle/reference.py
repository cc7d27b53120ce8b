"""ctypes wrapper of oracle/_ref/libref.so: the reference renderer's own
BuildBVH, TraverseBVH, AnyHitSegmentBVH, Intersect, Overlap and BSDF_PDF,
compiled from the reference's headers by `make -C oracle ref`.

TEST INFRASTRUCTURE ONLY: used to generate the golden fixtures under
tests/golden/ and, where the library has been built, to check the oracle
against the reference directly.  Absent on machines without the reference
source; callers test `available()` first.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import c_float, c_int, c_int64, c_size_t, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def load():
    global _lib
    if _lib is not None:
        return _lib
    lib = ctypes.CDLL(LIB)
    lib.ref_scene_create.argtypes = [c_void_p, c_size_t, c_int, c_int]
    lib.ref_scene_create.restype = c_void_p
    lib.ref_scene_destroy.argtypes = [c_void_p]
    lib.ref_scene_node_count.argtypes = [c_void_p]
    lib.ref_scene_node_count.restype = c_int64
    lib.ref_scene_nodes.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.ref_scene_indices.argtypes = [c_void_p, c_void_p]
    lib.ref_scene_light_count.argtypes = [c_void_p]
    lib.ref_scene_light_count.restype = c_int64
    lib.ref_scene_lights.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.ref_trace_rays.argtypes = [c_void_p, c_void_p, c_int64, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_void_p, c_int]
    lib.ref_segments_occluded.argtypes = [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_int]
    lib.ref_overlap.argtypes = [c_void_p, c_void_p, c_int64, c_void_p]
    lib.ref_bsdf_pdf.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.ref_bsdf_pdf.restype = c_float
    lib.ref_object_isect.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_int64, c_int, c_void_p,
                                     c_void_p, c_void_p]
    lib.ref_fill_torus.argtypes = [c_void_p, c_float, c_float, c_void_p]
    lib.ref_spectral_encode.argtypes = [c_void_p, c_void_p, c_int64, c_void_p, c_void_p]
    lib.ref_spectral_sample.argtypes = [c_void_p, c_int64, c_void_p, c_void_p]
    lib.ref_spectral_weights.argtypes = [c_void_p, c_int64, c_void_p, c_void_p]
    lib.ref_spectral_tables.argtypes = [c_void_p]
    lib.ref_tonemap.argtypes = [c_void_p, c_int64, c_int, c_float, c_int, c_void_p]
    lib.ref_intersect_eps.argtypes = [c_int]
    lib.ref_intersect_eps.restype = c_float
    _lib = lib
    return lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


class RefScene:
    """The reference's SceneObject array, BVH (BuildBVH) and light table."""

    def __init__(self, objects: np.ndarray, leaf_size: int = 8, bin_count: int = 12):
        lib = load()
        from aperture_b200 import OBJECT_DTYPE
        self._objs = np.ascontiguousarray(objects, dtype=OBJECT_DTYPE)
        self._h = lib.ref_scene_create(_p(self._objs), len(self._objs), leaf_size, bin_count)

    def __del__(self):
        if getattr(self, "_h", None):
            _lib.ref_scene_destroy(self._h)
            self._h = None

    def nodes(self):
        n = _lib.ref_scene_node_count(self._h)
        b = np.zeros((n, 6), np.float32)
        l = np.zeros((n, 4), np.int32)
        if n:
            _lib.ref_scene_nodes(self._h, _p(b), _p(l))
        return b, l

    def indices(self):
        idx = np.zeros(len(self._objs), np.int32)
        _lib.ref_scene_indices(self._h, _p(idx))
        return idx

    def lights(self):
        n = _lib.ref_scene_light_count(self._h)
        o = np.zeros(n, np.int32)
        p = np.zeros(n, np.float32)
        if n:
            _lib.ref_scene_lights(self._h, _p(o), _p(p))
        return o, p

    def trace(self, rays, any_hit=False, linear=False, threads=0):
        """(hit_object, t, position[n,3], normal[n,3], inside) per ray."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        obj = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        pos = np.empty((n, 3), np.float32)
        nrm = np.empty((n, 3), np.float32)
        ins = np.empty(n, np.int32)
        _lib.ref_trace_rays(self._h, _p(rays), n, int(any_hit), 1 if linear else 0, _p(obj), _p(t), _p(pos), _p(nrm),
                            _p(ins), threads)
        return obj, t, pos, nrm, ins

    def object_isect(self, obj: int, rays, depth: int = 0, grid=None, dims=(0, 0, 0)):
        """IntersectBase of one object (SDF volumes read `grid`): (t or -1, position, normal)."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        t = np.empty(n, np.float32)
        pos = np.empty((n, 3), np.float32)
        nrm = np.empty((n, 3), np.float32)
        g = np.ascontiguousarray(grid, np.float32) if grid is not None else np.zeros(1, np.float32)
        d = np.asarray(dims, np.int32)
        _lib.ref_object_isect(self._h, obj, _p(g), _p(d), _p(rays), n, depth, _p(t), _p(pos), _p(nrm))
        return t, pos, nrm

    def segments_occluded(self, seg6, depth, threads=0):
        seg6 = np.ascontiguousarray(seg6, np.float32).reshape(-1, 6)
        depth = np.ascontiguousarray(depth, np.int32)
        out = np.empty(len(seg6), np.int32)
        _lib.ref_segments_occluded(self._h, _p(seg6), _p(depth), len(seg6), _p(out), threads)
        return out

    def overlap(self, points):
        p = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.empty(len(p), np.int32)
        _lib.ref_overlap(self._h, _p(p), len(p), _p(out))
        return out


def bsdf_pdf(model: int, material, N, ray_dir, L) -> float:
    lib = load()
    f = lambda v: np.ascontiguousarray(v, np.float32)  # noqa: E731
    n, r, l = f(N), f(ray_dir), f(L)
    return lib.ref_bsdf_pdf(model, ctypes.addressof(material), _p(n), _p(r), _p(l))


def intersect_eps(depth: int) -> float:
    return load().ref_intersect_eps(depth)


def tonemap(rgb: np.ndarray, tone: int, exposure: float = 1.0, xyz_input: bool = False) -> np.ndarray:
    rgb = np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)
    out = np.empty(len(rgb), np.uint32)
    load().ref_tonemap(_p(rgb), len(rgb), tone, exposure, int(xyz_input), _p(out))
    return out


def fill_torus(dims, R: float, r: float) -> np.ndarray:
    d = np.asarray(dims, np.int32)
    out = np.empty(int(np.prod(dims)), np.float32)
    load().ref_fill_torus(_p(d), R, r, _p(out))
    return out


def spectral_encode(rgb=None, lam=None):
    n = len(rgb) if rgb is not None else len(lam)
    r = np.ascontiguousarray(rgb, np.float32) if rgb is not None else None
    l_ = np.ascontiguousarray(lam, np.float32) if lam is not None else None
    rk = np.empty((n, 4), np.float32) if r is not None else None
    lk = np.empty((n, 4), np.float32) if l_ is not None else None
    load().ref_spectral_encode(_p(r) if r is not None else None, _p(l_) if l_ is not None else None, n,
                               _p(rk) if rk is not None else None, _p(lk) if lk is not None else None)
    return rk, lk


def spectral_sample(u3):
    u3 = np.ascontiguousarray(u3, np.float32).reshape(-1, 3)
    lam, pdf = np.empty(len(u3), np.float32), np.empty(len(u3), np.float32)
    load().ref_spectral_sample(_p(u3), len(u3), _p(lam), _p(pdf))
    return lam, pdf


def spectral_weights(lam):
    lam = np.ascontiguousarray(lam, np.float32)
    d65, xyz = np.empty(lam.size, np.float32), np.empty((lam.size, 3), np.float32)
    load().ref_spectral_weights(_p(lam), lam.size, _p(d65), _p(xyz))
    return d65, xyz


def spectral_tables() -> np.ndarray:
    out = np.empty(17780, np.float32)
    load().ref_spectral_tables(_p(out))
    return out
