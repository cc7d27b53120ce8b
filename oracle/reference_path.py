"""ctypes wrapper of oracle/_ref/libref_path.so and libref_path_detmath.so:
the reference renderer's own path loop (CalculateRadiance,
core/render/render.cuh:460-999, and everything it calls) run on the host from
the build-time copy `make -C oracle ref-path` compiles (see
oracle/ref_path_patch.py for the edits and oracle/ref_path_harness.cu for the
driver).

TEST INFRASTRUCTURE ONLY: used to generate golden fixtures, to pin the oracle's
path loop against the reference's and as the timed CPU baseline of bench.py.
`detmath=True` selects the build whose transcendental functions are the
oracle's fixed definitions; the default build uses the host math library.
Absent where the reference sources were not present at build time; callers
test `available()` first.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_int, c_int64, c_size_t, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBS = {False: os.path.join(HERE, "_ref", "libref_path.so"),
        True: os.path.join(HERE, "_ref", "libref_path_detmath.so")}

_libs = {}

# The reference's defaults for the BVH of its scenes (BuildBVH leaf size and bins).
LEAF_SIZE, BIN_COUNT = 8, 12


def available(detmath: bool = False) -> bool:
    return os.path.exists(LIBS[detmath])


def load(detmath: bool = False):
    if detmath in _libs:
        return _libs[detmath]
    lib = ctypes.CDLL(LIBS[detmath])
    lib.refp_scene_create.argtypes = [c_void_p, c_size_t, c_int, c_int]
    lib.refp_scene_create.restype = c_void_p
    lib.refp_scene_destroy.argtypes = [c_void_p]
    lib.refp_detmath.restype = c_int
    lib.refp_render_paths.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int]
    lib.refp_render_paths.restype = c_int64
    lib.refp_render_image.argtypes = [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64, c_void_p,
                                      POINTER(c_int64), POINTER(c_int64), c_int]
    lib.refp_render_image.restype = c_int
    assert lib.refp_detmath() == int(detmath)
    _libs[detmath] = lib
    return lib


class RefPathScene:
    """A scene for the reference's path loop: the reference's SceneObjects,
    BuildBVH and light table (oracle/ref_scene_common.h)."""

    def __init__(self, objects: np.ndarray, detmath: bool = False, leaf_size: int = LEAF_SIZE,
                 bin_count: int = BIN_COUNT):
        from aperture_b200 import OBJECT_DTYPE
        self._lib = load(detmath)
        self._objs = np.ascontiguousarray(objects, dtype=OBJECT_DTYPE)
        self._h = self._lib.refp_scene_create(self._objs.ctypes.data, len(self._objs), leaf_size, bin_count)

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.refp_scene_destroy(self._h)
            self._h = None

    def render_paths(self, camera, params, tape: np.ndarray, threads: int = 0):
        """One ar_path_record per path (sample major) from uniforms read off
        `tape` (ar_rng_tape layout).  Returns (records, paths out of tape)."""
        from aperture_b200 import RECORD_DTYPE
        tape = np.ascontiguousarray(tape, np.float32)
        n = camera.width * camera.height * params.spp
        rec = np.zeros(n, RECORD_DTYPE)
        overflow = self._lib.refp_render_paths(self._h, ctypes.byref(camera), ctypes.byref(params),
                                               tape.ctypes.data, tape.shape[1], rec.ctypes.data, threads)
        if overflow < 0:
            raise ValueError("parameters the reference's RGB path loop cannot express "
                             "(rr_depth must be 3, sky 1, spectral 0, tri_light_nee 0)")
        return rec, int(overflow)

    def render_image(self, camera, params, pixel_begin: int = 0, pixel_end: int | None = None, step: int = 1,
                     threads: int = 0, accum: np.ndarray | None = None):
        """FP64 sums of spp samples of pixels pixel_begin, +step, ... < pixel_end
        from the harness's own generator; returns (accum, closest-hit queries,
        shadow queries)."""
        if pixel_end is None:
            pixel_end = camera.width * camera.height
        if accum is None:
            accum = np.zeros((camera.height * camera.width * 3,), np.float64)
        e, s = c_int64(0), c_int64(0)
        st = self._lib.refp_render_image(self._h, ctypes.byref(camera), ctypes.byref(params), pixel_begin, pixel_end,
                                         step, accum.ctypes.data, ctypes.byref(e), ctypes.byref(s), threads)
        if st != 0:
            raise ValueError("parameters the reference's RGB path loop cannot express")
        return accum, e.value, s.value


def guiding_faces() -> np.ndarray:
    """The reference's 20 face normals in its numbering (FaceNormal20FromIndex)."""
    lib = load(False)
    lib.refp_guiding_faces.argtypes = [c_void_p]
    out = np.empty((20, 3), np.float32)
    lib.refp_guiding_faces(out.ctypes.data)
    return out


def guiding_voxel(pos, dirs) -> np.ndarray:
    """pg::GetVoxelGrid per point and direction: int32 [n, 4] (x, y, z, face)."""
    lib = load(False)
    lib.refp_guiding_voxel.argtypes = [c_void_p, c_void_p, c_int64, c_void_p]
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
    out = np.empty((len(p), 4), np.int32)
    lib.refp_guiding_voxel(p.ctypes.data, d.ctypes.data, len(p), out.ctypes.data)
    return out


def guiding_sample(texels, probe_of, normal, query, u5, eval_dir):
    """Octahedron::SampleOctahedronHemisphere (uniforms from u5) and
    OctahedronHemispherePDF of eval_dir for probes given as texels
    [nprobes, 85, 4]: (directions [n, 3], sample pdfs, pdfs of eval_dir)."""
    lib = load(False)
    lib.refp_guiding_sample.argtypes = [c_void_p, c_int] + [c_void_p] * 5 + [c_int64] + [c_void_p] * 3
    t = np.ascontiguousarray(texels, np.float32).reshape(-1, 85, 4)
    po = np.ascontiguousarray(probe_of, np.int32).reshape(-1)
    n = len(po)
    a = [np.ascontiguousarray(x, np.float32).reshape(n, -1) for x in (normal, query, u5, eval_dir)]
    d = np.empty((n, 3), np.float32)
    p = np.empty(n, np.float32)
    e = np.empty(n, np.float32)
    lib.refp_guiding_sample(t.ctypes.data, len(t), po.ctypes.data, a[0].ctypes.data, a[1].ctypes.data,
                            a[2].ctypes.data, a[3].ctypes.data, n, d.ctypes.data, p.ctypes.data, e.ctypes.data)
    return d, p, e
