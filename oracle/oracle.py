"""ctypes wrapper of liboracle.so, the CPU restatement of the reference hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, as the checker.  The input format is
the public ar_object_desc (aperture_b200.OBJECT_DTYPE).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_float, c_int, c_int32, c_int64, c_size_t, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

PROXY_OBJECT_CENTER = 1
TRIANGLE_DEFAULT_GBUFFER = 2
TRIANGLE_SOLO_MEDIA = 4
REFERENCE_TRAVERSAL = 8
TIE_FIRST_FOUND, TIE_LOWEST_INDEX, SLAB_REFERENCE, SLAB_STANDARD = 0, 1, 0, 2

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    lib.or_scene_create.argtypes = [c_void_p, c_size_t, c_int, c_int, c_int]
    lib.or_scene_create.restype = c_void_p
    lib.or_scene_create_ex.argtypes = [c_void_p, c_size_t, c_void_p, c_size_t, c_int, c_int, c_int]
    lib.or_scene_create_ex.restype = c_void_p
    lib.or_scene_destroy.argtypes = [c_void_p]
    lib.or_scene_node_count.argtypes = [c_void_p]
    lib.or_scene_node_count.restype = c_int64
    lib.or_scene_nodes.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.or_scene_indices.argtypes = [c_void_p, c_void_p]
    lib.or_scene_light_count.argtypes = [c_void_p]
    lib.or_scene_light_count.restype = c_int64
    lib.or_scene_lights.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.or_trace_rays.argtypes = [c_void_p, c_void_p, c_int64, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                  c_int]
    lib.or_trace_rays_brute.argtypes = [c_void_p, c_void_p, c_int64, c_int, c_void_p, c_void_p, c_int]
    lib.or_camera_ray.argtypes = [c_void_p, c_int, c_int, c_float, c_float, c_void_p]
    lib.or_render_paths.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int]
    lib.or_render_paths.restype = c_int64
    lib.or_render_image.argtypes = [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64, c_void_p,
                                    POINTER(c_int64), POINTER(c_int64), c_int]
    lib.or_dn_record.argtypes = [c_void_p, c_void_p, c_int64, c_void_p, c_void_p]
    lib.or_dn_bilateral.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p]
    for f in ("or_sinf", "or_cosf", "or_expf", "or_logf"):
        getattr(lib, f).argtypes = [c_float]
        getattr(lib, f).restype = c_float
    lib.or_collect_rays.argtypes = [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_int64,
                                    POINTER(c_int64), c_void_p, c_int64, POINTER(c_int64)]
    lib.or_collect_rays.restype = c_int64
    lib.or_powf.argtypes = [c_float, c_float]
    lib.or_powf.restype = c_float
    lib.or_object_isect.argtypes = [c_void_p, c_int32, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p]
    lib.or_volume_grid.argtypes = [c_void_p, c_int32, c_void_p]
    lib.or_scene_set_spectral.argtypes = [c_void_p, c_void_p, c_size_t, c_int, c_int]
    lib.or_scene_set_spectral.restype = c_int
    lib.or_spectral_luts.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.or_spectral_sample.argtypes = [c_void_p, c_int64, c_void_p, c_void_p]
    lib.or_spectral_encode.argtypes = [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p]
    lib.or_spectral_interact.argtypes = [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p]
    lib.or_tonemap.argtypes = [c_void_p, c_int64, c_int, c_float, c_int, c_void_p]
    lib.or_trace_detail.argtypes = [c_void_p, c_void_p, c_int64, c_int] + [c_void_p] * 5 + [c_int]
    lib.or_segments_occluded.argtypes = [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_void_p, c_int]
    lib.or_overlap.argtypes = [c_void_p, c_void_p, c_int64, c_void_p]
    lib.or_bsdf_pdf.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.or_bsdf_pdf.restype = c_float
    lib.or_power_heuristic.argtypes = [c_float, c_float]
    lib.or_scene_set_medium.argtypes = [c_void_p, c_void_p]
    lib.or_scene_set_medium.restype = c_int
    lib.or_medium_density.argtypes = [c_void_p, c_void_p]
    lib.or_medium_density.restype = c_float
    lib.or_hg_sample.argtypes = [c_void_p, c_float, c_void_p, c_int64, c_void_p]
    lib.or_hg_phase.argtypes = [c_float, c_float]
    lib.or_hg_phase.restype = c_float
    lib.or_medium_track.argtypes = [c_void_p, c_void_p, c_int64, c_void_p, c_int, c_void_p]
    lib.or_power_heuristic.restype = c_float
    _lib = lib
    return lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


class OracleScene:
    def __init__(self, objects: np.ndarray, flags: int = 0, leaf_size: int = 8, bin_count: int = 12, volumes=None):
        """volumes: list of (SdfVolume, keep-alive) from aperture_b200.make_volume()."""
        lib = load()
        from aperture_b200 import OBJECT_DTYPE, SdfVolume
        self._objs = np.ascontiguousarray(objects, dtype=OBJECT_DTYPE)
        self._vols = volumes
        arr = (SdfVolume * len(volumes))(*[v for v, _ in volumes]) if volumes else None
        self._h = lib.or_scene_create_ex(_p(self._objs) if len(self._objs) else None, len(self._objs), arr,
                                         len(volumes) if volumes else 0, flags, leaf_size, bin_count)

    def __del__(self):
        if getattr(self, "_h", None):
            _lib.or_scene_destroy(self._h)
            self._h = None

    def nodes(self):
        n = _lib.or_scene_node_count(self._h)
        b = np.zeros((n, 6), np.float32)
        l = np.zeros((n, 4), np.int32)
        if n:
            _lib.or_scene_nodes(self._h, _p(b), _p(l))
        return b, l

    def indices(self):
        idx = np.zeros(len(self._objs), np.int32)
        if len(idx):
            _lib.or_scene_indices(self._h, _p(idx))
        return idx

    def lights(self):
        n = _lib.or_scene_light_count(self._h)
        o = np.zeros(n, np.int32)
        p = np.zeros(n, np.float32)
        if n:
            _lib.or_scene_lights(self._h, _p(o), _p(p))
        return o, p

    def trace(self, rays, any_hit=False, mode=TIE_LOWEST_INDEX | SLAB_STANDARD, threads=0, counters=False):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        obj = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        nv = np.empty(n, np.int32) if counters else None
        pt = np.empty(n, np.int32) if counters else None
        _lib.or_trace_rays(self._h, _p(rays), n, int(any_hit), mode, _p(obj), _p(t), _p(nv) if counters else None,
                           _p(pt) if counters else None, threads)
        if counters:
            return obj, t, nv, pt
        return obj, t

    def trace_detail(self, rays, mode=TIE_LOWEST_INDEX | SLAB_STANDARD, threads=0):
        """Closest hit with position, normal and inside flag:
        (hit_object, t, position[n,3], normal[n,3], inside)."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        obj = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        pos = np.empty((n, 3), np.float32)
        nrm = np.empty((n, 3), np.float32)
        ins = np.empty(n, np.int32)
        _lib.or_trace_detail(self._h, _p(rays), n, mode, _p(obj), _p(t), _p(pos), _p(nrm), _p(ins), threads)
        return obj, t, pos, nrm, ins

    def segments_occluded(self, seg6, depth, mode=TIE_LOWEST_INDEX | SLAB_STANDARD, threads=0):
        """AnyHitSegmentBVH of src.xyz -> dst.xyz segments at the given loop depths."""
        seg6 = np.ascontiguousarray(seg6, np.float32).reshape(-1, 6)
        depth = np.ascontiguousarray(depth, np.int32)
        out = np.empty(len(seg6), np.int32)
        _lib.or_segments_occluded(self._h, _p(seg6), _p(depth), len(seg6), mode, _p(out), threads)
        return out

    def overlap(self, points):
        p = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.empty(len(p), np.int32)
        _lib.or_overlap(self._h, _p(p), len(p), _p(out))
        return out

    def object_isect(self, obj: int, rays, depth: int = 0):
        """(t or -1, position[n,3], normal[n,3]) of one object for each ray at loop depth `depth`."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        t = np.empty(n, np.float32)
        pos = np.empty((n, 3), np.float32)
        nrm = np.empty((n, 3), np.float32)
        _lib.or_object_isect(self._h, obj, _p(rays), n, depth, _p(t), _p(pos), _p(nrm))
        return t, pos, nrm

    def volume_grid(self, v: int, dims) -> np.ndarray:
        out = np.zeros(int(np.prod(dims)), np.float32)
        _lib.or_volume_grid(self._h, v, _p(out))
        return out

    def set_spectral(self, tables: np.ndarray, res: int = 64, threads: int = 0) -> None:
        t = np.ascontiguousarray(tables, np.float32)
        if _lib.or_scene_set_spectral(self._h, _p(t), t.size, res, threads) != 0:
            raise ValueError("bad spectral tables or resolution")
        self.spec_res = res

    def set_medium(self, density, bounds_min=None, bounds_max=None, sigma_t_max=0.0, albedo=None, g=0.0) -> None:
        """The participating medium of Scene.set_medium (same arguments)."""
        from aperture_b200 import medium_desc
        if density is None:
            _lib.or_scene_set_medium(self._h, None)
            return
        d = np.ascontiguousarray(density)
        m = medium_desc(d, bounds_min, bounds_max, sigma_t_max, albedo, g)
        _lib.or_scene_set_medium(self._h, ctypes.byref(m))

    def medium_density(self, p3) -> float:
        p = np.ascontiguousarray(p3, np.float32)
        return float(_lib.or_medium_density(self._h, _p(p)))

    def medium_track(self, rays, seeds, ratio: bool = False) -> np.ndarray:
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        sd = np.ascontiguousarray(seeds, np.uint32)
        out = np.zeros(len(r), np.float32)
        _lib.or_medium_track(self._h, _p(r), len(r), _p(sd), 1 if ratio else 0, _p(out))
        return out

    def spectral_luts(self):
        lam = np.zeros((840, 4), np.float32)
        rgb = np.zeros((self.spec_res ** 3, 4), np.float32)
        _lib.or_spectral_luts(self._h, _p(lam), _p(rgb))
        return lam, rgb

    def spectral_interact(self, lam, rgb):
        """(Interact response, D65Norm, CMF xyz[n,3]) at wavelengths lam for colours rgb[n,3]."""
        lam = np.ascontiguousarray(lam, np.float32)
        rgb = np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)
        n = lam.size
        resp, d65, xyz = np.empty(n, np.float32), np.empty(n, np.float32), np.empty((n, 3), np.float32)
        _lib.or_spectral_interact(self._h, _p(lam), _p(rgb), n, _p(resp), _p(d65), _p(xyz))
        return resp, d65, xyz

    def trace_brute(self, rays, any_hit=False, threads=0):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        obj = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        _lib.or_trace_rays_brute(self._h, _p(rays), n, int(any_hit), _p(obj), _p(t), threads)
        return obj, t

    def render_paths(self, camera, params, tape: np.ndarray, threads=0):
        from aperture_b200 import RECORD_DTYPE
        tape = np.ascontiguousarray(tape, np.float32)
        n = camera.width * camera.height * params.spp
        assert tape.shape[0] == n
        rec = np.zeros(n, RECORD_DTYPE)
        over = _lib.or_render_paths(self._h, ctypes.byref(camera), ctypes.byref(params), _p(tape), tape.shape[1],
                                    _p(rec), threads)
        return rec, over

    def render_image(self, camera, params, pixel_begin=0, pixel_end=None, step=1, threads=0):
        """FP64 sums of pixels pixel_begin, +step, ... (others stay zero), query counts."""
        npix = camera.width * camera.height
        if pixel_end is None:
            pixel_end = npix
        acc = np.zeros((npix, 3), np.float64)
        e, s = c_int64(0), c_int64(0)
        _lib.or_render_image(self._h, ctypes.byref(camera), ctypes.byref(params), pixel_begin, pixel_end, step,
                             _p(acc), ctypes.byref(e), ctypes.byref(s), threads)
        return acc, e.value, s.value


def collect_rays(scene: "OracleScene", camera, params, pixel_begin, pixel_end, cap=2_000_000):
    """Extension and shadow queries of the CPU path loop over a pixel range."""
    ext = np.zeros((cap, 8), np.float32)
    sh = np.zeros((cap, 8), np.float32)
    ne, ns = c_int64(0), c_int64(0)
    _lib.or_collect_rays(scene._h, ctypes.byref(camera), ctypes.byref(params), pixel_begin, pixel_end, _p(ext), cap,
                         ctypes.byref(ne), _p(sh), cap, ctypes.byref(ns))
    return ext[:ne.value].copy(), sh[:ns.value].copy()


def camera_ray(camera, i, j, jx, jy) -> np.ndarray:
    lib = load()
    r = np.zeros(8, np.float32)
    lib.or_camera_ray(ctypes.byref(camera), i, j, jx, jy, _p(r))
    return r


def bsdf_pdf(model: int, material, N, ray_dir, L) -> float:
    """BSDF_PDF (RGB) of the restatement for one ar_material (ctypes struct)."""
    lib = load()
    f = lambda v: np.ascontiguousarray(v, np.float32)  # noqa: E731
    n, r, l = f(N), f(ray_dir), f(L)
    return lib.or_bsdf_pdf(model, ctypes.addressof(material), _p(n), _p(r), _p(l))


def power_heuristic(a: float, b: float) -> float:
    return load().or_power_heuristic(a, b)


def tonemap(rgb: np.ndarray, tone: int, exposure: float = 1.0, xyz_input: bool = False) -> np.ndarray:
    """The Tonemap kernel's output (0xAARRGGBB per pixel) for linear rgb[n, 3]."""
    rgb = np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)
    out = np.empty(len(rgb), np.uint32)
    load().or_tonemap(_p(rgb), len(rgb), tone, exposure, int(xyz_input), _p(out))
    return out


def spectral_sample(u3: np.ndarray):
    """SampleCIE1931 for uniforms u3[n, 3]: (lambda, pdf)."""
    u3 = np.ascontiguousarray(u3, np.float32).reshape(-1, 3)
    lam, pdf = np.empty(len(u3), np.float32), np.empty(len(u3), np.float32)
    load().or_spectral_sample(_p(u3), len(u3), _p(lam), _p(pdf))
    return lam, pdf


def spectral_encode(tables: np.ndarray, rgb=None, lam=None):
    """(RGBEncode kernels [n,4] or None, LambdaEncode kernels [n,4] or None)."""
    t = np.ascontiguousarray(tables, np.float32)
    n = len(rgb) if rgb is not None else len(lam)
    rk = np.empty((n, 4), np.float32) if rgb is not None else None
    lk = np.empty((n, 4), np.float32) if lam is not None else None
    r = np.ascontiguousarray(rgb, np.float32) if rgb is not None else None
    l_ = np.ascontiguousarray(lam, np.float32) if lam is not None else None
    load().or_spectral_encode(_p(t), _p(r) if r is not None else None, _p(l_) if l_ is not None else None, n,
                              _p(rk) if rk is not None else None, _p(lk) if lk is not None else None)
    return rk, lk


def hg_sample(d, g: float, u2) -> np.ndarray:
    """Henyey-Greenstein directions around d for an [n, 2] array of uniforms."""
    dd = np.ascontiguousarray(d, np.float32)
    u = np.ascontiguousarray(u2, np.float32).reshape(-1, 2)
    out = np.zeros((len(u), 3), np.float32)
    load().or_hg_sample(_p(dd), g, _p(u), len(u), _p(out))
    return out


def hg_phase(g: float, cos_t: float) -> float:
    return float(load().or_hg_phase(g, cos_t))


def dn_record(hits: np.ndarray | None, samples: np.ndarray | None, gbuffer: np.ndarray | None,
              stats: np.ndarray | None) -> None:
    """Records one frame into the denoiser buffers in place (numpy record arrays
    of 48-byte ar_screen_gbuffer / ar_screen_stats): RecordScreenGBuffer and
    RecordScreenStatisticBuffer (core/denoise/)."""
    lib = load()
    n = len(gbuffer) if gbuffer is not None else len(stats)
    h = np.ascontiguousarray(hits, np.float32) if hits is not None else None
    sm = np.ascontiguousarray(samples, np.float32) if samples is not None else None
    lib.or_dn_record(_p(h) if h is not None else None, _p(sm) if sm is not None else None, n,
                     _p(gbuffer) if gbuffer is not None else None, _p(stats) if stats is not None else None)


def dn_bilateral(hdr: np.ndarray, gbuffer: np.ndarray, stats: np.ndarray, width: int, height: int,
                 t_quantiles: np.ndarray) -> np.ndarray:
    """Bilateral16x16<7> of core/denoise/denoise.cuh over a whole image."""
    lib = load()
    hdr = np.ascontiguousarray(hdr, np.float32).reshape(-1)
    out = np.empty_like(hdr)
    tq = np.ascontiguousarray(t_quantiles, np.float32)
    lib.or_dn_bilateral(_p(hdr), _p(out), _p(gbuffer), _p(stats), width, height, _p(tq))
    return out
