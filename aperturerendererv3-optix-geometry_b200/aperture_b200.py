"""Python binding of the C ABI in include/aperture_b200.h (ctypes).

The shipped product is libaperture_b200.so; this module only marshals
arguments.  It never falls back to CPU code: if the shared library is missing
or no CUDA device is visible the calls raise.

Layouts mirror the C structs field by field; `OBJECT_DTYPE` is the numpy view
of ar_object_desc used to build large scenes without per-object Python work.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int32, c_int64, c_size_t, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("AR_LIBRARY") or os.path.join(HERE, "libaperture_b200.so")   # AR_LIBRARY: another build

AR_OK = 0
STATUS_NAMES = {0: "AR_OK", 1: "AR_ERR_INVALID_ARGUMENT", 2: "AR_ERR_CUDA", 3: "AR_ERR_OUT_OF_MEMORY",
                4: "AR_ERR_UNSUPPORTED", 5: "AR_ERR_DEVICE_FAULT", 6: "AR_ERR_NO_DEVICE",
                7: "AR_ERR_INTERNAL"}
OBJ_CUBE, OBJ_SPHERE, OBJ_SDF, OBJ_TRIANGLE = 0, 1, 2, 3
MAT_DIFFUSE, MAT_LIGHT, MAT_GLASS, MAT_GGX = 0, 1, 2, 3
MEM_HOST, MEM_DEVICE = 0, 1
DEBUG_MAX_HITS = 16
REFERENCE_SEED = 0x9E3779B97F4A7C15


class Vec3(ctypes.Structure):
    _fields_ = [("x", c_float), ("y", c_float), ("z", c_float)]


class Material(ctypes.Structure):
    _fields_ = [("shading_model", c_int32), ("albedo", Vec3), ("emissive", Vec3), ("specular", c_float),
                ("metallic", c_float), ("roughness", c_float), ("ior", c_float), ("sigma_a", c_float),
                ("abbe_number", c_float), ("tilt_number", c_float)]


class Vertex(ctypes.Structure):
    _fields_ = [("position", Vec3), ("normal", Vec3), ("u", c_float), ("v", c_float)]


class SdfParams(ctypes.Structure):
    _fields_ = [("info", c_float * 4), ("kind", c_int32), ("volume", c_int32)]


class ObjectDesc(ctypes.Structure):
    """ar_object_desc; `tri` (triangles) and `sdf` (SDF objects) share storage."""
    _fields_ = [("type", c_int32), ("center", Vec3), ("extent", Vec3), ("rotation_deg", Vec3),
                ("material", Material), ("tri", Vertex * 3), ("visible", c_int32), ("reserved", c_int32 * 3)]


class SdfVolume(ctypes.Structure):
    _fields_ = [("dims", c_int32 * 3), ("precision", c_int32), ("data", c_void_p), ("fill_kind", c_int32),
                ("fill_info", c_float * 4), ("reserved", c_int32)]


class MediumDesc(ctypes.Structure):
    """ar_medium_desc: a box of heterogeneous participating medium."""
    _fields_ = [("bounds_min", c_float * 3), ("bounds_max", c_float * 3), ("sigma_t_max", c_float),
                ("albedo", c_float * 3), ("g", c_float), ("dims", c_int32 * 3), ("precision", c_int32),
                ("density", c_void_p)]


SDF_TORUS, SDF_VOLUME = 0, 1
SDF_OFFSET = ObjectDesc.tri.offset   # ar_object_desc.sdf overlays tri[0]


def set_sdf(obj, kind: int, info=(0.0, 0.0, 0.0, 0.0), volume: int = 0) -> None:
    """Fill the sdf member of one ar_object_desc record (numpy structured scalar
    or array element view) -- it shares storage with tri[0]."""
    raw = obj.view(np.uint8) if isinstance(obj, np.ndarray) else None
    assert raw is not None, "pass a 1-element OBJECT_DTYPE array view"
    p = SdfParams()
    p.info[:] = [float(x) for x in info]
    p.kind, p.volume = kind, volume
    raw[SDF_OFFSET:SDF_OFFSET + ctypes.sizeof(SdfParams)] = np.frombuffer(bytes(p), np.uint8)


def get_sdf(obj) -> SdfParams:
    raw = obj.view(np.uint8)
    return SdfParams.from_buffer_copy(raw[SDF_OFFSET:SDF_OFFSET + ctypes.sizeof(SdfParams)].tobytes())


class Camera(ctypes.Structure):
    _fields_ = [("position", Vec3), ("direction", Vec3), ("fov_y_deg", c_float), ("width", c_int32),
                ("height", c_int32)]


class RenderParams(ctypes.Structure):
    _fields_ = [("spp", c_int32), ("max_depth", c_int32), ("rr_depth", c_int32), ("use_nee", c_int32),
                ("sky", c_int32), ("frame_offset", c_int32), ("seed", c_uint64), ("sort_rays", c_int32),
                ("wave_paths", c_int32), ("spectral", c_int32), ("tri_light_nee", c_int32)]


class PathRecord(ctypes.Structure):
    _fields_ = [("radiance", c_float * 3), ("segments", c_int32), ("uniforms", c_int32), ("nee_rays", c_int32),
                ("nee_depth_mask", c_int32), ("reserved", c_int32), ("hit_object", c_int32 * DEBUG_MAX_HITS)]


class SceneInfo(ctypes.Structure):
    _fields_ = [("objects", c_int64), ("triangles", c_int64), ("lights", c_int64), ("wide_nodes", c_int64),
                ("prim_refs", c_int64), ("device_bytes", c_int64), ("device", c_int32), ("camera_inside", c_int32)]


class BvhInfo(ctypes.Structure):
    _fields_ = [("wide_nodes", c_int64), ("prim_refs", c_int64), ("leaf_slots", c_int64), ("internal_slots", c_int64),
                ("stack_bound", c_int32), ("depth", c_int32)]


class RenderStats(ctypes.Structure):
    _fields_ = [("paths", c_int64), ("extension_rays", c_int64), ("shadow_rays", c_int64),
                ("kernel_launches", c_int64), ("extend_launches", c_int64), ("shadow_launches", c_int64),
                ("extend_node_visits", c_int64), ("extend_prim_tests", c_int64), ("shadow_node_visits", c_int64),
                ("shadow_prim_tests", c_int64),
                ("extend_ms", c_float), ("shadow_ms", c_float), ("total_ms", c_float), ("reserved", c_int32)]


assert ctypes.sizeof(ObjectDesc) == 208
assert ctypes.sizeof(PathRecord) == 96
class Job(ctypes.Structure):
    _fields_ = [("scene", c_void_p), ("camera", Camera), ("params", RenderParams), ("out_rgb", c_void_p),
                ("accum", c_void_p)]


class NrcConfig(ctypes.Structure):
    _fields_ = [("levels", c_int32), ("log2_entries", c_int32), ("base_resolution", c_int32),
                ("max_resolution", c_int32), ("bounds_min", c_float * 3), ("bounds_max", c_float * 3),
                ("train_paths", c_int32), ("train_batch", c_int32), ("train_steps", c_int32),
                ("max_train_vertices", c_int32), ("learning_rate", c_float), ("spread_c", c_float),
                ("seed", ctypes.c_uint64)]


class NrcFrameStats(ctypes.Structure):
    _fields_ = [("total_ms", c_float), ("render_ms", c_float), ("infer_ms", c_float), ("train_ms", c_float),
                ("queries", c_int64), ("train_samples", c_int64), ("extension_rays", c_int64),
                ("shadow_rays", c_int64), ("loss", c_float), ("reserved", c_int32)]


NRC_PARAMS = 21504


def nrc_config(levels=16, log2_entries=19, base_resolution=16, max_resolution=2048, bounds=None,
               train_paths=65536, train_batch=16384, train_steps=4, max_train_vertices=8, learning_rate=1e-2,
               spread_c=0.01, seed=1) -> NrcConfig:
    c = NrcConfig(levels, log2_entries, base_resolution, max_resolution)
    if bounds is not None:
        c.bounds_min[:] = [float(x) for x in bounds[0]]
        c.bounds_max[:] = [float(x) for x in bounds[1]]
    c.train_paths, c.train_batch, c.train_steps = train_paths, train_batch, train_steps
    c.max_train_vertices, c.learning_rate, c.spread_c, c.seed = max_train_vertices, learning_rate, spread_c, seed
    return c


class GuideConfig(ctypes.Structure):
    _fields_ = [("probe_capacity", c_int32), ("log2_table", c_int32)]


class GuideStats(ctypes.Structure):
    _fields_ = [("frames", c_int64), ("probes", c_int64), ("samples", c_int64), ("dropped", c_int64),
                ("alpha", c_float), ("reserved", c_int32)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("iterations_per_graph", c_int32), ("candidates", c_int32), ("path_budget", c_int64),
                ("best_ms", c_float), ("default_ms", c_float), ("trace_blocks_per_sm", c_int32),
                ("shade_blocks_per_sm", c_int32)]


class BatchStats(ctypes.Structure):
    _fields_ = [("total_ms", c_float), ("iterations_per_graph", c_int32), ("paths", c_int64),
                ("extension_rays", c_int64), ("shadow_rays", c_int64), ("graph_launches", c_int64),
                ("graph_nodes", c_int64), ("kernel_launches", c_int64), ("loop_passes", c_int64)]


class ScreenGBuffer(ctypes.Structure):
    """ar_screen_gbuffer: per-pixel guide values of the denoiser (half fields as uint16 bits)."""
    _fields_ = [("albedo", ctypes.c_uint16 * 3), ("normal", ctypes.c_uint16 * 3), ("metallic", ctypes.c_uint16),
                ("roughness", ctypes.c_uint16), ("depth", c_float), ("valid_frames", ctypes.c_uint32),
                ("frames", ctypes.c_uint32), ("shading_model", ctypes.c_uint16 * 6), ("reserved", ctypes.c_uint32 * 2)]


class ScreenStats(ctypes.Structure):
    """ar_screen_stats: per-pixel Box-Cox moments of the denoiser."""
    _fields_ = [("num", ctypes.c_uint32), ("mean", c_float * 3), ("m2_div_n", c_float * 3),
                ("m3_div_n", c_float * 3), ("reserved", ctypes.c_uint32 * 2)]


OBJECT_DTYPE = np.dtype(ObjectDesc)
GBUFFER_DTYPE = np.dtype(ScreenGBuffer)
STATS_DTYPE = np.dtype(ScreenStats)
RECORD_DTYPE = np.dtype(PathRecord)

EXPORTED_SYMBOLS = ("ar_version", "ar_get_last_error_string", "ar_scene_create", "ar_scene_create_ex",
                    "ar_scene_destroy",
                    "ar_scene_get_info", "ar_bvh_build_info", "ar_render", "ar_trace_rays", "ar_trace_rays_static",
                    "ar_render_debug_paths", "ar_rng_tape", "ar_tonemap", "ar_accum_resolve", "ar_tone_curve",
                    "ar_scene_set_spectral", "ar_scene_get_spectral_luts", "ar_render_batch",
                    "ar_scene_set_medium", "ar_nrc_create", "ar_nrc_destroy", "ar_nrc_render_frame",
                    "ar_nrc_get_params", "ar_nrc_set_params", "ar_nrc_infer", "ar_nrc_train", "ar_nrc_gradients",
                    "ar_batch_autotune", "ar_nrc_set_option", "ar_guide_create", "ar_guide_destroy", "ar_guide_render_frame",
                    "ar_guide_get_stats", "ar_guide_get_probe", "ar_guide_probe_eval", "ar_render_frame_denoise",
                    "ar_denoise_record", "ar_denoise_bilateral", "ar_scene_set_spectral_ex", "ar_spectral_rgb_lut")


class ArError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libaperture_b200.so and declare the prototypes; raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built; run `make -C {HERE}`")
    lib = ctypes.CDLL(path)
    lib.ar_version.restype = c_int32
    lib.ar_get_last_error_string.restype = c_char_p
    lib.ar_scene_create.argtypes = [c_void_p, c_size_t, c_int32, POINTER(c_void_p)]
    lib.ar_scene_create.restype = c_int32
    lib.ar_scene_create_ex.argtypes = [c_void_p, c_size_t, c_void_p, c_size_t, c_int32, POINTER(c_void_p)]
    lib.ar_scene_create_ex.restype = c_int32
    lib.ar_scene_destroy.argtypes = [c_void_p]
    lib.ar_scene_destroy.restype = None
    lib.ar_scene_get_info.argtypes = [c_void_p, POINTER(SceneInfo)]
    lib.ar_scene_get_info.restype = c_int32
    lib.ar_bvh_build_info.argtypes = [c_void_p, c_size_t, c_void_p, c_size_t, POINTER(BvhInfo)]
    lib.ar_bvh_build_info.restype = c_int32
    lib.ar_render.argtypes = [c_void_p, POINTER(Camera), POINTER(RenderParams), c_void_p, c_void_p, c_int32,
                              c_void_p, POINTER(RenderStats)]
    lib.ar_render.restype = c_int32
    lib.ar_trace_rays.argtypes = [c_void_p, c_void_p, c_size_t, c_int32, c_void_p, c_void_p, c_int32, c_void_p]
    lib.ar_trace_rays.restype = c_int32
    lib.ar_trace_rays_static.argtypes = [c_void_p, c_void_p, c_size_t, c_int32, c_void_p, c_void_p, c_void_p]
    lib.ar_trace_rays_static.restype = c_int32
    lib.ar_render_debug_paths.argtypes = [c_void_p, POINTER(Camera), POINTER(RenderParams), c_void_p, c_int32,
                                          c_void_p]
    lib.ar_render_debug_paths.restype = c_int32
    lib.ar_rng_tape.argtypes = [POINTER(Camera), POINTER(RenderParams), c_int32, c_void_p, c_int32, c_void_p]
    lib.ar_rng_tape.restype = c_int32
    lib.ar_tonemap.argtypes = [c_void_p, c_size_t, c_int32, c_float, c_int32, c_void_p, c_int32, c_void_p]
    lib.ar_tonemap.restype = c_int32
    lib.ar_accum_resolve.argtypes = [c_void_p, c_size_t, c_double, c_void_p, c_int32, c_void_p]
    lib.ar_accum_resolve.restype = c_int32
    lib.ar_tone_curve.argtypes = [c_void_p, c_int32, c_void_p]
    lib.ar_tone_curve.restype = c_int32
    lib.ar_scene_set_spectral.argtypes = [c_void_p, c_void_p, c_size_t, c_int32]
    lib.ar_scene_set_spectral.restype = c_int32
    lib.ar_scene_get_spectral_luts.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.ar_scene_get_spectral_luts.restype = c_int32
    lib.ar_scene_set_medium.argtypes = [c_void_p, c_void_p]
    lib.ar_scene_set_medium.restype = c_int32
    lib.ar_render_batch.argtypes = [c_void_p, c_int32, c_int32, c_int64, POINTER(BatchStats), c_void_p]
    lib.ar_render_batch.restype = c_int32
    lib.ar_guide_create.argtypes = [c_void_p, POINTER(GuideConfig), POINTER(c_void_p)]
    lib.ar_guide_destroy.argtypes = [c_void_p]
    lib.ar_guide_render_frame.argtypes = [c_void_p, POINTER(Camera), POINTER(RenderParams), c_void_p, c_void_p, c_void_p]
    lib.ar_guide_get_stats.argtypes = [c_void_p, POINTER(GuideStats)]
    lib.ar_guide_get_probe.argtypes = [c_void_p, c_int32, c_void_p]
    lib.ar_scene_set_spectral_ex.argtypes = [c_void_p, c_void_p, c_size_t, c_int32, c_int32]
    lib.ar_spectral_rgb_lut.argtypes = [c_void_p, c_size_t, c_int32, c_int32, c_void_p, c_void_p]
    lib.ar_scene_set_spectral_ex.restype = c_int32
    lib.ar_spectral_rgb_lut.restype = c_int32
    lib.ar_guide_probe_eval.argtypes = [c_void_p, c_int32] + [c_void_p] * 6 + [c_int64] + [c_void_p] * 4
    for f in ("ar_guide_create", "ar_guide_destroy", "ar_guide_render_frame", "ar_guide_get_stats", "ar_guide_get_probe",
              "ar_guide_probe_eval"):
        getattr(lib, f).restype = c_int32
    lib.ar_render_frame_denoise.argtypes = [c_void_p, POINTER(Camera), POINTER(RenderParams), c_void_p, c_void_p,
                                            c_void_p, c_void_p, c_void_p]
    lib.ar_denoise_record.argtypes = [c_void_p, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p]
    lib.ar_denoise_bilateral.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p]
    for f in ("ar_render_frame_denoise", "ar_denoise_record", "ar_denoise_bilateral"):
        getattr(lib, f).restype = c_int32
    lib.ar_batch_autotune.argtypes = [c_void_p, c_int32, c_int32, POINTER(BatchTuning), c_void_p]
    lib.ar_batch_autotune.restype = c_int32
    lib.ar_nrc_create.argtypes = [c_void_p, POINTER(NrcConfig), POINTER(c_void_p)]
    lib.ar_nrc_destroy.argtypes = [c_void_p]
    lib.ar_nrc_render_frame.argtypes = [c_void_p, POINTER(Camera), POINTER(RenderParams), c_void_p, c_void_p,
                                        c_int32, POINTER(NrcFrameStats), c_void_p]
    lib.ar_nrc_get_params.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.ar_nrc_set_params.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.ar_nrc_infer.argtypes = [c_void_p, c_void_p, c_size_t, c_void_p]
    lib.ar_nrc_train.argtypes = [c_void_p, c_void_p, c_size_t, c_int32, c_void_p]
    lib.ar_nrc_gradients.argtypes = [c_void_p, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p]
    lib.ar_nrc_set_option.argtypes = [c_void_p, c_int32, c_int32]
    lib.ar_nrc_set_option.restype = c_int32
    for f in ("ar_nrc_create", "ar_nrc_destroy", "ar_nrc_render_frame", "ar_nrc_get_params", "ar_nrc_set_params",
              "ar_nrc_infer", "ar_nrc_train", "ar_nrc_gradients"):
        getattr(lib, f).restype = c_int32
    _lib = lib
    return lib


def _check(status: int) -> None:
    if status != AR_OK:
        msg = _lib.ar_get_last_error_string().decode(errors="replace")
        raise ArError(status, msg)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def make_camera(position, direction, fov_y_deg, width, height) -> Camera:
    return Camera(Vec3(*map(float, position)), Vec3(*map(float, direction)), float(fov_y_deg), int(width),
                  int(height))


def make_params(spp=1, max_depth=8, rr_depth=3, use_nee=1, sky=1, frame_offset=0, seed=REFERENCE_SEED,
                sort_rays=0, wave_paths=0, spectral=0, tri_light_nee=0) -> RenderParams:
    return RenderParams(int(spp), int(max_depth), int(rr_depth), int(use_nee), int(sky), int(frame_offset),
                        int(seed) & 0xFFFFFFFFFFFFFFFF, int(sort_rays), int(wave_paths), int(spectral),
                        int(tri_light_nee))


def medium_desc(density: np.ndarray, bounds_min, bounds_max, sigma_t_max, albedo, g) -> MediumDesc:
    """ar_medium_desc for a [z, y, x] grid (the array must stay alive while used)."""
    m = MediumDesc()
    m.bounds_min[:] = [float(x) for x in bounds_min]
    m.bounds_max[:] = [float(x) for x in bounds_max]
    m.sigma_t_max = float(sigma_t_max)
    m.albedo[:] = [float(x) for x in albedo]
    m.g = float(g)
    m.dims[:] = [density.shape[2], density.shape[1], density.shape[0]]
    m.precision = 16 if density.dtype == np.float16 else 32
    m.density = density.ctypes.data
    return m


class Scene:
    """Owns one ar_scene handle (the SceneRenderer of the reference)."""

    def __init__(self, objects: np.ndarray, device: int = 0, volumes=None):
        """volumes: list of (SdfVolume, keep-alive array or None) from make_volume()."""
        lib = load_library()
        objects = np.ascontiguousarray(objects, dtype=OBJECT_DTYPE)
        self._objects_keepalive = objects
        h = c_void_p()
        if volumes:
            arr = (SdfVolume * len(volumes))(*[v for v, _ in volumes])
            _check(lib.ar_scene_create_ex(_ptr(objects) if len(objects) else None, len(objects), arr, len(volumes),
                                          device, ctypes.byref(h)))
        else:
            _check(lib.ar_scene_create(_ptr(objects) if len(objects) else None, len(objects), device,
                                       ctypes.byref(h)))
        self._h = h
        self.num_objects = len(objects)

    def set_spectral(self, lut_res: int = 64, tables: np.ndarray | None = None, method: int = 0) -> None:
        """Enable spectral rendering: the reference's tables (spectral_tables.load()
        unless given) and an lut_res^3 RGB lookup table built on the device
        (method LUT_SIMT, or LUT_TENSOR on the tcgen05 tensor cores)."""
        if tables is None:
            import spectral_tables
            tables = spectral_tables.load()[0]
        t = np.ascontiguousarray(tables, np.float32)
        _check(_lib.ar_scene_set_spectral_ex(self._h, _ptr(t), t.size, lut_res, int(method)))
        self.lut_res = lut_res

    def set_medium(self, density, bounds_min=None, bounds_max=None, sigma_t_max: float = 0.0, albedo=None,
                   g: float = 0.0) -> None:
        """Attach a participating medium; density is a [z, y, x] float32 or
        float16 array (x fastest), None removes the medium."""
        if density is None:
            _check(_lib.ar_scene_set_medium(self._h, None))
            return
        d = np.ascontiguousarray(density)
        if d.dtype not in (np.float32, np.float16) or d.ndim != 3:
            raise ValueError("density must be a 3-d float32 or float16 array")
        m = medium_desc(d, bounds_min, bounds_max, sigma_t_max, albedo, g)
        _check(_lib.ar_scene_set_medium(self._h, ctypes.byref(m)))

    def spectral_luts(self):
        """(lambda table [840, 4], rgb table [res^3, 4]) as built on the device."""
        lam = np.zeros((840, 4), np.float32)
        rgb = np.zeros((self.lut_res ** 3, 4), np.float32)
        _check(_lib.ar_scene_get_spectral_luts(self._h, _ptr(lam), _ptr(rgb)))
        return lam, rgb

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.ar_scene_destroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self) -> int:
        return self._h.value

    def info(self) -> SceneInfo:
        si = SceneInfo()
        _check(_lib.ar_scene_get_info(self._h, ctypes.byref(si)))
        return si

    def render(self, camera: Camera, params: RenderParams, accum: np.ndarray | None = None,
               stream: int = 0, want_stats: bool = True, out: np.ndarray | None = None):
        """Host-buffer render; returns (image[h, w, 3] float32, RenderStats).
        out: a caller-owned float32 host array of h*w*3 values to write into
        (page-locked memory makes the copy back a direct DMA)."""
        if out is None:
            out = np.empty((camera.height, camera.width, 3), np.float32)
        else:
            if not (out.dtype == np.float32 and out.flags.c_contiguous and out.size == camera.height * camera.width * 3):
                raise ValueError("out must be a C-contiguous float32 array of height * width * 3 values")
            out = out.reshape(camera.height, camera.width, 3)
        st = RenderStats()
        acc_ptr = None
        if accum is not None:
            assert accum.dtype == np.float64 and accum.flags.c_contiguous
            acc_ptr = _ptr(accum)
        _check(_lib.ar_render(self._h, ctypes.byref(camera), ctypes.byref(params), _ptr(out), acc_ptr, MEM_HOST,
                              c_void_p(stream), ctypes.byref(st) if want_stats else None))
        return out, st

    def render_device(self, camera: Camera, params: RenderParams, out_ptr: int, accum_ptr: int | None = None,
                      stream: int = 0, stats: RenderStats | None = None) -> None:
        """Device-buffer render into caller-owned device memory (pointers)."""
        _check(_lib.ar_render(self._h, ctypes.byref(camera), ctypes.byref(params), c_void_p(out_ptr),
                              c_void_p(accum_ptr) if accum_ptr else None, MEM_DEVICE, c_void_p(stream),
                              ctypes.byref(stats) if stats is not None else None))

    def trace_rays(self, rays: np.ndarray, any_hit: bool = False):
        """rays: float32 [n, 8] (origin, tmin, direction, tmax) -> (hit_object int32[n], t float32[n])."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = rays.shape[0]
        obj = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        _check(_lib.ar_trace_rays(self._h, _ptr(rays), n, int(any_hit), _ptr(obj), _ptr(t), MEM_HOST, None))
        return obj, t

    def trace_rays_device(self, rays_ptr: int, n: int, any_hit: bool, obj_ptr: int, t_ptr: int | None,
                          stream: int = 0) -> None:
        _check(_lib.ar_trace_rays(self._h, c_void_p(rays_ptr), n, int(any_hit), c_void_p(obj_ptr),
                                  c_void_p(t_ptr) if t_ptr else None, MEM_DEVICE, c_void_p(stream)))

    def trace_rays_static(self, rays_ptr: int, n: int, any_hit: bool, obj_ptr: int, t_ptr: int | None,
                          stream: int = 0) -> None:
        """ar_trace_rays_static: device buffers, no allocation by the library."""
        _check(_lib.ar_trace_rays_static(self._h, c_void_p(rays_ptr), n, int(any_hit), c_void_p(obj_ptr),
                                         c_void_p(t_ptr) if t_ptr else None, c_void_p(stream)))

    def debug_paths(self, camera: Camera, params: RenderParams) -> np.ndarray:
        n = camera.width * camera.height * params.spp
        rec = np.zeros(n, RECORD_DTYPE)
        _check(_lib.ar_render_debug_paths(self._h, ctypes.byref(camera), ctypes.byref(params), _ptr(rec), MEM_HOST,
                                          None))
        return rec


def bvh_build_info(objects: np.ndarray, volumes=None) -> BvhInfo:
    """The shape of the BVH Scene(objects, volumes=volumes) would build, built
    on the host alone (no device); raises if the structure check fails."""
    lib = load_library()
    objects = np.ascontiguousarray(objects, dtype=OBJECT_DTYPE)
    info = BvhInfo()
    arr = (SdfVolume * len(volumes))(*[v for v, _ in volumes]) if volumes else None
    _check(lib.ar_bvh_build_info(_ptr(objects) if len(objects) else None, len(objects), arr,
                                 len(volumes) if volumes else 0, ctypes.byref(info)))
    return info


def rng_tape(camera: Camera, params: RenderParams, per_path: int) -> np.ndarray:
    load_library()
    n = camera.width * camera.height * params.spp
    out = np.empty((n, per_path), np.float32)
    _check(_lib.ar_rng_tape(ctypes.byref(camera), ctypes.byref(params), int(per_path), _ptr(out), MEM_HOST, None))
    return out


TONE_NONE, TONE_GAMMA, TONE_ACES = 0, 1, 2


def tonemap(rgb: np.ndarray, tone: int = TONE_ACES, exposure: float = 1.0, xyz_input: bool = False) -> np.ndarray:
    """Linear rgb[n, 3] (host) -> 0xAARRGGBB per pixel, the reference's LDR format."""
    lib = load_library()
    rgb = np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)
    out = np.empty(len(rgb), np.uint32)
    _check(lib.ar_tonemap(_ptr(rgb), len(rgb), tone, exposure, int(xyz_input), _ptr(out), MEM_HOST, None))
    return out


def make_volume(dims, data: np.ndarray | None = None, precision: int = 32, fill_kind: int = SDF_TORUS,
                fill_info=(0.375, 0.125, 0.0, 0.0)):
    """An ar_sdf_volume: host data (float32 or float16 array of dims[2]*dims[1]*dims[0]
    values, x fastest) or, without data, filled on the device from fill_kind."""
    v = SdfVolume()
    v.dims[:] = [int(d) for d in dims]
    v.precision = precision
    keep = None
    if data is not None:
        keep = np.ascontiguousarray(data, np.float16 if precision == 16 else np.float32).reshape(-1)
        assert keep.size == int(np.prod(dims))
        v.data = keep.ctypes.data
    v.fill_kind = fill_kind
    v.fill_info[:] = [float(x) for x in fill_info]
    return v, keep


def _job_array(jobs):
    arr = (Job * len(jobs))()
    for k, (scene, cam, params, out_ptr, acc_ptr) in enumerate(jobs):
        arr[k].scene = scene.handle
        arr[k].camera = cam
        arr[k].params = params
        arr[k].out_rgb = out_ptr
        arr[k].accum = acc_ptr
    return arr


LUT_SIMT, LUT_TENSOR = 0, 1


def spectral_rgb_lut(res: int, method: int, tables: np.ndarray | None = None, out=None):
    """ar_spectral_rgb_lut: the res^3 x 4 RGB lookup table built on the current
    device into a torch tensor (allocated unless given); returns (table, ms)."""
    import torch
    load_library()
    if tables is None:
        import spectral_tables
        tables = spectral_tables.load()[0]
    t = np.ascontiguousarray(tables, np.float32)
    if out is None:
        out = torch.empty(res * res * res * 4, dtype=torch.float32, device="cuda")
    ms = ctypes.c_float(0.0)
    _check(_lib.ar_spectral_rgb_lut(_ptr(t), t.size, res, int(method), c_void_p(out.data_ptr()), ctypes.byref(ms)))
    return out, ms.value


def autotune_batch(jobs, probe_spp: int = 4, stream: int = 0) -> BatchTuning:
    """ar_batch_autotune: choose graph length and path budget for this batch
    shape; later render_batch calls with both left at 0 use the choice."""
    lib = load_library()
    arr = _job_array(jobs)
    t = BatchTuning()
    _check(lib.ar_batch_autotune(arr, len(jobs), probe_spp, ctypes.byref(t), c_void_p(stream)))
    return t


def render_batch(jobs, iterations_per_graph: int = 0, path_budget: int = 0, stream: int = 0) -> BatchStats:
    """jobs: sequence of (Scene, Camera, RenderParams, out_rgb device pointer, accum device pointer or None)."""
    lib = load_library()
    arr = (Job * len(jobs))()
    for k, (scene, cam, params, out_ptr, acc_ptr) in enumerate(jobs):
        arr[k].scene = scene.handle
        arr[k].camera = cam
        arr[k].params = params
        arr[k].out_rgb = out_ptr
        arr[k].accum = acc_ptr
    st = BatchStats()
    _check(lib.ar_render_batch(arr, len(jobs), iterations_per_graph, path_budget, ctypes.byref(st), c_void_p(stream)))
    return st


class RadianceCache:
    """ar_nrc: the learned radiance cache of a scene."""

    def __init__(self, scene: "Scene", config: NrcConfig | None = None):
        lib = load_library()
        self.config = config or nrc_config()
        self._scene = scene
        h = c_void_p()
        _check(lib.ar_nrc_create(scene.handle, ctypes.byref(self.config), ctypes.byref(h)))
        self._h = h
        self.table_floats = self.config.levels * (1 << self.config.log2_entries) * 2

    def render_frame(self, camera: Camera, params: RenderParams, out_ptr: int | None, accum_ptr: int | None,
                     train: bool = True, stats: bool = False, stream: int = 0):
        st = NrcFrameStats() if stats else None
        _check(_lib.ar_nrc_render_frame(self._h, ctypes.byref(camera), ctypes.byref(params),
                                        c_void_p(out_ptr) if out_ptr else None,
                                        c_void_p(accum_ptr) if accum_ptr else None, int(train),
                                        ctypes.byref(st) if st is not None else None, c_void_p(stream)))
        return st

    def set_spectral(self, mode: int) -> None:
        """Cache mode before the first frame: 0 RGB, 4 four wavelengths per path
        (16 spectral bins)."""
        _check(_lib.ar_nrc_set_option(self._h, 2, int(mode)))
        self.spectral = int(mode)

    @staticmethod
    def _samples(samples: np.ndarray) -> np.ndarray:
        """Training samples as rows of 20 floats (16-float rows get 4 zeros)."""
        s = np.ascontiguousarray(samples, np.float32)
        s = s.reshape(-1, s.shape[-1]) if s.ndim > 1 else s.reshape(-1, 20)
        if s.shape[1] == 16:
            s = np.concatenate([s, np.zeros((len(s), 4), np.float32)], axis=1)
        return np.ascontiguousarray(s)

    def set_tensor_path(self, tcgen05: bool) -> None:
        """Inference kernel: tcgen05.mma with tensor-memory accumulators, or mma.sync."""
        _check(_lib.ar_nrc_set_option(self._h, 1, 1 if tcgen05 else 0))

    def params(self):
        t = np.empty(self.table_floats, np.float32)
        w = np.empty(NRC_PARAMS, np.float32)
        _check(_lib.ar_nrc_get_params(self._h, _ptr(t), _ptr(w)))
        return t, w

    def set_params(self, table: np.ndarray | None, weights: np.ndarray | None) -> None:
        t = None if table is None else np.ascontiguousarray(table, np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        _check(_lib.ar_nrc_set_params(self._h, _ptr(t) if t is not None else None, _ptr(w) if w is not None else None))

    def infer(self, vertices: np.ndarray) -> np.ndarray:
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 16)
        out = np.empty((len(v), 16 if getattr(self, "spectral", 0) else 3), np.float32)
        _check(_lib.ar_nrc_infer(self._h, _ptr(v), len(v), _ptr(out)))
        return out

    def train(self, samples: np.ndarray, steps: int) -> np.ndarray:
        s = self._samples(samples)
        losses = np.zeros(max(steps, 1), np.float32)
        _check(_lib.ar_nrc_train(self._h, _ptr(s), len(s), steps, _ptr(losses)))
        return losses[:steps]

    def gradients(self, samples: np.ndarray):
        s = self._samples(samples)
        tg = np.empty(self.table_floats, np.float32)
        wg = np.empty(NRC_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        _check(_lib.ar_nrc_gradients(self._h, _ptr(s), len(s), _ptr(tg), _ptr(wg), _ptr(loss)))
        return tg, wg, float(loss[0])

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.ar_nrc_destroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _dptr(x) -> c_void_p | None:
    """Device address of a torch tensor (or an int address), None for None."""
    if x is None:
        return None
    return c_void_p(x if isinstance(x, int) else x.data_ptr())


def render_frame_denoise(scene: "Scene", camera: Camera, params: RenderParams, out_ptr, accum_ptr, gbuffer, stats,
                         stream: int = 0) -> None:
    """ar_render_frame_denoise: one interactive frame (spp = 1) that records the
    denoiser's guide buffers; device buffers as torch tensors or addresses."""
    _check(_lib.ar_render_frame_denoise(scene.handle, ctypes.byref(camera), ctypes.byref(params), _dptr(out_ptr),
                                        _dptr(accum_ptr), _dptr(gbuffer), _dptr(stats), c_void_p(stream)))


def denoise_record(hits, samples, n: int, gbuffer, stats, stream: int = 0) -> None:
    """ar_denoise_record on device buffers (torch tensors or addresses)."""
    load_library()
    _check(_lib.ar_denoise_record(_dptr(hits), _dptr(samples), n, _dptr(gbuffer), _dptr(stats), c_void_p(stream)))


def denoise_bilateral(hdr_in, hdr_out, gbuffer, stats, width: int, height: int, stream: int = 0) -> None:
    """ar_denoise_bilateral on device buffers (torch tensors or addresses)."""
    load_library()
    _check(_lib.ar_denoise_bilateral(_dptr(hdr_in), _dptr(hdr_out), _dptr(gbuffer), _dptr(stats), width, height,
                                     c_void_p(stream)))


def guide_probe_eval(texels: np.ndarray, probe_of, normal, query, u5, eval_dir, pos):
    """ar_guide_probe_eval on host arrays: texels [nprobes, 85, 4]; per query
    probe index, normal, texel weights, 5 uniforms, evaluation direction and
    point.  Returns (sample directions [n, 3], sample pdfs, pdfs of eval_dir,
    (voxel, face) keys as uint64)."""
    load_library()
    t = np.ascontiguousarray(texels, np.float32).reshape(-1, 85, 4)
    po = np.ascontiguousarray(probe_of, np.int32).reshape(-1)
    n = len(po)
    arrs = [np.ascontiguousarray(a, np.float32).reshape(n, -1) for a in (normal, query, u5, eval_dir, pos)]
    d = np.empty((n, 3), np.float32)
    p = np.empty(n, np.float32)
    e = np.empty(n, np.float32)
    k = np.empty(n, np.uint64)
    _check(_lib.ar_guide_probe_eval(_ptr(t), len(t), _ptr(po), *[_ptr(a) for a in arrs], n, _ptr(d), _ptr(p), _ptr(e),
                                    _ptr(k)))
    return d, p, e, k


class PathGuide:
    """ar_guide: path-guiding probes of a scene for interactive frames."""

    def __init__(self, scene: "Scene", probe_capacity: int = 0, log2_table: int = 0):
        lib = load_library()
        self._scene = scene
        h = c_void_p()
        cfg = GuideConfig(probe_capacity, log2_table)
        _check(lib.ar_guide_create(scene.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h

    def render_frame(self, camera: Camera, params: RenderParams, out_ptr: int | None, accum_ptr: int | None,
                     stream: int = 0) -> None:
        _check(_lib.ar_guide_render_frame(self._h, ctypes.byref(camera), ctypes.byref(params),
                                          c_void_p(out_ptr) if out_ptr else None,
                                          c_void_p(accum_ptr) if accum_ptr else None, c_void_p(stream)))

    def stats(self) -> GuideStats:
        st = GuideStats()
        _check(_lib.ar_guide_get_stats(self._h, ctypes.byref(st)))
        return st

    def probe(self, index: int) -> np.ndarray:
        out = np.empty((88, 4), np.float32)
        _check(_lib.ar_guide_get_probe(self._h, index, _ptr(out)))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.ar_guide_destroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

