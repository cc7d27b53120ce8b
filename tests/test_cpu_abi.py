"""The C ABI without a GPU: the library loads, exports exactly what the header
declares, its structs have the header's layout, and every call that needs a
device reports AR_ERR_NO_DEVICE (or rejects its arguments) instead of crashing.

No test here launches a kernel; they run on a CPU-only host.
"""
import ctypes
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import aperture_b200 as ab
import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "aperture_b200.h")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def header_functions() -> list[str]:
    """Names of the functions include/aperture_b200.h declares."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(ar_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_binding_symbols():
    assert header_functions() == sorted(ab.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol(lib):
    for name in header_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", ab.LIB_PATH], capture_output=True, text=True)
    if out.returncode == 0:
        exported = set(re.findall(r"\bT (ar_\w+)$", out.stdout, flags=re.M))
        assert exported == set(header_functions()), exported ^ set(header_functions())


def test_version(lib):
    assert lib.ar_version() == 1


STRUCTS = {
    "ar_vec3": ab.Vec3, "ar_material": ab.Material, "ar_vertex": ab.Vertex, "ar_object_desc": ab.ObjectDesc,
    "ar_camera": ab.Camera, "ar_render_params": ab.RenderParams, "ar_path_record": ab.PathRecord,
    "ar_scene_info": ab.SceneInfo, "ar_render_stats": ab.RenderStats,
    "ar_screen_gbuffer": ab.ScreenGBuffer, "ar_screen_stats": ab.ScreenStats,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_struct_layout_matches_header(tmp_path):
    """sizeof/offsetof from a C compile of the header equal the ctypes layout."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        c, f, v = ln.split()
        got[(c, f)] = int(v)
    for cname, cls in STRUCTS.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)
    assert ctypes.sizeof(ab.ObjectDesc) == 208 and ctypes.sizeof(ab.PathRecord) == 96


def test_null_arguments_are_rejected(lib):
    cam = scenes.box_camera(8, 8)
    p = ab.make_params(spp=1)
    st = lib.ar_render(None, ctypes.byref(cam), ctypes.byref(p), None, None, ab.MEM_HOST, None, None)
    assert st == 1
    assert b"NULL" in lib.ar_get_last_error_string() or b"null" in lib.ar_get_last_error_string().lower()
    assert lib.ar_scene_get_info(None, ctypes.byref(ab.SceneInfo())) == 1
    assert lib.ar_trace_rays(None, None, 0, 0, None, None, ab.MEM_HOST, None) == 1
    assert lib.ar_trace_rays_static(None, None, 0, 0, None, None, None) == 1
    lib.ar_scene_destroy(None)  # no-op


def test_sort_rays_is_rejected(lib):
    """Ray sorting beyond material buckets is not built: asking for it fails
    with AR_ERR_UNSUPPORTED instead of being ignored (checked on the parameter
    path shared by every render entry point, before any device work)."""
    cam = scenes.box_camera(8, 8)
    p = ab.make_params(spp=1, sort_rays=1)
    out = np.zeros(64 * 4, np.float32)
    st = lib.ar_rng_tape(ctypes.byref(cam), ctypes.byref(p), 4, out.ctypes.data, ab.MEM_HOST, None)
    assert st == 4
    assert b"sort_rays" in lib.ar_get_last_error_string()


def test_scene_create_rejects_bad_input(lib):
    h = ctypes.c_void_p()
    assert lib.ar_scene_create(None, 3, 0, ctypes.byref(h)) == 1
    objs = scenes.box_scene()
    assert lib.ar_scene_create(objs.ctypes.data, len(objs), 0, None) == 1


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_scene_create_without_device_reports_no_device(lib):
    objs = scenes.box_scene()
    with pytest.raises(ab.ArError) as e:
        ab.Scene(objs)
    assert e.value.status == 6
    assert "device" in str(e.value).lower()


def test_scene_generators_are_deterministic():
    a, b = scenes.spheres_scene(), scenes.spheres_scene()
    assert a.tobytes() == b.tobytes()
    tris = int(np.count_nonzero(a["type"] == ab.OBJ_TRIANGLE))
    assert tris == 800 * 1280 + 2
    assert int(np.count_nonzero(a["material"]["shading_model"] == ab.MAT_LIGHT)) == 16
    box = scenes.box_scene()
    assert box.tobytes() == scenes.box_scene().tobytes()
    assert int(np.count_nonzero(box["type"] == ab.OBJ_TRIANGLE)) == 10 + 2 * 12
