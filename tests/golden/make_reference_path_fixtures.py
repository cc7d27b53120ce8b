"""Generate tests/golden/reference_paths.npz: per-path records of the reference
renderer's own path loop (CalculateRadiance, core/render/render.cuh:460-999,
with Trace, NEE, the BSDFs, NEE samplers, BVH traversal and Overlap under it),
run on the host from the build-time copy `make -C oracle ref-path` compiles
(oracle/ref_path_patch.py lists the edits, oracle/ref_path_harness.cu drives
it through the per-pixel part of RenderCamera, core/scene.cu:213-240).

Two builds are recorded: the reference's arithmetic with the oracle's fixed
transcendental functions (libref_path_detmath.so), and with the host math
library (libref_path.so).  The uniforms come from a seeded tape (numpy PCG64,
values in (0, 1]); each scene stores the tape's seed and shape, and the
SHA-256 of its object array so that a changed generator is caught.

Scenes (RGB, NEE on, Russian roulette from non-delta depth 3, sky on):
  box          config 1 (scenes.box_scene()), 48x48, 2 spp, depth 8
  spheres      24 icospheres (1 subdivision) + ground + 4 light spheres,
               64x36, 2 spp, depth 12
  spheres_deep 200 icospheres (2 subdivisions, 64,002 triangles) + 8 light
               spheres, 48x27, 2 spp, depth 12

Run from the repository root after `make -C oracle ref-path`:
    python tests/golden/make_reference_path_fixtures.py
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "aperturerendererv3-optix-geometry_b200"), os.path.join(ROOT, "oracle")]

import reference_path  # noqa: E402
import scenes  # noqa: E402
from aperture_b200 import make_params  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_paths.npz")
TAPE_LEN = 768


def path_scenes():
    """name -> (objects, camera, params, tape seed)"""
    out = {}
    box = scenes.box_scene()
    out["box"] = (box, scenes.box_camera(48, 48), make_params(spp=2, max_depth=8), 101)
    sph = scenes.spheres_scene(n_spheres=24, n_lights=4, box=20.0, subdivisions=1)
    cam = scenes.spheres_camera(64, 36)
    cam.position.z = -45.0
    out["spheres"] = (sph, cam, make_params(spp=2, max_depth=12), 102)
    deep = scenes.spheres_scene(n_spheres=200, n_lights=8, box=60.0, subdivisions=2)
    cam = scenes.spheres_camera(48, 27)
    cam.position.z = -35.0
    out["spheres_deep"] = (deep, cam, make_params(spp=2, max_depth=12), 103)
    return out


def tape_for(seed: int, n_paths: int) -> np.ndarray:
    """Uniforms in (0, 1], one row of TAPE_LEN per path."""
    u = np.random.default_rng(seed).random((n_paths, TAPE_LEN), dtype=np.float32)
    return (np.float32(1.0) - u).astype(np.float32)


def camera_array(cam) -> np.ndarray:
    return np.array([cam.width, cam.height, cam.position.x, cam.position.y, cam.position.z, cam.direction.x,
                     cam.direction.y, cam.direction.z, cam.fov_y_deg], np.float64)


def main():
    out = {}
    for name, (objs, cam, params, seed) in path_scenes().items():
        n = cam.width * cam.height * params.spp
        tape = tape_for(seed, n)
        det, ov = reference_path.RefPathScene(objs, detmath=True).render_paths(cam, params, tape)
        assert ov == 0, f"{name}: tape too short"
        host, ov = reference_path.RefPathScene(objs, detmath=False).render_paths(cam, params, tape)
        assert ov == 0, f"{name}: tape too short"
        out[f"{name}_sha"] = np.frombuffer(hashlib.sha256(objs.tobytes()).digest(), np.uint8)
        out[f"{name}_camera"] = camera_array(cam)
        out[f"{name}_params"] = np.array([params.spp, params.max_depth, params.rr_depth, params.use_nee, params.sky],
                                         np.int32)
        out[f"{name}_tape"] = np.array([seed, n, TAPE_LEN], np.int64)
        for f in ("segments", "uniforms", "nee_rays", "nee_depth_mask"):
            out[f"{name}_{f}"] = det[f].astype(np.int32)
            out[f"{name}_host_{f}"] = host[f].astype(np.int32)
        out[f"{name}_hit_object"] = det["hit_object"].astype(np.int32)
        out[f"{name}_host_hit_object"] = host["hit_object"].astype(np.int32)
        out[f"{name}_radiance"] = det["radiance"].astype(np.float32)
        out[f"{name}_host_radiance"] = host["radiance"].astype(np.float32)
        print(f"{name}: {n} paths, {det['segments'].sum()} segments, {det['nee_rays'].sum()} shadow rays")
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
