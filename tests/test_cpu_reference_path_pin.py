"""The oracle's path loop against the reference's own path loop.

tests/golden/reference_paths.npz holds per-path records of the reference's
CalculateRadiance (core/render/render.cuh:460-999) and everything it calls,
run on the host from a build-time copy of the reference's sources
(tests/golden/make_reference_path_fixtures.py, oracle/ref_path_patch.py) with
the uniforms read from a seeded tape.  The oracle (oracle/oracle.c), in the
reference's modes -- triangle proxies at the object centre, the default
G-buffer on triangle hits, solo traces inside triangle media, the reference's
slab test and first-found tie rule -- replays the same tape:

* against the build whose transcendental functions are the oracle's fixed
  definitions: every field of every path bit for bit (closest-hit object per
  segment, segment count, uniforms consumed, shadow rays and their depths,
  radiance);
* against the build with the host math library (the reference's arithmetic
  as its host compiler runs it): the path structure identical on >= 99.9 % of
  the paths; radiance within 1e-5 relative on >= 98.5 % of them and within
  5e-3 on all (last-ulp differences of sinf/cosf/powf between math libraries,
  amplified along the path), image means within 1e-6.

The GPU core computes the oracle's non-reference modes: object materials on
triangles, lowest-index ties, the standard slab test, and inside a glass
triangle mesh the whole scene traced (the reference traces only the triangle
the path entered and, on a miss, restarts the path at the world origin).  The
chain test shows that the two modes agree path for path on scenes the
reference can express the same way -- triangle materials equal to the
reference's default G-buffer, no glass triangles -- which closes the chain
GPU = oracle = reference (tests/test_gpu_reference_path_pin.py runs that chain
on the GPU).
"""
import hashlib
import os
import sys

import numpy as np
import pytest

import aperture_b200 as ab
import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "reference_paths.npz")
REF_FLAGS = (oracle.PROXY_OBJECT_CENTER | oracle.TRIANGLE_DEFAULT_GBUFFER | oracle.TRIANGLE_SOLO_MEDIA
             | oracle.REFERENCE_TRAVERSAL)
SCENES = ["box", "spheres", "spheres_deep"]
FIELDS = ("segments", "uniforms", "nee_rays", "nee_depth_mask")


def _gen():
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_reference_path_fixtures as g
    return g


@pytest.fixture(scope="module")
def fx():
    return np.load(FIX)


@pytest.fixture(scope="module")
def cases(fx):
    g = _gen()
    out = {}
    for name, (objs, cam, params, seed) in g.path_scenes().items():
        digest = np.frombuffer(hashlib.sha256(objs.tobytes()).digest(), np.uint8)
        assert np.array_equal(digest, fx[f"{name}_sha"]), f"scene generator changed for {name}"
        n = cam.width * cam.height * params.spp
        assert np.array_equal(fx[f"{name}_tape"], [seed, n, g.TAPE_LEN])
        out[name] = (objs, cam, params, g.tape_for(seed, n))
    return out


@pytest.fixture(scope="module")
def oracle_records(cases):
    out = {}
    for name, (objs, cam, params, tape) in cases.items():
        rec, overflow = oracle.OracleScene(objs, flags=REF_FLAGS).render_paths(cam, params, tape)
        assert overflow == 0
        out[name] = rec
    return out


def default_gbuffer_materials(objs):
    """Triangles' materials set to the G-buffer the reference's triangle
    intersector leaves on its hits (IntersectTriangleObject,
    core/render/intersection.cuh:17, 63): white albedo, no emission, zero
    specular/metallic/roughness, IOR 1.5, sigma_a 100; shading models kept."""
    o = objs.copy()
    tri = o["type"] == ab.OBJ_TRIANGLE
    m = o["material"]
    for f in "xyz":
        m["albedo"][f][tri] = 1.0
        m["emissive"][f][tri] = 0.0
    m["specular"][tri] = 0.0
    m["metallic"][tri] = 0.0
    m["roughness"][tri] = 0.0
    m["ior"][tri] = 1.5
    m["sigma_a"][tri] = 100.0
    o["material"] = m
    return o


def without_glass_triangles(objs):
    """Glass triangles become diffuse: inside a glass triangle mesh the
    reference traces only the entered triangle (render.cuh:91-94) and the GPU
    core the whole scene, a documented deviation."""
    o = objs.copy()
    m = o["material"]
    glass = (o["type"] == ab.OBJ_TRIANGLE) & (m["shading_model"] == ab.MAT_GLASS)
    m["shading_model"][glass] = ab.MAT_DIFFUSE
    o["material"] = m
    return o


@pytest.mark.parametrize("name", SCENES)
def test_oracle_equals_reference_path_loop_fixed_math(fx, oracle_records, name):
    o = oracle_records[name]
    for f in FIELDS:
        assert np.array_equal(o[f], fx[f"{name}_{f}"]), f
    assert np.array_equal(o["hit_object"], fx[f"{name}_hit_object"])
    assert np.array_equal(o["radiance"].view(np.uint32), fx[f"{name}_radiance"].view(np.uint32))
    assert fx[f"{name}_segments"].sum() > 2000 and fx[f"{name}_nee_rays"].sum() > 1000


@pytest.mark.parametrize("name", SCENES)
def test_oracle_vs_reference_path_loop_host_math(fx, oracle_records, name):
    o = oracle_records[name]
    same = np.all(o["hit_object"] == fx[f"{name}_host_hit_object"], axis=1)
    for f in FIELDS:
        same &= o[f] == fx[f"{name}_host_{f}"]
    assert same.mean() >= 0.999
    a = o["radiance"].astype(np.float64)
    b = fx[f"{name}_host_radiance"].astype(np.float64)
    err = np.abs(a - b) / np.maximum(np.abs(b), 1e-30)
    err[(a == 0) & (b == 0)] = 0.0
    e = err[same].max(axis=1)
    assert (e <= 1e-5).mean() >= 0.985
    assert e.max() <= 5e-3
    assert abs(a.mean() - b.mean()) <= 1e-6 * abs(b.mean())


@pytest.mark.parametrize("name", SCENES)
def test_gpu_modes_equal_reference_modes_on_default_materials(cases, name):
    """The oracle as the GPU core runs it (object materials, lowest-index ties,
    standard slab test, bounds-centred proxies, whole-scene traces inside glass
    meshes) on the scene whose triangle materials are the reference's default
    G-buffer and which has no glass triangles equals the reference-mode oracle
    on that scene path for path -- and so the reference itself."""
    objs, cam, params, tape = cases[name]
    objs = without_glass_triangles(objs)
    g, overflow = oracle.OracleScene(default_gbuffer_materials(objs), flags=0).render_paths(cam, params, tape)
    assert overflow == 0
    o, overflow = oracle.OracleScene(objs, flags=REF_FLAGS).render_paths(cam, params, tape)
    assert overflow == 0
    for f in FIELDS:
        assert np.array_equal(g[f], o[f]), f
    assert np.array_equal(g["hit_object"], o["hit_object"])
    assert np.array_equal(g["radiance"].view(np.uint32), o["radiance"].view(np.uint32))


def test_live_reference_path_loop_when_built():
    """With oracle/_ref/libref_path*.so present (built from the reference's
    sources), compare on a fresh tape and a camera the fixtures do not use."""
    import reference_path
    if not (reference_path.available(True) and reference_path.available(False)):
        pytest.skip("reference path libraries not built (no reference sources)")
    import scenes
    objs = scenes.box_scene()
    cam = scenes.box_camera(24, 24)
    cam.position.x = 0.1
    params = ab.make_params(spp=3, max_depth=10)
    n = cam.width * cam.height * params.spp
    tape = (np.float32(1.0) - np.random.default_rng(77).random((n, 640), dtype=np.float32)).astype(np.float32)
    r, ov = reference_path.RefPathScene(objs, detmath=True).render_paths(cam, params, tape)
    o, ov2 = oracle.OracleScene(objs, flags=REF_FLAGS).render_paths(cam, params, tape)
    assert ov == 0 and ov2 == 0
    for f in FIELDS + ("hit_object",):
        assert np.array_equal(r[f], o[f]), f
    assert np.array_equal(r["radiance"].view(np.uint32), o["radiance"].view(np.uint32))
