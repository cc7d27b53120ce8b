"""The oracle against the reference renderer's own code.

tests/golden/reference_queries.npz holds outputs of the reference's
BuildBVH, light table, TraverseBVH (closest and any hit), AnyHitSegmentBVH,
Overlap, BSDF_PDF, INTERSECT_EPS and tone curves, compiled from the reference's headers and
run on the host (tests/golden/make_reference_fixtures.py).  The oracle must
reproduce them:

* BVH nodes, leaf order and light table: bit for bit (the oracle's
  PROXY_OBJECT_CENTER option gives the reference's triangle proxies).
* Closest hits in the reference's traversal mode (first-found ties, the
  reference's slab test): the same object for every ray except coplanar ties;
  triangle hits bit for bit (distance, position); cube and sphere hits within
  a small relative error.  The reference normalises with rsqrtf, the oracle
  with 1/sqrtf (the fixed rounding contract of this project): a 1-ulp
  difference in the local ray direction that the sphere quadratic amplifies.
* Any-hit flags, segment occlusion, Overlap and the INTERSECT_EPS table:
  exactly.  BSDF_PDF: within 2e-6 relative (normalisation as above).

When oracle/_ref/libref.so is present (built from the reference sources with
`make -C oracle ref`) the last test also compares on fresh random queries.
"""
import hashlib
import os

import numpy as np
import pytest

import oracle
import reference
from aperture_b200 import Material, Vec3

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "reference_queries.npz")


@pytest.fixture(scope="module")
def fx():
    return np.load(FIX)


def fixture_scenes():
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_reference_fixtures import fixture_scenes as fs
    return fs()


SCENES = ["box", "spheres"]


@pytest.fixture(scope="module")
def scene_objs(fx):
    out = {}
    for name, (objs, _, _) in fixture_scenes().items():
        digest = np.frombuffer(hashlib.sha256(objs.tobytes()).digest(), np.uint8)
        assert np.array_equal(digest, fx[f"{name}_sha256"]), f"scene generator changed for {name}"
        out[name] = objs
    return out


def _oracle(objs):
    return oracle.OracleScene(objs, flags=oracle.PROXY_OBJECT_CENTER)


REF_MODE = oracle.TIE_FIRST_FOUND | oracle.SLAB_REFERENCE


def _u32(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("name", SCENES)
def test_bvh_and_lights_bit_exact(fx, scene_objs, name):
    osc = _oracle(scene_objs[name])
    b6, l4 = osc.nodes()
    assert np.array_equal(_u32(b6), _u32(fx[f"{name}_node_bounds"]))
    assert np.array_equal(l4, fx[f"{name}_node_links"])
    assert np.array_equal(osc.indices(), fx[f"{name}_indices"])
    lo, lp = osc.lights()
    assert np.array_equal(lo, fx[f"{name}_light_object"])
    assert np.array_equal(_u32(lp), _u32(fx[f"{name}_light_prob"]))


def _coplanar_tie(objs, rays, k, a, b):
    """Objects a and b are hit at the same distance (to 1e-6) along ray k."""
    ta = oracle.OracleScene(objs[[a]], flags=oracle.PROXY_OBJECT_CENTER).trace(rays[k:k + 1])[1]
    tb = oracle.OracleScene(objs[[b]], flags=oracle.PROXY_OBJECT_CENTER).trace(rays[k:k + 1])[1]
    return abs(float(ta[0]) - float(tb[0])) <= 1e-6 * max(1.0, abs(float(ta[0])))


@pytest.mark.parametrize("name", SCENES)
def test_closest_hits_match_reference(fx, scene_objs, name):
    objs = scene_objs[name]
    rays = fx[f"{name}_rays"]
    ref_obj = fx[f"{name}_hit_object"]
    obj, t, pos, nrm, ins = _oracle(objs).trace_detail(rays, mode=REF_MODE)
    diff = np.nonzero(obj != ref_obj)[0]
    for k in diff:
        assert ref_obj[k] >= 0 and obj[k] >= 0 and _coplanar_tie(objs, rays, k, ref_obj[k], obj[k]), k
    assert len(diff) <= 2
    same = (obj == ref_obj) & (ref_obj >= 0)
    tri = same & (objs["type"][np.maximum(ref_obj, 0)] == 3)
    ana = same & ~tri
    assert tri.sum() > 500
    assert np.array_equal(_u32(t[tri]), _u32(fx[f"{name}_hit_t"][tri]))
    assert np.array_equal(_u32(pos[tri]), _u32(fx[f"{name}_hit_pos"][tri]))
    np.testing.assert_allclose(nrm[tri], fx[f"{name}_hit_normal"][tri], rtol=0, atol=2.5e-7)
    if ana.any():
        np.testing.assert_allclose(t[ana], fx[f"{name}_hit_t"][ana], rtol=2e-4)
        np.testing.assert_allclose(pos[ana], fx[f"{name}_hit_pos"][ana], rtol=0, atol=5e-4)
        np.testing.assert_allclose(nrm[ana], fx[f"{name}_hit_normal"][ana], rtol=0, atol=2e-4)
    miss = ref_obj < 0
    assert np.all(obj[miss] < 0)


@pytest.mark.parametrize("name", SCENES)
def test_any_hit_segments_overlap_match_reference(fx, scene_objs, name):
    osc = _oracle(scene_objs[name])
    any_obj, _ = osc.trace(fx[f"{name}_any_rays"], any_hit=True, mode=REF_MODE)
    assert np.array_equal((any_obj >= 0).astype(np.int8), fx[f"{name}_any_hit"])
    occ = osc.segments_occluded(fx[f"{name}_segments"], fx[f"{name}_segment_depth"], mode=REF_MODE)
    assert np.array_equal(occ.astype(np.int8), fx[f"{name}_segment_occluded"])
    assert np.array_equal(osc.overlap(fx[f"{name}_overlap_points"]), fx[f"{name}_overlap_object"])


def test_intersect_eps_table(fx):
    L = oracle.load()
    ours = [np.float32(1e-3) * np.float32(L.or_expf(float(min(d * 0.5, 4.0)))) for d in range(10)]
    assert np.array_equal(_u32(np.array(ours, np.float32)), _u32(fx["intersect_eps"]))


def _material(fx, i):
    m = Material()
    m.shading_model = int(fx["bsdf_model"][i])
    m.albedo = Vec3(*fx["bsdf_albedo"][i].tolist())
    m.specular, m.metallic, m.roughness = (float(x) for x in fx["bsdf_smr"][i])
    m.ior, m.sigma_a = 1.5, 1.0
    return m


def test_bsdf_pdf_matches_reference(fx):
    got = np.array([oracle.bsdf_pdf(int(fx["bsdf_model"][i]), _material(fx, i), *fx["bsdf_dirs"][i])
                    for i in range(len(fx["bsdf_model"]))], np.float32)
    np.testing.assert_allclose(got, fx["bsdf_pdf"], rtol=2e-6, atol=0)
    assert np.count_nonzero(fx["bsdf_pdf"]) > 100


@pytest.mark.skipif(not reference.available(), reason="oracle/_ref/libref.so not built (needs the reference sources)")
def test_live_against_reference_build(scene_objs):
    """Fresh queries against the reference build itself."""
    rng = np.random.default_rng(99)
    objs = scene_objs["spheres"]
    rs = reference.RefScene(objs)
    osc = _oracle(objs)
    rays = np.zeros((20_000, 8), np.float32)
    rays[:, :3] = rng.uniform(-22, 22, (len(rays), 3))
    d = rng.normal(size=(len(rays), 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3], rays[:, 7] = 1e-4, np.inf
    r_obj, r_t, *_ = rs.trace(rays)
    o_obj, o_t, *_ = osc.trace_detail(rays, mode=REF_MODE)
    assert (r_obj == o_obj).mean() > 0.9995
    tri = (r_obj == o_obj) & (r_obj >= 0) & (objs["type"][np.maximum(r_obj, 0)] == 3)
    assert np.array_equal(_u32(r_t[tri]), _u32(o_t[tri]))
    seg = rng.uniform(-23, 23, (20_000, 6)).astype(np.float32)
    dep = rng.integers(0, 12, len(seg)).astype(np.int32)
    assert np.array_equal(rs.segments_occluded(seg, dep), osc.segments_occluded(seg, dep, mode=REF_MODE))


@pytest.mark.parametrize("tone", [0, 1, 2])
@pytest.mark.parametrize("xyz", [0, 1])
def test_tonemap_matches_reference(fx, tone, xyz):
    """The Tonemap kernel's packed 0xAARRGGBB output: identical except where
    the fixed powf and the host powf round differently across a 1/255 step
    (at most 1 LSB, on a few pixels in 10^4)."""
    got = oracle.tonemap(fx["tonemap_hdr"], tone, 1.7, bool(xyz))
    ref = fx[f"tonemap_t{tone}_x{xyz}"]
    diff = got != ref
    assert diff.mean() <= 5e-4
    for shift in (24, 16, 8, 0):
        d = ((got >> shift) & 255).astype(np.int32) - ((ref >> shift) & 255).astype(np.int32)
        assert np.abs(d).max() <= 1


def test_sdf_objects_match_reference(fx):
    """SDF intersection (sphere tracing in the object's box, central-difference
    normal) of an analytic torus and a grid-sampled torus at loop depths 0 and
    5: the same rays hit; distance within 2e-6 relative and normal within 2e-5
    (the normalisation of the local ray direction differs, as for spheres).
    The grid itself (FillSDFVolume of the torus functor) is bit-identical."""
    import scenes
    objs, vols = scenes.sdf_box_scene()
    assert np.array_equal(np.frombuffer(hashlib.sha256(objs.tobytes()).digest(), np.uint8), fx["sdf_sha256"])
    osc = oracle.OracleScene(objs, volumes=vols, flags=oracle.PROXY_OBJECT_CENTER)
    grid = osc.volume_grid(0, tuple(vols[0][0].dims))
    assert np.array_equal(np.frombuffer(hashlib.sha256(grid.tobytes()).digest(), np.uint8), fx["sdf_grid_sha256"])
    rays = fx["sdf_rays"]
    for obj in (len(objs) - 2, len(objs) - 1):
        for depth in (0, 5):
            ref = fx[f"sdf_o{obj}_d{depth}"]
            t, pos, nrm = osc.object_isect(obj, rays, depth)
            hit = ref[:, 0] >= 0
            assert hit.sum() > 150
            assert np.array_equal(t >= 0, hit)
            np.testing.assert_allclose(t[hit], ref[hit, 0], rtol=2e-6)
            np.testing.assert_allclose(pos[hit], ref[hit, 1:4], rtol=0, atol=2e-6)
            np.testing.assert_allclose(nrm[hit], ref[hit, 4:7], rtol=0, atol=2e-5)
