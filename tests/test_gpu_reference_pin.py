"""The CUDA core's ray queries against the reference renderer's own outputs
(tests/golden/reference_queries.npz, made by the reference's TraverseBVH over
its own BuildBVH; see tests/golden/make_reference_fixtures.py).

The core traverses its own 8-wide quantised BVH and breaks exact-distance ties
towards the lower object index, where the reference keeps the first primitive
its traversal finds; every other closest hit must name the same object, at the
same distance bit for bit for triangles (the reference's Moller-Trumbore
arithmetic) and within the rsqrtf-vs-1/sqrtf difference for cubes and spheres.
Any-hit flags must agree exactly.
"""
import hashlib
import os

import numpy as np
import pytest

import oracle
from aperture_b200 import Scene

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(HERE, "golden", "reference_queries.npz"))


def _scenes():
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_reference_fixtures import fixture_scenes
    return fixture_scenes()


def _u32(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["box", "spheres"])
def test_gpu_queries_match_reference(fx, name):
    objs = _scenes()[name][0]
    assert np.array_equal(np.frombuffer(hashlib.sha256(objs.tobytes()).digest(), np.uint8), fx[f"{name}_sha256"])
    scene = Scene(objs)
    rays = fx[f"{name}_rays"]
    ref_obj, ref_t = fx[f"{name}_hit_object"], fx[f"{name}_hit_t"]
    obj, t = scene.trace_rays(rays)
    for k in np.nonzero(obj != ref_obj)[0]:
        a, b = int(ref_obj[k]), int(obj[k])
        assert a >= 0 and b >= 0, k
        ta = oracle.OracleScene(objs[[a]]).trace(rays[k:k + 1])[1][0]
        tb = oracle.OracleScene(objs[[b]]).trace(rays[k:k + 1])[1][0]
        assert abs(float(ta) - float(tb)) <= 1e-6 * max(1.0, abs(float(ta))), k   # coplanar tie
        assert b < a                                                               # lowest index wins
    same = (obj == ref_obj) & (ref_obj >= 0)
    tri = same & (objs["type"][np.maximum(ref_obj, 0)] == 3)
    assert tri.sum() > 500
    assert np.array_equal(_u32(t[tri]), _u32(ref_t[tri]))
    ana = same & ~tri
    if ana.any():
        np.testing.assert_allclose(t[ana], ref_t[ana], rtol=2e-4)
    any_obj, _ = scene.trace_rays(fx[f"{name}_any_rays"], any_hit=True)
    assert np.array_equal((any_obj >= 0).astype(np.int8), fx[f"{name}_any_hit"])
