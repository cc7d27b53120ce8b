"""The oracle itself, on the CPU: its BVH traversal against a brute-force scan,
the structure of the reference BVH it builds, its light table, its fixed math
functions against float64 numpy, and the committed algorithmic-bytes fixture.

These checks pin the parts of the oracle that the GPU parity tests lean on.
"""
import json
import os

import numpy as np
import pytest

import oracle
import scenes
from test_gpu_trace import random_rays

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def box_oracle(box_objects):
    return oracle.OracleScene(box_objects)


@pytest.fixture(scope="module")
def spheres_oracle(small_spheres_objects):
    return oracle.OracleScene(small_spheres_objects)


def _bits(t):
    return np.ascontiguousarray(t, np.float32).view(np.uint32)


@pytest.mark.parametrize("which", ["box", "spheres"])
def test_bvh_closest_hit_equals_brute_force(which, box_oracle, spheres_oracle):
    osc, lo, hi = (box_oracle, -0.7, 0.7) if which == "box" else (spheres_oracle, -25.0, 25.0)
    rays = random_rays(20_000 if which == "box" else 5_000, lo, hi, 11)
    obj, t = osc.trace(rays)
    bobj, bt = osc.trace_brute(rays)
    assert np.array_equal(obj, bobj)
    hit = bobj >= 0
    assert hit.mean() > 0.2
    assert np.array_equal(_bits(t[hit]), _bits(bt[hit]))


@pytest.mark.parametrize("which", ["box", "spheres"])
def test_bvh_any_hit_agrees_with_closest_hit(which, box_oracle, spheres_oracle):
    osc, lo, hi = (box_oracle, -0.7, 0.7) if which == "box" else (spheres_oracle, -25.0, 25.0)
    rays = random_rays(20_000 if which == "box" else 5_000, lo, hi, 12)
    rays[:, 7] = np.random.default_rng(13).uniform(0.05, 1.5 if which == "box" else 30.0, len(rays))
    any_obj, _ = osc.trace(rays, any_hit=True)
    bobj, _ = osc.trace_brute(rays)
    assert np.array_equal(any_obj >= 0, bobj >= 0)


def test_reference_traversal_differs_only_on_ties(box_oracle):
    """First-found ties (the reference's rule) and lowest-index ties pick
    objects at the same distance; only coplanar primitives can differ."""
    rays = random_rays(20_000, -0.7, 0.7, 14)
    o_ref, t_ref = box_oracle.trace(rays, mode=oracle.TIE_FIRST_FOUND | oracle.SLAB_REFERENCE)
    o_low, t_low = box_oracle.trace(rays)
    hit = o_low >= 0
    assert np.array_equal(o_ref >= 0, hit)
    assert np.array_equal(_bits(t_ref[hit]), _bits(t_low[hit]))
    assert (o_ref == o_low).mean() > 0.98


def test_reference_bvh_structure(spheres_oracle, small_spheres_objects):
    """BuildBVH invariants: a permutation of the primitives in leaves of at most
    8, each child box inside its parent's, every leaf box around its triangles."""
    b, l = spheres_oracle.nodes()
    idx = spheres_oracle.indices()
    n = len(small_spheres_objects)
    assert np.array_equal(np.sort(idx), np.arange(n))
    leaves = l[:, 3] > 0
    assert l[leaves, 3].max() <= 8
    assert l[leaves, 3].sum() == n
    inner = np.nonzero(~leaves)[0]
    for c in (0, 1):
        ch = l[inner, c]
        assert np.all(b[ch, :3] >= b[inner, :3]) and np.all(b[ch, 3:] <= b[inner, 3:])
    tri = small_spheres_objects["type"] == 3
    world = _triangle_world_vertices(small_spheres_objects)
    for k in np.nonzero(leaves)[0][:400]:
        prims = idx[l[k, 2]:l[k, 2] + l[k, 3]]
        for p in prims:
            if tri[p]:
                v = world[p]
                assert np.all(v.min(0) >= b[k, :3] - 1e-4) and np.all(v.max(0) <= b[k, 3:] + 1e-4)


def _triangle_world_vertices(objs):
    """Triangle vertices in world space (object rotation is identity in the
    sphere scene; the centre is added)."""
    pos = np.stack([np.stack([objs["tri"][:, k]["position"][f] for f in "xyz"], -1) for k in range(3)], 1)
    c = np.stack([objs["center"][f] for f in "xyz"], -1)
    assert np.all(np.stack([objs["rotation_deg"][f] for f in "xyz"], -1) == 0)
    return pos + c[:, None, :]


def test_light_table(spheres_oracle, small_spheres_objects):
    lobj, prob = spheres_oracle.lights()
    assert len(lobj) == 8
    assert np.all(small_spheres_objects["material"]["shading_model"][lobj] == 1)
    assert abs(float(prob.astype(np.float64).sum()) - 1.0) < 1e-5
    assert np.all(prob > 0)


def _ulps(got, ref):
    got = np.asarray(got, np.float64)
    sp = np.spacing(np.abs(ref.astype(np.float32))).astype(np.float64)
    return float(np.max(np.abs(got - ref) / sp))


def test_fixed_math_accuracy():
    """The fixed sin/cos/exp/log/pow that both the GPU and the oracle use
    (Cody-Waite reduction + Taylor series) stay within a few ulp."""
    L = oracle.load()
    rng = np.random.default_rng(0)
    x = rng.uniform(-100, 100, 4000).astype(np.float32)
    assert _ulps([L.or_sinf(float(v)) for v in x], np.sin(x.astype(np.float64))) <= 2.0
    assert _ulps([L.or_cosf(float(v)) for v in x], np.cos(x.astype(np.float64))) <= 2.0
    e = rng.uniform(-80, 80, 4000).astype(np.float32)
    assert _ulps([L.or_expf(float(v)) for v in e], np.exp(e.astype(np.float64))) <= 1.0
    g = np.exp(rng.uniform(-80, 80, 4000)).astype(np.float32)
    assert _ulps([L.or_logf(float(v)) for v in g], np.log(g.astype(np.float64))) <= 2.0
    b = rng.uniform(0.01, 10, 4000).astype(np.float32)
    p = rng.uniform(-5, 5, 4000).astype(np.float32)
    assert _ulps([L.or_powf(float(u), float(v)) for u, v in zip(b, p)],
                 np.power(b.astype(np.float64), p.astype(np.float64))) <= 32.0
    assert L.or_sinf(0.0) == 0.0 and L.or_expf(0.0) == 1.0 and L.or_logf(1.0) == 0.0
    assert L.or_powf(2.0, 10.0) == 1024.0


def test_algorithmic_bytes_fixture():
    """The committed roofline numerator: B = 32 V_node + 40 V_prim per query."""
    with open(os.path.join(GOLDEN, "algorithmic_bytes.json")) as f:
        ab = json.load(f)
    for k in ("extension", "shadow"):
        q = ab[k]
        assert q["queries"] > 10_000
        assert abs(q["bytes_per_query"] - (32 * q["mean_node_visits"] + 40 * q["mean_prim_tests"])) < 1e-6
        assert 100 < q["bytes_per_query"] < 10_000


def test_algorithmic_bytes_counters_small_sample():
    """The counters behind the fixture, on a tiny sample of the same workload:
    visits and tests are positive and an any-hit query never tests more
    primitives than the closest-hit query along the same segment."""
    objs = scenes.spheres_scene(n_spheres=60, n_lights=4, box=20.0)
    osc = oracle.OracleScene(objs)
    rays = random_rays(4000, -20, 20, 15)
    rays[:, 7] = 25.0
    _, _, nv, pt = osc.trace(rays, counters=True)
    _, _, nva, pta = osc.trace(rays, any_hit=True, counters=True)
    assert nv.min() >= 1 and pt.max() > 0
    assert np.all(pta <= pt)
