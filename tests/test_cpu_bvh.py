"""The BVH builder on the host alone (ar_bvh_build_info): structure checks that
need no GPU -- every primitive record in exactly one leaf slot, child indices
in range, one internal slot per node below the root -- and the shape the
SAH-optimal 8-wide collapse gives (slot fill, stack bound within the traversal
kernels' stack), on the scenes the GPU tests and the benchmark use and on
degenerate inputs."""
import numpy as np
import pytest

import scenes
from aperture_b200 import ArError, OBJECT_DTYPE, bvh_build_info

STACK_MAX = 128   # kStackShared + kStackOverflow entries per ray in the traversal kernels


def _check_shape(info, prims):
    assert info.prim_refs == prims
    assert info.internal_slots == info.wide_nodes - 1
    assert 1 <= info.leaf_slots <= prims
    assert 0 <= info.stack_bound < STACK_MAX
    assert info.depth >= 1


def test_box_scene():
    objs = scenes.box_scene()
    info = bvh_build_info(objs)
    _check_shape(info, len(objs))


def test_sphere_field_slot_fill():
    """40 icospheres of 1280 triangles + ground + 16 lights: the collapse plan
    fills most of the 8 slots of a node (the greedy collapse left fewer than 4)."""
    objs = scenes.spheres_scene(n_spheres=40)
    info = bvh_build_info(objs)
    _check_shape(info, len(objs))
    slots = info.leaf_slots + info.internal_slots
    assert slots / info.wide_nodes > 5.0


def test_sdf_scene_with_volumes():
    """Signed-distance objects are tested after traversal, not in the BVH."""
    objs, vols = scenes.sdf_box_scene(grid=16)
    info = bvh_build_info(objs, volumes=vols)
    n_sdf = int(np.sum(np.asarray(objs["type"]) == 2))
    assert n_sdf == 2
    _check_shape(info, len(objs) - n_sdf)


def test_coincident_centroids():
    """64 identical spheres: every split position ties; the build still ends
    with valid leaves of at most 4 records."""
    objs = scenes.sphere_objects([(0.5, 0.5, 0.5)] * 64, [0.25] * 64)
    scenes.diffuse(objs, (0.5, 0.5, 0.5))
    info = bvh_build_info(objs)
    _check_shape(info, 64)
    assert info.leaf_slots >= 16


def test_single_object_and_empty():
    one = scenes.sphere_objects([(0.0, 0.0, 0.0)], [1.0])
    scenes.diffuse(one, (0.5, 0.5, 0.5))
    info = bvh_build_info(one)
    assert (info.wide_nodes, info.prim_refs, info.leaf_slots, info.internal_slots) == (1, 1, 1, 0)
    empty = np.zeros(0, dtype=OBJECT_DTYPE)
    info = bvh_build_info(empty)
    assert (info.wide_nodes, info.prim_refs) == (0, 0)


def test_invalid_object_rejected():
    objs = scenes.sphere_objects([(0.0, 0.0, 0.0), (1.0, 0.0, 0.0)], [1.0, 1.0])
    scenes.diffuse(objs, (0.5, 0.5, 0.5))
    objs[1]["center"]["x"] = np.nan
    with pytest.raises(ArError) as e:
        bvh_build_info(objs)
    assert e.value.status == 1
