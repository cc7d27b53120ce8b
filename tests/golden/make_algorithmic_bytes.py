"""Generate tests/golden/algorithmic_bytes.json: bytes per BVH query of the
reference algorithm on the benchmark scene (config 2).

Per query, B = 32 * V_node + 40 * V_prim, where V_node / V_prim are the node
visits and primitive tests of TraverseBVH (core/render/intersection.cuh:235-370)
on the reference's binned-SAH binary BVH (BuildBVH, core/bvh/bvh.cuh:142-422,
12 bins, leaf size 8, 32-byte nodes) with a standard slab test; 40 = a 36-byte
world-space triangle plus its 4-byte index.  Triangle proxies are centred on the
triangle bounds: with the reference's own proxies (every triangle of a mesh
centred at the mesh position, core/helper/scene_helper.h:488-545) the builder
puts a whole 1280-triangle icosphere into one leaf, which would inflate B by two
orders of magnitude.  The sampled queries are the extension rays and shadow
segments of the CPU path loop over 64 pixel strips of the 1920x1080 image at
1 spp, max depth 12.

Run from the repository root:  python tests/golden/make_algorithmic_bytes.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "aperturerendererv3-optix-geometry_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
import scenes  # noqa: E402
from aperture_b200 import make_params  # noqa: E402


def main():
    objs = scenes.spheres_scene()
    cam = scenes.spheres_camera(1920, 1080)
    p = make_params(spp=1, max_depth=12)
    osc = oracle.OracleScene(objs)
    npix = cam.width * cam.height
    ext, sh = [], []
    for k in range(64):
        b = (k * npix) // 64
        e, s = oracle.collect_rays(osc, cam, p, b, b + 512, cap=200_000)
        ext.append(e)
        sh.append(s)
    ext = np.concatenate(ext)
    sh = np.concatenate(sh)
    out = {"scene": "config2 spheres_scene() seed 0xA11CE+2, camera spheres_camera(1920,1080), 1 spp, depth 12",
           "node_bytes": 32, "prim_bytes": 40, "pixels_sampled": 64 * 512}
    for name, rays, any_hit in (("extension", ext, False), ("shadow", sh, True)):
        _, _, nv, pt = osc.trace(rays, any_hit=any_hit, counters=True,
                                 mode=oracle.TIE_LOWEST_INDEX | oracle.SLAB_STANDARD)
        out[name] = {"queries": int(len(rays)), "mean_node_visits": float(nv.mean()),
                     "mean_prim_tests": float(pt.mean()),
                     "bytes_per_query": float(32 * nv.mean() + 40 * pt.mean())}
    out["queries_per_path"] = (len(ext) + len(sh)) / (64 * 512)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "algorithmic_bytes.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
