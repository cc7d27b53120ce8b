"""Generate tests/golden/reference_guiding.npz: the reference's path-guiding
probe math on seeded inputs, run on the host from the build-time copy that
`make -C oracle ref-path` compiles (oracle/ref_path_harness.cu):

  faces    FaceNormal20FromIndex, its 20 face normals in its numbering
           (core/guiding/guiding_bin.cuh:40-66)
  voxel    GetVoxelGrid of points and directions (guiding_bin.cuh:102-114)
  dir/pdf  SampleOctahedronHemisphere of 8 probes (random RGB leaves with
           their mips) for random normals, texel weights and uniforms
           (core/guiding/octahedron.cuh:343-364)
  epdf     OctahedronHemispherePDF of random directions (octahedron.cuh:366-380)

The inputs are stored beside the outputs.  Run from the repository root after
`make -C oracle ref-path`:
    python tests/golden/make_reference_guiding_fixture.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "aperturerendererv3-optix-geometry_b200"), os.path.join(ROOT, "oracle")]

import guiding_oracle  # noqa: E402
import reference_path  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_guiding.npz")


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def inputs(seed: int = 20251204, nprobes: int = 8, n: int = 8000):
    rng = np.random.default_rng(seed)
    texels = np.zeros((nprobes, 85, 4), np.float32)
    for p in range(nprobes):
        leaves = rng.exponential(1.0, (64, 3)) * (rng.random((64, 1)) < 0.8)   # some empty texels
        texels[p, :, :3] = guiding_oracle.build_mips(leaves).astype(np.float32)
    probe_of = rng.integers(0, nprobes, n).astype(np.int32)
    normal = unit(rng, n)
    q = rng.uniform(0.05, 1.0, (n, 3))
    query = (q / q.sum(axis=1, keepdims=True)).astype(np.float32)
    u5 = (np.float32(1.0) - rng.random((n, 5), dtype=np.float32)).astype(np.float32)
    eval_dir = unit(rng, n)
    pos = rng.uniform(-5.0, 5.0, (n, 3)).astype(np.float32)
    return dict(texels=texels, probe_of=probe_of, normal=normal, query=query, u5=u5, eval_dir=eval_dir, pos=pos)


def main():
    x = inputs()
    d, p, e = reference_path.guiding_sample(x["texels"], x["probe_of"], x["normal"], x["query"], x["u5"],
                                            x["eval_dir"])
    out = dict(x)
    out.update(faces=reference_path.guiding_faces(), voxel=reference_path.guiding_voxel(x["pos"], x["eval_dir"]),
               dir=d, pdf=p, epdf=e)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
