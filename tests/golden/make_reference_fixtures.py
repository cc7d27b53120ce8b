"""Generate tests/golden/reference_queries.npz: outputs of the reference
renderer's own code on two seeded scenes, to pin the oracle and the CUDA core.

The reference functions are compiled from the reference's headers by
`make -C oracle ref` (oracle/ref_harness.cu -> oracle/_ref/libref.so) and run
on the host here: SceneObject construction and BuildBVH (core/bvh/bvh.cuh),
the light table of UpdateSceneToDeviceIfDirty (core/scene.cu:1046-1080),
TraverseBVH closest and any hit (core/render/intersection.cuh:235-370),
AnyHitSegmentBVH (372-397), Overlap (399-414), BSDF_PDF (RGB,
core/render/material.cuh:332-387), INTERSECT_EPS (core/config.cuh:3) and the
Tonemap kernel's curves (core/tonemap.cuh) at exposure 1.7, and the SDF
intersector (IntersectBase / sdf::IntersectSDFObject with the torus and
volume functors, core/object/sdf/) with the grid FillSDFVolume writes, and the
spectral pieces (RGBEncode / LambdaEncode, SampleCIE1931, D65Norm,
LambdaToCIE1931_XYZ).

Scenes: config 1 (scenes.box_scene()) and a small sphere field
(scenes.spheres_scene(n_spheres=24, n_lights=4, box=20, subdivisions=1):
1920 triangles + ground quad + 4 analytic light spheres).  Each scene's
object array is recorded by its SHA-256 so that a changed generator is caught.

Run from the repository root after `make -C oracle ref`:
    python tests/golden/make_reference_fixtures.py
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "aperturerendererv3-optix-geometry_b200"), os.path.join(ROOT, "oracle")]

import reference  # noqa: E402
import scenes  # noqa: E402
from aperture_b200 import Material, Vec3  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_queries.npz")


def fixture_scenes():
    return {
        "box": (scenes.box_scene(), -0.7, 0.7),
        "spheres": (scenes.spheres_scene(n_spheres=24, n_lights=4, box=20.0, subdivisions=1), -22.0, 22.0),
    }


def random_rays(rng, n, lo, hi, tmin=1e-4):
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmin
    r[:, 4:7] = d
    r[:, 7] = np.inf
    return r


def object_points(rng, objs, n):
    """Points around the centres of the analytic objects (cubes, spheres) --
    the only ones Overlap can report -- and of random other objects."""
    c = np.stack([objs["center"][f] for f in "xyz"], -1)
    e = np.stack([objs["extent"][f] for f in "xyz"], -1)
    analytic = np.nonzero(objs["type"] <= 1)[0]
    k = np.where(rng.random(n) < 0.75, rng.choice(analytic, n), rng.integers(0, len(objs), n))
    return (c[k] + rng.uniform(-1.5, 1.5, (n, 3)) * np.maximum(e[k], 0.02)).astype(np.float32)


def main():
    out = {}
    rng = np.random.default_rng(20251203)
    for name, (objs, lo, hi) in fixture_scenes().items():
        rs = reference.RefScene(objs)
        b6, l4 = rs.nodes()
        lo_obj, lo_prob = rs.lights()
        rays = random_rays(rng, 2000, lo, hi)
        obj, t, pos, nrm, ins = rs.trace(rays)
        any_rays = random_rays(rng, 1000, lo, hi)
        any_rays[:, 7] = rng.uniform(0.05, (hi - lo) * 0.6, len(any_rays))
        any_obj = rs.trace(any_rays, any_hit=True)[0]
        seg = rng.uniform(lo * 1.05, hi * 1.05, (2000, 6)).astype(np.float32)
        depth = rng.integers(0, 12, len(seg)).astype(np.int32)
        occ = rs.segments_occluded(seg, depth)
        pts = object_points(rng, objs, 600)
        ovl = rs.overlap(pts)
        p = f"{name}_"
        out.update({
            p + "sha256": np.frombuffer(hashlib.sha256(objs.tobytes()).digest(), np.uint8),
            p + "node_bounds": b6, p + "node_links": l4, p + "indices": rs.indices(),
            p + "light_object": lo_obj, p + "light_prob": lo_prob,
            p + "rays": rays, p + "hit_object": obj, p + "hit_t": t, p + "hit_pos": pos, p + "hit_normal": nrm,
            p + "hit_inside": ins,
            p + "any_rays": any_rays, p + "any_hit": (any_obj >= 0).astype(np.int8),
            p + "segments": seg, p + "segment_depth": depth, p + "segment_occluded": occ.astype(np.int8),
            p + "overlap_points": pts, p + "overlap_object": ovl,
        })
    out["intersect_eps"] = np.array([reference.intersect_eps(d) for d in range(10)], np.float32)

    n = 600
    model = rng.choice([0, 1, 2, 3], n).astype(np.int32)
    albedo = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    spec = rng.uniform(0, 1, (n, 3)).astype(np.float32)       # specular, metallic, roughness
    spec[:, 2] = rng.uniform(0.01, 1.0, n)
    dirs = rng.normal(size=(n, 3, 3))
    dirs /= np.linalg.norm(dirs, axis=2, keepdims=True)
    dirs = dirs.astype(np.float32)                              # N, ray direction, light direction
    pdf = np.zeros(n, np.float32)
    for i in range(n):
        m = Material()
        m.shading_model = int(model[i])
        m.albedo = Vec3(*albedo[i].tolist())
        m.specular, m.metallic, m.roughness = (float(x) for x in spec[i])
        m.ior, m.sigma_a = 1.5, 1.0
        pdf[i] = reference.bsdf_pdf(int(model[i]), m, dirs[i, 0], dirs[i, 1], dirs[i, 2])
    out.update({"bsdf_model": model, "bsdf_albedo": albedo, "bsdf_smr": spec, "bsdf_dirs": dirs, "bsdf_pdf": pdf})

    # Tonemap kernel (core/scene.cu:180-199) with Gamma / ACES / XYZ2SRGBLinearD65
    hdr = np.exp(rng.normal(-1.0, 2.0, (4000, 3))).astype(np.float32)
    hdr[:100] = 0.0
    out["tonemap_hdr"] = hdr
    for tone in (0, 1, 2):
        for xyz in (0, 1):
            out[f"tonemap_t{tone}_x{xyz}"] = reference.tonemap(hdr, tone, 1.7, bool(xyz))
    # SDF objects (IntersectBase -> sdf::IntersectSDFObject): an analytic torus and
    # a torus sampled on a 64^3 grid (FillSDFVolume), at loop depths 0 and 5
    objs, vols = scenes.sdf_box_scene()
    rs = reference.RefScene(objs)
    dims = tuple(vols[0][0].dims)
    grid = reference.fill_torus(dims, vols[0][0].fill_info[0], vols[0][0].fill_info[1])
    out["sdf_sha256"] = np.frombuffer(hashlib.sha256(objs.tobytes()).digest(), np.uint8)
    out["sdf_grid_sha256"] = np.frombuffer(hashlib.sha256(grid.tobytes()).digest(), np.uint8)
    rays = []
    for obj in (len(objs) - 2, len(objs) - 1):     # aimed at points inside each object's box
        c = np.array([objs["center"][obj][f] for f in "xyz"])
        e = np.array([objs["extent"][obj][f] for f in "xyz"])
        o = rng.uniform(-0.55, 0.55, (500, 3))
        d = c + rng.uniform(-1, 1, (500, 3)) * e - o
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        r = np.zeros((500, 8), np.float32)
        r[:, :3], r[:, 4:7], r[:, 3], r[:, 7] = o, d, 1e-4, np.inf
        rays.append(r)
    rays = np.concatenate(rays)
    out["sdf_rays"] = rays
    for obj in (len(objs) - 2, len(objs) - 1):
        for depth in (0, 5):
            t, pos, nrm = rs.object_isect(obj, rays, depth, grid, dims)
            out[f"sdf_o{obj}_d{depth}"] = np.concatenate([t[:, None], pos, nrm], 1).astype(np.float32)
    # spectral: the reference's encoders on its own self-test inputs, wavelength
    # sampling for uniform triples, D65 and colour-matching weights there
    import spectral_tables
    tab, it, gt = spectral_tables.load()
    rk, lk = reference.spectral_encode(it[:3].T.copy(), it[3].copy())
    out["spec_rgb_k"], out["spec_lam_k"] = rk, lk
    u3 = rng.random((500, 3)).astype(np.float32)
    lam, pdf = reference.spectral_sample(u3)
    d65, xyz = reference.spectral_weights(lam)
    out.update({"spec_u3": u3, "spec_lambda": lam, "spec_pdf": pdf, "spec_d65": d65, "spec_xyz": xyz,
                "spec_tables_sha256": np.frombuffer(hashlib.sha256(tab.tobytes()).digest(), np.uint8)})
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
