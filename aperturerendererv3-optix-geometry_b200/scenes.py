"""Seeded synthetic scenes of the benchmark configurations.

Every scene is an array of ar_object_desc (aperture_b200.OBJECT_DTYPE) built
the way the reference builds scenes: one SceneObject per primitive; a triangle
mesh is a run of OBJ_TRIANGLE objects whose centre is the mesh position and
whose vertices are in object space (core/helper/scene_helper.h:453-545).
Materials follow the reference factories (core/render/object.cuh:124-217).

Generators use numpy's PCG64 with seed 0xA11CE + config number.
  box_scene     -- config 1: unit box, 2 seeded cubes, ceiling light, 256^2.
  spheres_scene -- config 2: 800 icospheres x 1280 triangles (+ ground quad,
                   16 emissive spheres), 1920x1080.
  sdf_box_scene -- config 1 plus two signed-distance tori (object/sdf): an
                   analytic one and one sampled on a grid (float or half).
"""
from __future__ import annotations

import numpy as np

from aperture_b200 import (MAT_DIFFUSE, MAT_GGX, MAT_GLASS, MAT_LIGHT, OBJ_CUBE, OBJ_SDF, OBJ_SPHERE, OBJ_TRIANGLE,
                           OBJECT_DTYPE, SDF_TORUS, SDF_VOLUME, make_camera, make_volume, set_sdf)

SEED_BASE = 0xA11CE
THICK = 0.01  # SceneHelper::THICK (scene_helper.h:14)


def _empty(n: int) -> np.ndarray:
    a = np.zeros(n, OBJECT_DTYPE)
    a["visible"] = 1
    m = a["material"]
    m["ior"] = 1.5
    m["sigma_a"] = 100.0
    m["abbe_number"] = 20.0
    return a


def _set3(field, values) -> None:
    v = np.asarray(values, np.float32)
    field["x"] = v[..., 0]
    field["y"] = v[..., 1]
    field["z"] = v[..., 2]


def diffuse(a: np.ndarray, albedo) -> None:
    """Material::CreateDiffusePureColor"""
    a["material"]["shading_model"] = MAT_DIFFUSE
    _set3(a["material"]["albedo"], np.broadcast_to(np.asarray(albedo, np.float32), (len(a), 3)))


def light(a: np.ndarray, emissive) -> None:
    """Material::CreateLight"""
    a["material"]["shading_model"] = MAT_LIGHT
    _set3(a["material"]["albedo"], np.zeros((len(a), 3), np.float32))
    _set3(a["material"]["emissive"], np.broadcast_to(np.asarray(emissive, np.float32), (len(a), 3)))


def ggx(a: np.ndarray, base_color, roughness, metallic, specular) -> None:
    """Material::CreateGGXPureColor (clamps as the factory does)"""
    m = a["material"]
    m["shading_model"] = MAT_GGX
    _set3(m["albedo"], np.broadcast_to(np.asarray(base_color, np.float32), (len(a), 3)))
    m["roughness"] = np.clip(np.asarray(roughness, np.float32), 0.01, 1.0)
    m["metallic"] = np.clip(np.asarray(metallic, np.float32), 0.0, 1.0)
    m["specular"] = np.clip(np.asarray(specular, np.float32), 0.0, 1.0)


def glass(a: np.ndarray, color, ior, sigma_a, abbe=20.0, tilt=0.0) -> None:
    """Material::CreateGlassPureColor"""
    m = a["material"]
    m["shading_model"] = MAT_GLASS
    _set3(m["albedo"], np.broadcast_to(np.asarray(color, np.float32), (len(a), 3)))
    m["ior"] = ior
    m["sigma_a"] = sigma_a
    m["abbe_number"] = abbe
    m["tilt_number"] = tilt


def triangles(positions: np.ndarray, normals: np.ndarray, center=(0.0, 0.0, 0.0), rotation=(0.0, 0.0, 0.0)) -> np.ndarray:
    """OBJ_TRIANGLE objects from object-space positions/normals [n, 3, 3]."""
    positions = np.asarray(positions, np.float32)
    normals = np.asarray(normals, np.float32)
    n = positions.shape[0]
    a = _empty(n)
    a["type"] = OBJ_TRIANGLE
    _set3(a["center"], np.broadcast_to(np.asarray(center, np.float32), (n, 3)))
    _set3(a["extent"], np.ones((n, 3), np.float32))
    _set3(a["rotation_deg"], np.broadcast_to(np.asarray(rotation, np.float32), (n, 3)))
    _set3(a["tri"]["position"], positions)
    _set3(a["tri"]["normal"], normals)
    return a


def quad(p0, p1, p2, p3, normal) -> tuple[np.ndarray, np.ndarray]:
    pos = np.array([[p0, p1, p2], [p0, p2, p3]], np.float32)
    nrm = np.broadcast_to(np.asarray(normal, np.float32), (2, 3, 3)).copy()
    return pos, nrm


def box_mesh(half) -> tuple[np.ndarray, np.ndarray]:
    """12 outward-facing triangles of an axis-aligned box centred at the origin."""
    hx, hy, hz = half
    c = np.array([[sx * hx, sy * hy, sz * hz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)], np.float32)
    # corner index = (sx>0)*4 + (sy>0)*2 + (sz>0)
    faces = [((4, 6, 7, 5), (1, 0, 0)), ((0, 1, 3, 2), (-1, 0, 0)), ((2, 3, 7, 6), (0, 1, 0)),
             ((0, 4, 5, 1), (0, -1, 0)), ((1, 5, 7, 3), (0, 0, 1)), ((0, 2, 6, 4), (0, 0, -1))]
    pos, nrm = [], []
    for (a, b, cc, d), n in faces:
        p, q = quad(c[a], c[b], c[cc], c[d], n)
        pos.append(p)
        nrm.append(q)
    return np.concatenate(pos), np.concatenate(nrm)


def cube_object(center, extent, rotation=(0.0, 0.0, 0.0)) -> np.ndarray:
    a = _empty(1)
    a["type"] = OBJ_CUBE
    _set3(a["center"], np.asarray([center], np.float32))
    _set3(a["extent"], np.asarray([extent], np.float32))
    _set3(a["rotation_deg"], np.asarray([rotation], np.float32))
    return a


def sphere_objects(centers, radii) -> np.ndarray:
    centers = np.asarray(centers, np.float32)
    n = centers.shape[0]
    a = _empty(n)
    a["type"] = OBJ_SPHERE
    _set3(a["center"], centers)
    r = np.asarray(radii, np.float32)
    _set3(a["extent"], np.stack([r, r, r], -1))
    return a


def box_scene(seed: int = SEED_BASE + 1, light_as: str = "cube") -> np.ndarray:
    """Config 1: five walls of the unit box [-0.5, 0.5]^3 (open towards +z),
    two seeded Y-rotated cubes (0.3 and 0.3x0.6x0.3) and a 0.25 x 0.25 ceiling
    light of radiance (17, 12, 4).  The light is a thin OBJ_CUBE (the reference's
    Cornell-box convention, scene_helper.h:68-73) because the reference's NEE
    samples only cubes and spheres; light_as="triangles" gives the 2-triangle quad."""
    rng = np.random.default_rng(seed)
    h = 0.5
    walls = [
        (quad((-h, -h, -h), (-h, -h, h), (h, -h, h), (h, -h, -h), (0, 1, 0)), (0.73, 0.73, 0.73)),   # floor
        (quad((-h, h, -h), (h, h, -h), (h, h, h), (-h, h, h), (0, -1, 0)), (0.73, 0.73, 0.73)),      # ceiling
        (quad((-h, -h, -h), (h, -h, -h), (h, h, -h), (-h, h, -h), (0, 0, 1)), (0.73, 0.73, 0.73)),   # back
        (quad((-h, -h, -h), (-h, h, -h), (-h, h, h), (-h, -h, h), (1, 0, 0)), (0.65, 0.05, 0.05)),   # left
        (quad((h, -h, -h), (h, -h, h), (h, h, h), (h, h, -h), (-1, 0, 0)), (0.12, 0.45, 0.15)),      # right
    ]
    parts = []
    for (pos, nrm), albedo in walls:
        t = triangles(pos, nrm)
        diffuse(t, albedo)
        parts.append(t)
    for half, xr, zr in (((0.15, 0.15, 0.15), (0.05, 0.25), (-0.05, 0.25)),
                         ((0.15, 0.30, 0.15), (-0.28, -0.05), (-0.32, -0.05))):
        cx = rng.uniform(*xr)
        cz = rng.uniform(*zr)
        yaw = rng.uniform(-45.0, 45.0)
        pos, nrm = box_mesh(half)
        t = triangles(pos, nrm, center=(cx, -h + half[1], cz), rotation=(0.0, yaw, 0.0))
        diffuse(t, (0.73, 0.73, 0.73))
        parts.append(t)
    if light_as == "cube":
        L = cube_object((0.0, h - THICK, 0.0), (0.125, THICK, 0.125))
    else:
        pos, nrm = quad((-0.125, h - 1e-3, -0.125), (0.125, h - 1e-3, -0.125), (0.125, h - 1e-3, 0.125),
                        (-0.125, h - 1e-3, 0.125), (0, -1, 0))
        L = triangles(pos, nrm)
    light(L, (17.0, 12.0, 4.0))
    parts.append(L)
    return np.concatenate(parts)


def box_camera(width=256, height=256):
    return make_camera((0.0, 0.0, 1.9), (0.0, 0.0, -1.0), 40.0, width, height)


def icosphere(subdivisions: int = 3) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: vertices [v, 3] (float64) and faces [f, 3]; 20 * 4^s faces."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = [np.array(p, np.float64) / np.linalg.norm(p) for p in verts]
    for _ in range(subdivisions):
        cache: dict[tuple[int, int], int] = {}

        def mid(a: int, b: int) -> int:
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(v), np.array(faces, np.int64)


def spheres_scene(seed: int = SEED_BASE + 2, n_spheres: int = 800, subdivisions: int = 3, n_lights: int = 16,
                  box: float = 100.0) -> np.ndarray:
    """Config 2: n_spheres icospheres (1280 triangles each at 3 subdivisions),
    radius U(0.5, 3), centres uniform in [-box, box]^3; materials 60% Lambert
    (albedo U(0.05, 0.9)^3), 30% GGX conductor (roughness U(0.05, 0.5), F0
    U(0.5, 1)^3), 10% glass (IOR 1.5, clear); a 2-triangle ground quad below the
    box; n_lights emissive analytic spheres of radiance U(5, 20)."""
    rng = np.random.default_rng(seed)
    V, F = icosphere(subdivisions)
    unit_pos = V[F].astype(np.float32)         # [f, 3, 3]
    unit_nrm = unit_pos.copy()
    nf = F.shape[0]
    radii = rng.uniform(0.5, 3.0, n_spheres).astype(np.float32)
    centers = rng.uniform(-box, box, (n_spheres, 3)).astype(np.float32)
    kind = rng.random(n_spheres)
    albedo = rng.uniform(0.05, 0.9, (n_spheres, 3)).astype(np.float32)
    rough = rng.uniform(0.05, 0.5, n_spheres).astype(np.float32)
    f0 = rng.uniform(0.5, 1.0, (n_spheres, 3)).astype(np.float32)
    a = triangles(np.tile(unit_pos, (n_spheres, 1, 1)) * np.repeat(radii, nf)[:, None, None],
                  np.tile(unit_nrm, (n_spheres, 1, 1)))
    _set3(a["center"], np.repeat(centers, nf, axis=0))
    m = a["material"]
    sid = np.repeat(np.arange(n_spheres), nf)
    lam = kind[sid] < 0.6
    met = (kind[sid] >= 0.6) & (kind[sid] < 0.9)
    gla = kind[sid] >= 0.9
    m["shading_model"] = np.where(lam, MAT_DIFFUSE, np.where(met, MAT_GGX, MAT_GLASS))
    alb = np.where(lam[:, None], albedo[sid], np.where(met[:, None], f0[sid], 1.0)).astype(np.float32)
    _set3(m["albedo"], alb)
    m["roughness"] = np.where(met, np.clip(rough[sid], 0.01, 1.0), 0.0)
    m["metallic"] = np.where(met, 1.0, 0.0)
    m["specular"] = np.where(met, 0.5, 0.0)
    m["ior"] = 1.5
    m["sigma_a"] = np.where(gla, 0.0, 100.0)
    g = 10.0 * box
    y = -box - 4.0
    pos, nrm = quad((-g, y, -g), (-g, y, g), (g, y, g), (g, y, -g), (0, 1, 0))
    ground = triangles(pos, nrm)
    diffuse(ground, (0.5, 0.5, 0.5))
    lc = rng.uniform(-box, box, (n_lights, 3)).astype(np.float32)
    lr = rng.uniform(0.5, 3.0, n_lights).astype(np.float32)
    le = rng.uniform(5.0, 20.0, n_lights).astype(np.float32)
    L = sphere_objects(lc, lr)
    light(L, np.stack([le, le, le], -1))
    return np.concatenate([a, ground, L])


def spheres_camera(width=1920, height=1080, fov=60.0):
    d = np.array([0.0, -40.0, 150.0])
    return make_camera((0.0, 30.0, -150.0), d / np.linalg.norm(d), fov, width, height)


def sdf_object(center, extent, rotation=(0.0, 0.0, 0.0), kind: int = SDF_TORUS, info=(0.375, 0.125, 0.0, 0.0),
               volume: int = 0) -> np.ndarray:
    """One OBJ_SDF object: the box [-extent, extent] around centre holds the
    unit-box signed distance (AdditionalObjectInfo / SDFInfo of the reference)."""
    a = _empty(1)
    a["type"] = OBJ_SDF
    _set3(a["center"], np.asarray([center], np.float32))
    _set3(a["extent"], np.asarray([extent], np.float32))
    _set3(a["rotation_deg"], np.asarray([rotation], np.float32))
    set_sdf(a[0:1], kind, info, volume)
    return a


def sdf_box_scene(seed: int = SEED_BASE + 3, precision: int = 32, grid: int = 64):
    """The config-1 box with a glass analytic torus and a GGX torus sampled on
    a grid^3 volume (FillSDFVolume of the torus functor), both rotated.
    Returns (objects, volumes) for Scene(objects, volumes=volumes)."""
    rng = np.random.default_rng(seed)
    base = box_scene()
    tor = sdf_object((0.18, -0.3, 0.12), (0.16, 0.16, 0.16), (20.0, float(rng.uniform(-40, 40)), 0.0), SDF_TORUS,
                     (0.3, 0.12, 0.0, 0.0))
    glass(tor, (0.95, 0.95, 0.95), 1.5, 0.5)
    vol = sdf_object((-0.2, -0.25, -0.05), (0.2, 0.15, 0.2), (0.0, float(rng.uniform(-40, 40)), -15.0), SDF_VOLUME,
                     (0.0, 0.0, 0.0, 0.0), 0)
    ggx(vol, (0.9, 0.6, 0.3), 0.3, 1.0, 0.5)
    volumes = [make_volume((grid, grid, grid), None, precision, SDF_TORUS, (0.32, 0.14, 0.0, 0.0))]
    return np.concatenate([base, tor, vol]), volumes


def fbm_density(seed: int = SEED_BASE + 3, n: int = 128, octaves: int = 6, base: int = 4) -> np.ndarray:
    """[n, n, n] float32 density in [0, 1]: fractal Brownian motion of seeded
    value noise (lattice values U(0, 1), trilinear), frequencies base * 2^o with
    gain 1/2, then a soft threshold that leaves clouds and clear gaps."""
    rng = np.random.default_rng(seed)
    x = (np.arange(n, dtype=np.float64) + 0.5) / n
    acc = np.zeros((n, n, n), np.float64)
    amp, norm = 1.0, 0.0
    for o in range(octaves):
        f = base << o
        lat = rng.random((f + 1, f + 1, f + 1))
        g = x * f
        i0 = np.minimum(np.floor(g).astype(np.int64), f - 1)
        t = g - i0
        # separable trilinear: interpolate along x, then y, then z
        a = lat[:, :, i0] * (1 - t) + lat[:, :, i0 + 1] * t
        a = a[:, i0, :] * (1 - t)[None, :, None] + a[:, i0 + 1, :] * t[None, :, None]
        a = a[i0, :, :] * (1 - t)[:, None, None] + a[i0 + 1, :, :] * t[:, None, None]
        acc += amp * a
        norm += amp
        amp *= 0.5
    v = acc / norm
    return np.clip((v - 0.42) * 4.0, 0.0, 1.0).astype(np.float32)


def medium_box_scene(seed: int = SEED_BASE + 3, precision: int = 16, grid: int = 256, medium_grid: int = 128):
    """Config 3: the SDF box scene (a grid^3 sampled torus, float or half) plus a
    heterogeneous medium filling the box: a medium_grid^3 fBm density (6
    octaves, seeded) scaled to sigma_t max 2.0, single-scatter albedo 0.8,
    Henyey-Greenstein g = 0.3.  Returns (objects, volumes, medium) where
    medium holds the keyword arguments of Scene.set_medium."""
    objects, volumes = sdf_box_scene(seed, precision, grid)
    d = fbm_density(seed, medium_grid)
    medium = dict(density=d.astype(np.float16 if precision == 16 else np.float32),
                  bounds_min=(-0.5, -0.5, -0.5), bounds_max=(0.5, 0.5, 0.5),
                  sigma_t_max=2.0, albedo=(0.8, 0.8, 0.8), g=0.3)
    return objects, volumes, medium


def spline_cameras(seed: int = SEED_BASE + 4, frames: int = 300, width: int = 1920, height: int = 1080,
                   fov: float = 60.0, control: int = 8):
    """Config 4's camera path: a closed Catmull-Rom spline through `control`
    seeded points on a ring around the config-2 scene (radius U(120, 180),
    height U(15, 60)), looking at seeded points near the centre; one camera
    per frame, uniform in the spline parameter."""
    rng = np.random.default_rng(seed)
    ang = np.sort(rng.uniform(0.0, 2.0 * np.pi, control))
    rad = rng.uniform(120.0, 180.0, control)
    pts = np.stack([rad * np.cos(ang), rng.uniform(15.0, 60.0, control), rad * np.sin(ang)], 1)
    tgt = rng.uniform(-30.0, 30.0, (control, 3)) * np.array([1.0, 0.3, 1.0])

    def cr(p, i, t):
        p0, p1, p2, p3 = (p[(i + k) % control] for k in (-1, 0, 1, 2))
        return 0.5 * ((2 * p1) + (-p0 + p2) * t + (2 * p0 - 5 * p1 + 4 * p2 - p3) * t * t
                      + (-p0 + 3 * p1 - 3 * p2 + p3) * t * t * t)

    cams = []
    for f in range(frames):
        u = f / frames * control
        i, t = int(u), u - int(u)
        pos, look = cr(pts, i, t), cr(tgt, i, t)
        d = look - pos
        cams.append(make_camera(pos, d / np.linalg.norm(d), fov, width, height))
    return cams
