"""Seeded synthetic workloads with the shapes of the benchmark configurations.

Each builder returns ``(world, render_config)``.  Scenes are generated with numpy's
seeded generator; object order follows the reference's loaders (it fixes primitive ids).

  box_room        256x256, 64 spp, depth 8, NEE: the examples/scenes/cornell.toml geometry with
                  a white x15 ceiling light (scene.rs loader order: boxes, rect_xy, rect_xz, rect_yz)
  random_spheres  1920x1080, 256 spp, depth 16: 22x22 jittered grid of r=0.2 spheres plus ground
                  and three hero spheres (the pattern of scene.rs:2051-2216, seeded, 484 small spheres)
  dense_mesh      1920x1080, 128 spp (144 strata), depth 8, NEE: displaced icosphere of 20*4^L
                  triangles (L=8: 1,310,720), GGX per 1024-triangle patch, plane ground, three disk
                  lights, a fog box
  diff_quads      512x512, 64 spp, depth 6: 1000 GGX quads + 4 emissive quads (the differentiable
                  rendering scene)
"""
from __future__ import annotations

import numpy as np

from . import abi
from . import scene as S


def box_room(width=256, height=256, spp=64, max_depth=8, seed=31337):
    w = S.World()
    white = S.Lambertian((0.73, 0.73, 0.73))
    red = S.Lambertian((0.65, 0.05, 0.05))
    green = S.Lambertian((0.12, 0.45, 0.15))
    light = S.Emissive((1.0, 1.0, 1.0), 15.0)
    # [[box]] entries (tall box first, as in the TOML file)
    w.add(S.Translate(S.RotateY(S.make_box((0, 0, 0), (165, 330, 165), white), 15.0), (265, 0, 295)))
    w.add(S.Translate(S.RotateY(S.make_box((0, 0, 0), (165, 165, 165), white), -18.0), (130, 0, 65)))
    w.add(S.XyRect(0, 555, 0, 555, 555, white))           # back wall
    w.add(S.XzRect(213, 343, 227, 332, 554, light))       # ceiling light
    w.add(S.XzRect(0, 555, 0, 555, 0, white))             # floor
    w.add(S.XzRect(0, 555, 0, 555, 555, white))           # ceiling
    w.add(S.YzRect(0, 555, 0, 555, 0, red))               # x = 0, red
    w.add(S.YzRect(0, 555, 0, 555, 555, green))           # x = 555, green
    # emissive rect_xz -> LightInfo::Rect (scene.rs:1607-1619)
    w.add_light(S.LightInfo.Rect((213, 554, 227), (130, 0, 0), (0, 0, 105), (0, -1, 0), (15.0, 15.0, 15.0)))
    w.camera = S.CameraConfig(look_from=(278, 278, -800), look_at=(278, 278, 0), vfov_degrees=40.0,
                              aspect_ratio=width / height, aperture=0.0, focus_dist=1.0)
    cfg = S.RenderConfig(width=width, height=height, samples_per_pixel=spp, max_depth=max_depth, seed=seed,
                         background=abi.BG_SOLID, bg_color=(0, 0, 0))
    return w, cfg


def random_spheres(width=1920, height=1080, spp=256, max_depth=16, seed=31337, scene_seed=7, grid=11):
    rng = np.random.default_rng(scene_seed)
    w = S.World()
    w.add(S.Sphere((0, -1000, 0), 1000.0, S.Lambertian((0.5, 0.5, 0.5))))
    w.add(S.Sphere((0, 1, 0), 1.0, S.Dielectric(1.5)))
    w.add(S.Sphere((-4, 1, 0), 1.0, S.Lambertian((0.4, 0.2, 0.1))))
    w.add(S.Sphere((4, 1, 0), 1.0, S.Metal((0.7, 0.6, 0.5), 0.0)))
    glass = S.Dielectric(1.5)
    for a in range(-grid, grid):
        for b in range(-grid, grid):
            choose = rng.random()
            cx, cz = a + 0.9 * rng.random(), b + 0.9 * rng.random()
            if choose < 0.8:
                alb = rng.random(3) * rng.random(3)
                m = S.Lambertian(tuple(alb))
            elif choose < 0.95:
                alb = 0.5 + 0.5 * rng.random(3)
                m = S.Metal(tuple(alb), 0.5 * rng.random())
            else:
                m = glass
            w.add(S.Sphere((cx, 0.2, cz), 0.2, m))
    w.camera = S.CameraConfig(look_from=(13, 2, 3), look_at=(0, 0, 0), vfov_degrees=20.0,
                              aspect_ratio=width / height, aperture=0.1, focus_dist=10.0)
    cfg = S.RenderConfig(width=width, height=height, samples_per_pixel=spp, max_depth=max_depth, seed=seed,
                         background=abi.BG_SKY)
    return w, cfg


# ----------------------------------------------------------------------------- Perlin noise
def _perlin_tables(seed):
    rng = np.random.default_rng(seed)
    p = rng.permutation(256)
    return np.concatenate([p, p]).astype(np.int64)


def _fade(t):
    return t * t * t * (t * (t * 6 - 15) + 10)


def _grad(h, x, y, z):
    # Improved-noise gradient selection (Perlin 2002)
    h = h & 15
    u = np.where(h < 8, x, y)
    v = np.where(h < 4, y, np.where((h == 12) | (h == 14), x, z))
    return np.where(h & 1, -u, u) + np.where(h & 2, -v, v)


def perlin3(p, perm):
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    X, Y, Z = (np.floor(x).astype(np.int64) & 255, np.floor(y).astype(np.int64) & 255,
               np.floor(z).astype(np.int64) & 255)
    x, y, z = x - np.floor(x), y - np.floor(y), z - np.floor(z)
    u, v, w = _fade(x), _fade(y), _fade(z)
    A = perm[X] + Y
    AA, AB = perm[A] + Z, perm[A + 1] + Z
    B = perm[X + 1] + Y
    BA, BB = perm[B] + Z, perm[B + 1] + Z
    lerp = lambda t, a, b: a + t * (b - a)
    return lerp(w,
                lerp(v, lerp(u, _grad(perm[AA], x, y, z), _grad(perm[BA], x - 1, y, z)),
                     lerp(u, _grad(perm[AB], x, y - 1, z), _grad(perm[BB], x - 1, y - 1, z))),
                lerp(v, lerp(u, _grad(perm[AA + 1], x, y, z - 1), _grad(perm[BA + 1], x - 1, y, z - 1)),
                     lerp(u, _grad(perm[AB + 1], x, y - 1, z - 1), _grad(perm[BB + 1], x - 1, y - 1, z - 1))))


def icosphere_soup(level: int) -> np.ndarray:
    """Triangle soup (T, 3, 3) of a unit icosphere with 20*4^level faces, in recursive order
    (each run of 4^k consecutive triangles is one patch of a level-k subdivision)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]])
    tri = v[f]
    norm = lambda x: x / np.linalg.norm(x, axis=-1, keepdims=True)
    for _ in range(level):
        a, b, c = tri[:, 0], tri[:, 1], tri[:, 2]
        ab, bc, ca = norm(a + b), norm(b + c), norm(c + a)
        tri = np.stack([np.stack([a, ab, ca], 1), np.stack([ab, b, bc], 1), np.stack([ca, bc, c], 1),
                        np.stack([ab, bc, ca], 1)], axis=1).reshape(-1, 3, 3)
    return tri


def dense_mesh(width=1920, height=1080, spp=128, max_depth=8, seed=31337, scene_seed=11, level=8,
               amplitude=0.05, patch=1024, fog=True):
    rng = np.random.default_rng(scene_seed)
    tri = icosphere_soup(level)
    pts = tri.reshape(-1, 3)
    perm = _perlin_tables(scene_seed)
    n = np.zeros(pts.shape[0])
    for o in range(3):                                   # 3 octaves
        n += perlin3(pts * (2.0 * 2 ** o) + 0.5, perm) / (2 ** o)
    pts = pts * (1.0 + amplitude * n)[:, None]
    T = tri.shape[0]
    n_patch = (T + patch - 1) // patch
    w = S.World()
    mats = []
    for k in range(n_patch):
        m = S.Microfacet((0.8, 0.75, 0.7), roughness=float(rng.uniform(0.05, 0.6)), metallic=0.5)
        mats.append(m)
        w.material_index(m)
    w.add(S.Plane((0, -1.1, 0), (0, 1, 0), S.Lambertian((0.5, 0.5, 0.5))))
    disk_pos = [(-2.5, 3.0, 1.5), (2.5, 3.5, 1.0), (0.0, 3.0, -2.5)]
    for k, c in enumerate(disk_pos):
        e = float(rng.uniform(5.0, 20.0))
        nrm = -np.asarray(c) / np.linalg.norm(c)
        w.add(S.Disk(c, tuple(nrm), 0.6, S.Emissive((1.0, 1.0, 1.0), e)))
        w.add_light(S.LightInfo.Disk(c, tuple(nrm), 0.6, (e, e, e)))
    if fog:
        w.add(S.ConstantMedium(S.make_box((-4, -1.1, -4), (4, 4, 4), None), 0.01, (1.0, 1.0, 1.0)))
    mesh_mat = np.repeat(np.arange(n_patch, dtype=np.int32), patch)[:T]
    mat_idx = np.array([w.material_index(m) for m in mats], dtype=np.int32)
    w.add_mesh(S.Mesh(positions=pts, indices=np.arange(3 * T, dtype=np.uint32).reshape(T, 3),
                      tri_material=mat_idx[mesh_mat]))
    w.camera = S.CameraConfig(look_from=(0.0, 0.6, 4.2), look_at=(0, 0, 0), vfov_degrees=40.0,
                              aspect_ratio=width / height)
    cfg = S.RenderConfig(width=width, height=height, samples_per_pixel=spp, max_depth=max_depth, seed=seed,
                         background=abi.BG_SOLID, bg_color=(0.05, 0.05, 0.08))
    return w, cfg


def diff_quads(width=512, height=512, spp=64, max_depth=6, seed=31337, scene_seed=5, n_quads=1000):
    rng = np.random.default_rng(scene_seed)
    w = S.World()
    for _ in range(n_quads):
        c = rng.uniform(-4, 4, 3)
        a = rng.normal(size=3)
        a /= np.linalg.norm(a)
        b = rng.normal(size=3)
        b -= a * (a @ b)
        b /= np.linalg.norm(b)
        su, sv = rng.uniform(0.4, 1.2, 2)
        q = c - 0.5 * su * a - 0.5 * sv * b
        m = S.Microfacet(tuple(rng.uniform(0.1, 0.9, 3)), roughness=float(rng.uniform(0.1, 0.8)), metallic=0.3)
        w.add(S.Quad(tuple(q), tuple(su * a), tuple(sv * b), m))
    for k in range(4):
        x, z = (-3 + 6 * (k % 2)), (-3 + 6 * (k // 2))
        e = float(rng.uniform(15.0, 30.0))
        q, u, v = (x - 1.5, 6.0, z - 1.5), (3.0, 0, 0), (0, 0, 3.0)
        em = S.Emissive((1.0, 1.0, 1.0), e)
        w.add(S.Quad(q, u, v, em))
        nrm = np.cross(u, v)
        nrm = nrm / np.linalg.norm(nrm)
        w.add_light(S.LightInfo.Rect(q, u, v, tuple(nrm), (e, e, e)), material=em)
    w.camera = S.CameraConfig(look_from=(0, 2, 14), look_at=(0, 0, 0), vfov_degrees=40.0,
                              aspect_ratio=width / height)
    cfg = S.RenderConfig(width=width, height=height, samples_per_pixel=spp, max_depth=max_depth, seed=seed,
                         background=abi.BG_SOLID, bg_color=(0.0, 0.0, 0.0))
    return w, cfg


def uneven_scene(rng, n_prims, width, height, spp, max_depth=8, seed=31337):
    """One scene of the batched workload: n_prims random spheres, quads and triangles with
    mixed Lambertian / Metal / Dielectric / GGX materials over a ground quad, lit by a sky and
    one or two NEE lights (built with vectorized bulk arrays)."""
    w = S.World()
    w.add(S.Quad((-20, 0, -20), (40, 0, 0), (0, 0, 40), S.Lambertian((0.5, 0.5, 0.5))))
    extent = max(1.5, 0.25 * n_prims ** (1 / 3))
    size = 0.6 * extent / max(1.0, n_prims ** (1 / 3))
    kinds = rng.integers(0, 3, n_prims)
    r = rng.random(n_prims)
    centers = rng.uniform(-extent, extent, (n_prims, 3))
    centers[:, 1] = rng.uniform(0.1, 2 * extent, n_prims)
    mats = S.material_array(n_prims)
    lam, met, die = r < 0.5, (r >= 0.5) & (r < 0.7), (r >= 0.7) & (r < 0.8)
    ggx = r >= 0.8
    mats["kind"] = np.select([lam, met, die, ggx], [abi.MAT_LAMBERTIAN, abi.MAT_METAL, abi.MAT_DIELECTRIC,
                                                    abi.MAT_MICROFACET])
    mats["color"] = rng.random((n_prims, 3)) * 0.8 + 0.1
    mats["color"][met] = 0.5 + 0.5 * rng.random((int(met.sum()), 3))
    mats["fuzz"] = np.where(met, 0.3 * rng.random(n_prims), 0.0)
    mats["ior"] = 1.5
    mats["roughness"] = np.where(ggx, rng.uniform(0.05, 0.7, n_prims), 0.0)
    mats["metallic"] = np.where(ggx, rng.random(n_prims), 0.0)
    sz = size * rng.uniform(0.5, 1.5, n_prims)
    a = rng.normal(size=(n_prims, 3))
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    b = rng.normal(size=(n_prims, 3))
    b -= a * (a * b).sum(1, keepdims=True)
    b /= np.linalg.norm(b, axis=1, keepdims=True)
    objs = np.zeros(n_prims, dtype=S.OBJECT_DTYPE)
    objs["material"] = np.arange(n_prims)
    objs["transform"] = -1
    sph, quad, tri = kinds == 0, kinds == 1, kinds == 2
    objs["kind"] = np.select([sph, quad, tri], [abi.OBJ_SPHERE, abi.OBJ_QUAD, abi.OBJ_TRIANGLE])
    p = objs["p"]
    p[sph, 0:3] = centers[sph]
    p[sph, 3] = sz[sph]
    s2 = (2 * sz)[:, None]
    q = centers - sz[:, None] * (a + b)
    p[quad, 0:3] = q[quad]
    p[quad, 3:6] = (s2 * a)[quad]
    p[quad, 6:9] = (s2 * b)[quad]
    p[tri, 0:3] = centers[tri]
    p[tri, 3:6] = (centers + s2 * a)[tri]
    p[tri, 6:9] = (centers + s2 * b)[tri]
    w.add_bulk(objs, mats)
    for k in range(int(rng.integers(1, 3))):
        e = float(rng.uniform(5, 20))
        if rng.random() < 0.5:
            c = (float(rng.uniform(-extent, extent)), 3.0 * extent, float(rng.uniform(-extent, extent)))
            rad = 0.3 * extent
            w.add(S.Sphere(c, rad, S.Emissive((1, 1, 1), e)))
            w.add_light(S.LightInfo.Sphere(c, rad, (e, e, e)))
        else:
            qq, u, v = (-0.5 * extent, 3.0 * extent, -0.5 * extent), (extent, 0, 0), (0, 0, extent)
            w.add(S.Quad(qq, u, v, S.Emissive((1, 1, 1), e)))
            w.add_light(S.LightInfo.Rect(qq, u, v, (0, -1, 0), (e, e, e)))
    w.camera = S.CameraConfig(look_from=(0.0, 1.5 * extent, 3.5 * extent), look_at=(0, 0.5 * extent, 0),
                              vfov_degrees=45.0, aspect_ratio=width / height)
    cfg = S.RenderConfig(width=width, height=height, samples_per_pixel=spp, max_depth=max_depth, seed=seed,
                         background=abi.BG_SKY)
    return w, cfg


def batched(n_scenes=64, seed=3, res_choices=(128, 256, 512, 1024), spp_choices=(16, 64, 256), min_prims=10,
            max_prims=50000, max_depth=8):
    """The batched uneven workload: n_scenes seeded scenes with primitive counts log-uniform in
    [min_prims, max_prims], square resolutions and spp drawn from the given sets."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_scenes):
        n = int(round(np.exp(rng.uniform(np.log(min_prims), np.log(max_prims)))))
        r = int(rng.choice(res_choices))
        spp = int(rng.choice(spp_choices))
        out.append(uneven_scene(rng, n, r, r, spp, max_depth=max_depth, seed=31337 + i))
    return out


def material_zoo(width=160, height=120, spp=16, max_depth=8, seed=31337, background=abi.BG_SOLID):
    """A lit room with one sphere per remaining material (material.rs:396-865), Blends included
    (one with an emissive leaf, one nested two deep)."""
    w = S.World()
    white = S.Lambertian((0.73, 0.73, 0.73))
    red = S.Lambertian((0.65, 0.05, 0.05))
    light = S.Emissive((1.0, 1.0, 1.0), 12.0)
    w.add(S.XzRect(-6, 6, -6, 6, 0, white))                      # floor
    w.add(S.XyRect(-6, 6, 0, 8, -4, S.Lambertian((0.4, 0.5, 0.7))))   # back wall
    w.add(S.YzRect(0, 8, -6, 6, -6, red))
    w.add(S.XzRect(-1.5, 1.5, -1.5, 1.5, 7.9, light))
    w.add_light(S.LightInfo.Rect((-1.5, 7.9, -1.5), (3, 0, 0), (0, 0, 3), (0, -1, 0), (12.0, 12.0, 12.0)))
    glow = S.Emissive((1.0, 0.6, 0.2), 4.0)
    mats = [
        S.Blend(red, S.Metal((0.8, 0.8, 0.9), 0.1), 0.4),
        S.Blend(glow, S.Lambertian((0.2, 0.6, 0.3)), 0.3),
        S.Blend(S.Blend(S.Velvet((0.5, 0.1, 0.4), 1.0), S.Toon((0.9, 0.7, 0.1), 4, 0.5), 0.5), white, 0.7),
        S.Transparent(),
        S.Iridescent((0.9, 0.9, 0.9), 380.0, 1.33, 0.0),
        S.Iridescent((0.8, 0.9, 1.0), 520.0, 1.5, 0.2),
        S.Toon((0.2, 0.5, 0.9), 3, 0.0),
        S.Anisotropic((0.9, 0.8, 0.6), 0.4, 0.05, 0),
        S.Clearcoat((0.7, 0.1, 0.1), 0.8, 1.5),
        S.Velvet((0.3, 0.1, 0.5), 1.2),
        S.Translucent((0.3, 0.8, 0.3), 0.6, 0.5),
        S.Subsurface((0.9, 0.7, 0.6), 0.3, (0.9, 0.3, 0.3)),
    ]
    for k, m in enumerate(mats):
        x = -4.5 + 3.0 * (k % 4)
        z = -2.0 + 2.2 * (k // 4)
        w.add(S.Sphere((x, 0.9, z), 0.9, m))
    w.camera = S.CameraConfig(look_from=(0, 4.5, 9.5), look_at=(0, 1.2, 0), vfov_degrees=50.0,
                              aspect_ratio=width / height, aperture=0.0, focus_dist=1.0)
    cfg = S.RenderConfig(width=width, height=height, samples_per_pixel=spp, max_depth=max_depth, seed=seed,
                         background=background, bg_color=(0.05, 0.05, 0.08))
    return w, cfg


CONFIGS = {
    "box_room": box_room,
    "random_spheres": random_spheres,
    "dense_mesh": dense_mesh,
    "diff_quads": diff_quads,
    "material_zoo": material_zoo,
}
