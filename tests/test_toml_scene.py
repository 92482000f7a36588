"""The TOML scene front end (luminara_b200.toml_scene) against the reference's load_scene rules.

Scenes here are written for these tests in the reference's file format.  Loaded scenes are
compared with the same scene built by hand through the scene builder (identical keyed oracle
renders), and the loader's defaults, light harvesting, transform order, mesh files and
error reporting are checked.  When the reference source tree is present, every shipped
example scene must either load or fail with UnsupportedSceneError.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
from luminara_b200 import abi
from luminara_b200 import scene as S
from luminara_b200.toml_scene import UnsupportedSceneError, blackbody_to_rgb, load_scene, load_scene_file

BOX_ROOM = """
[render]
width = 24
height = 18
samples = 4
max_depth = 5
seed = 7
pixel_filter = "gaussian"
tone_map = "aces"
bloom = 0.2
background = { type = "black" }

[camera]
look_from = [278.0, 278.0, -800.0]
look_at = [278.0, 278.0, 0.0]
vfov = 40.0

[[rect_yz]]
y = [0.0, 555.0]
z = [0.0, 555.0]
k = 555.0
material = { type = "lambertian", color = [0.12, 0.45, 0.15] }

[[rect_yz]]
y = [0.0, 555.0]
z = [0.0, 555.0]
k = 0.0
material = { type = "lambertian", color = [0.65, 0.05, 0.05] }

[[rect_xz]]
x = [213.0, 343.0]
z = [227.0, 332.0]
k = 554.0
material = { type = "emissive", color = [1.0, 1.0, 1.0], intensity = 15.0 }

[[rect_xz]]
x = [0.0, 555.0]
z = [0.0, 555.0]
k = 0.0
material = { type = "matte", color = [0.73, 0.73, 0.73] }

[[rect_xy]]
x = [0.0, 555.0]
y = [0.0, 555.0]
k = 555.0
material = { type = "lambertian", color = [0.73, 0.73, 0.73] }

[[box]]
min = [0.0, 0.0, 0.0]
max = [165.0, 330.0, 165.0]
rotate_y = 15.0
translate = [265.0, 0.0, 295.0]
material = { type = "pbr", color = [0.8, 0.8, 0.8], roughness = 0.3 }

[[sphere]]
center = [190.0, 90.0, 190.0]
radius = 90.0
material = { type = "glass" }
"""


def hand_built_box_room():
    # the reference's object order: spheres, boxes, rect_xy, rect_xz, rect_yz
    w2 = S.World()
    w2.add(S.Sphere((190, 90, 190), 90, S.Dielectric(1.5)))
    box = S.make_box((0, 0, 0), (165, 330, 165), S.Microfacet((0.8, 0.8, 0.8), roughness=0.3))
    w2.add(S.Translate(S.RotateY(box, 15.0), (265, 0, 295)))
    w2.add(S.XyRect(0, 555, 0, 555, 555, S.Lambertian((0.73, 0.73, 0.73))))
    light = S.Emissive((1.0, 1.0, 1.0), 15.0)
    w2.add(S.XzRect(213, 343, 227, 332, 554, light))
    w2.add(S.XzRect(0, 555, 0, 555, 0, S.Lambertian((0.73, 0.73, 0.73))))
    w2.add(S.YzRect(0, 555, 0, 555, 555, S.Lambertian((0.12, 0.45, 0.15))))
    w2.add(S.YzRect(0, 555, 0, 555, 0, S.Lambertian((0.65, 0.05, 0.05))))
    w2.add_light(S.LightInfo.Rect((213, 554, 227), (130, 0, 0), (0, 0, 105), (0, -1, 0), (15.0, 15.0, 15.0)), light)
    w2.camera = S.CameraConfig(look_from=(278, 278, -800), look_at=(278, 278, 0), vfov_degrees=40.0,
                               aspect_ratio=24 / 18)
    cfg = S.RenderConfig(width=24, height=18, samples_per_pixel=4, max_depth=5, seed=7,
                         pixel_filter=abi.FILTER_GAUSSIAN, background=abi.BG_SOLID, bg_color=(0.0, 0.0, 0.0))
    return w2, cfg


def test_loaded_scene_renders_like_the_hand_built_scene():
    cfg, world, post = load_scene(BOX_ROOM)
    assert post == {"tone_map": "aces", "bloom": 0.2}
    assert (cfg.width, cfg.height, cfg.samples_per_pixel, cfg.max_depth, cfg.seed) == (24, 18, 4, 5, 7)
    assert cfg.pixel_filter == abi.FILTER_GAUSSIAN and cfg.background == abi.BG_SOLID
    assert world.camera.aspect_ratio == pytest.approx(24 / 18)
    assert len(world.lights) == 1 and world.lights[0].normal == (0.0, -1.0, 0.0)
    assert world.light_material_indices()[0] >= 0
    w2, cfg2 = hand_built_box_room()
    a, _ = O.OracleScene(world).render(cfg, mode=O.MODE_KEYED)
    b, _ = O.OracleScene(w2).render(cfg2, mode=O.MODE_KEYED)
    assert a.max() > 0
    np.testing.assert_array_equal(a, b)


def test_defaults_match_the_reference():
    cfg, world, post = load_scene("[[sphere]]\ncenter = [0, 0, -1]\nradius = 0.5\n"
                                  "material = { type = \"metal\", color = [0.8, 0.8, 0.8] }\n")
    assert (cfg.width, cfg.height, cfg.samples_per_pixel, cfg.max_depth, cfg.seed) == (800, 450, 100, 50, 31337)
    assert cfg.background == abi.BG_SKY and cfg.exposure == 1.0 and cfg.pixel_filter == abi.FILTER_BOX
    cam = world.camera
    assert (cam.look_from, cam.look_at, cam.vup, cam.vfov_degrees, cam.aperture, cam.focus_dist) == \
        ((0.0, 1.0, 3.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 40.0, 0.0, 1.0)
    assert cam.aspect_ratio == pytest.approx(800 / 450)
    m = world.materials[0]
    assert m.kind == abi.MAT_METAL and m.fuzz == 0.0
    assert post == {} and world.lights == []


def test_light_harvesting_follows_the_reference():
    text = """
[[sphere]]
center = [0.0, 5.0, 0.0]
radius = 1.0
translate = [10.0, 0.0, 0.0]
material = { type = "emissive", color = [1.0, 0.5, 0.25], intensity = 4.0 }

[[light]]
position = [1.0, 2.0, 3.0]

[[disk]]
center = [0.0, 3.0, 0.0]
normal = [0.0, -2.0, 0.0]
radius = 0.5
material = { type = "blackbody", temperature = 3000.0, intensity = 2.0 }

[[quad]]
q = [0.0, 4.0, 0.0]
u = [2.0, 0.0, 0.0]
v = [0.0, 0.0, 1.0]
material = { type = "emissive", color = [2.0, 2.0, 2.0] }

[[rect_xy]]
x = [0.0, 1.0]
y = [0.0, 1.0]
k = 0.0
material = { type = "emissive", color = [1.0, 1.0, 1.0] }

[[rect_xz]]
x = [0.0, 1.0]
z = [0.0, 1.0]
k = 9.0
material = { type = "blackbody", temperature = 5000.0 }
"""
    cfg, world, _ = load_scene(text)
    L = world.lights
    assert [l.kind for l in L] == [abi.LIGHT_SPHERE, abi.LIGHT_SPHERE, abi.LIGHT_DISK, abi.LIGHT_RECT]
    assert L[0].p0 == (0.0, 5.0, 0.0) and L[0].emission == (4.0, 2.0, 1.0)      # untransformed centre
    assert L[1].radius == 0.1 and L[1].emission == (10.0, 10.0, 10.0)           # [[light]] defaults
    assert L[2].normal == (0.0, -1.0, 0.0)
    np.testing.assert_allclose(L[2].emission, np.array(blackbody_to_rgb(3000.0)) * 2.0)
    assert L[3].normal == (0.0, 1.0, 0.0) or L[3].normal == (0.0, -1.0, 0.0)
    np.testing.assert_allclose(np.cross((2, 0, 0), (0, 0, 1)) / 2.0, L[3].normal)
    # emissive rect_xy and blackbody rect_xz are not harvested; the [[light]] sphere is an object
    assert world.n_prims() == 6
    idx = world.light_material_indices()
    assert all(i >= 0 for i in idx) and world.materials[idx[1]].intensity == 10.0


def test_blackbody_colour():
    r, g, b = blackbody_to_rgb(1000.0)
    assert r == 1.0 and b == 0.0 and 0.0 < g < 0.5
    r, g, b = blackbody_to_rgb(40000.0)
    assert b == 1.0 and r < g < 1.0
    r, g, b = blackbody_to_rgb(6600.0)
    assert r == 1.0 and b == 1.0 and g > 0.95
    assert blackbody_to_rgb(100.0) == blackbody_to_rgb(1000.0)          # clamped range
    for t in np.linspace(1000, 40000, 97):
        assert all(0.0 <= c <= 1.0 for c in blackbody_to_rgb(t))


def test_transforms_keep_the_reference_order():
    text = """
[[sphere]]
center = [1.0, 0.0, 0.0]
radius = 0.5
rotate_z = 90.0
translate = [0.0, 2.0, 0.0]
scale = 2.0
material = { type = "lambertian", color = [0.5, 0.5, 0.5] }

[[box]]
min = [0.0, 0.0, 0.0]
max = [1.0, 2.0, 3.0]
scale = 2.0
rotate_x = 10.0
rotate_y = 20.0
translate = [1.0, 1.0, 1.0]
material = { type = "lambertian", color = [0.5, 0.5, 0.5] }
"""
    _, world, _ = load_scene(text)
    sph, box = world.objects
    assert [op for op, _ in sph.xforms] == [abi.XF_ROTATE_Z, abi.XF_TRANSLATE, abi.XF_SCALE]
    assert [op for op, _ in box.xforms] == [abi.XF_SCALE, abi.XF_ROTATE_X, abi.XF_ROTATE_Y, abi.XF_TRANSLATE]


def test_meshes_from_obj_and_ply(tmp_path):
    (tmp_path / "quad.obj").write_text(
        "# two triangles, one fan quad with normals\n"
        "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvn 0 0 2\n"
        "f 1//1 2//1 3//1 4//1\nf 1 2 3\n")
    (tmp_path / "tri.ply").write_text(
        "ply\nformat ascii 1.0\nelement vertex 4\nproperty float x\nproperty float y\nproperty float z\n"
        "element face 1\nproperty list uchar int vertex_indices\nend_header\n"
        "0 0 0\n1 0 0\n1 1 0\n0 1 0\n4 0 1 2 3\n")
    (tmp_path / "scene.toml").write_text(
        '[[mesh]]\nfile = "quad.obj"\nscale = 2.0\noffset = [0.0, 0.0, 1.0]\n'
        'material = { type = "lambertian", color = [0.5, 0.5, 0.5] }\n'
        '[[mesh]]\nfile = "tri.ply"\nmaterial = { type = "metal", color = [0.9, 0.9, 0.9], fuzz = 0.1 }\n')
    cfg, world, _ = load_scene_file(str(tmp_path / "scene.toml"))
    assert [len(m.indices) for m in world.meshes] == [2, 1, 2]      # smooth run, flat run, ply
    smooth, flat, ply = world.meshes
    np.testing.assert_allclose(smooth.positions[:3], [[0, 0, 1], [2, 0, 1], [2, 2, 1]])
    np.testing.assert_allclose(smooth.normals, np.tile([0, 0, 1.0], (6, 1)))
    assert flat.normals is None and ply.normals is None
    np.testing.assert_allclose(ply.positions[3:], [[0, 0, 0], [1, 1, 0], [0, 1, 0]])
    img, _ = O.OracleScene(world).render(S.RenderConfig(width=8, height=6, samples_per_pixel=1, max_depth=2),
                                         mode=O.MODE_KEYED)
    assert np.isfinite(img).all()


def test_adaptive_keys_reach_the_render_config():
    cfg, _, _ = load_scene("[render]\nadaptive = true\nadaptive_threshold = 0.05\nsamples = 64\n")
    assert cfg.adaptive and cfg.adaptive_threshold == 0.05
    cfg, _, _ = load_scene("[render]\nsamples = 64\n")
    assert not cfg.adaptive and cfg.adaptive_threshold == 0.03          # render.rs:455-456


OTHER_MATERIALS = """
[render]
width = 32
height = 24
samples = 4
background = { type = "starfield", star_density = 0.5 }

[[sphere]]
center = [0.0, 0.0, 0.0]
radius = 1.0
material = { type = "toon", color = [0.2, 0.5, 0.9] }

[[sphere]]
center = [2.0, 0.0, 0.0]
radius = 1.0
material = { type = "brushed", color = [0.8, 0.8, 0.85], roughness_u = 0.05 }

[[sphere]]
center = [4.0, 0.0, 0.0]
radius = 1.0
material = { type = "blend", ratio = 0.25, material_a = { type = "velvet", color = [0.5, 0.1, 0.1] }, material_b = { type = "sss", color = [0.9, 0.7, 0.6] } }

[[sphere]]
center = [6.0, 0.0, 0.0]
radius = 1.0
material = { type = "opacity", opacity = 1.5, material = { type = "clearcoat", color = [0.8, 0.1, 0.05] } }

[[sphere]]
center = [8.0, 0.0, 0.0]
radius = 1.0
material = { type = "iridescent", thickness = 500 }

[[sphere]]
center = [10.0, 0.0, 0.0]
radius = 1.0
material = { type = "translucent", color = [0.7, 0.9, 0.7] }
"""


def test_other_materials_and_starfield():
    cfg, world, _ = load_scene(OTHER_MATERIALS)
    assert cfg.background == abi.BG_STARFIELD and cfg.bg_star_density == 0.5 and cfg.bg_star_brightness == 5.0
    kinds = [o.material.kind for o in world.objects]
    assert kinds == [abi.MAT_TOON, abi.MAT_ANISOTROPIC, abi.MAT_BLEND, abi.MAT_BLEND, abi.MAT_IRIDESCENT,
                     abi.MAT_TRANSLUCENT]
    toon, aniso, blend, opac, irid, transl = [o.material for o in world.objects]
    assert tuple(toon.extra) == (3, 0.5)                                     # scene.rs:1991-1996 defaults
    assert tuple(aniso.extra) == (0.05, 0.5, 1)
    assert blend.extra[0] == 0.25 and [c.kind for c in blend.children] == [abi.MAT_VELVET, abi.MAT_SUBSURFACE]
    assert tuple(blend.children[1].color2) == (0.8, 0.5, 0.5) and blend.children[1].extra[0] == 0.5
    assert opac.extra[0] == 1.0 and [c.kind for c in opac.children] == [abi.MAT_CLEARCOAT, abi.MAT_TRANSPARENT]
    assert tuple(irid.color) == (0.9, 0.9, 0.9) and irid.extra[0] == 500 and irid.ior == 1.4
    assert tuple(transl.extra) == (0.5, 0.8)
    img, st = O.OracleScene(world).render(cfg, mode=O.MODE_KEYED)
    assert np.isfinite(img).all() and st.paths == 32 * 24 * 4


def _write_hdr(path, img, rle):
    """Radiance RGBE writer (test fixture): flat or new-style RLE scanlines (literal runs)."""
    h, w, _ = img.shape
    m = img.max(axis=2)
    e = np.where(m > 1e-32, np.floor(np.log2(np.maximum(m, 1e-32))) + 1, 0).astype(np.int32)
    mant = np.where(m[..., None] > 1e-32, img / np.ldexp(1.0, e - 8)[..., None], 0)
    rgbe = np.concatenate([np.clip(mant, 0, 255).astype(np.uint8), np.where(m > 1e-32, e + 128, 0)[..., None]
                           .astype(np.uint8)], axis=2)
    with open(path, "wb") as f:
        f.write(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {h} +X {w}\n".encode())
        for y in range(h):
            if not rle:
                f.write(rgbe[y].tobytes())
                continue
            f.write(bytes([2, 2, w >> 8, w & 255]))
            for c in range(4):
                row = rgbe[y, :, c]
                for x0 in range(0, w, 128):
                    chunk = row[x0:x0 + 128]
                    f.write(bytes([len(chunk)]) + chunk.tobytes())
    return rgbe


@pytest.mark.parametrize("rle", [False, True])
def test_env_map_hdr_and_png(tmp_path, rle):
    from luminara_b200.toml_scene import load_env_map
    rng = np.random.default_rng(1)
    img = (rng.random((6, 16, 3)) * 4.0).astype(np.float32)
    rgbe = _write_hdr(str(tmp_path / "sky.hdr"), img, rle)
    got = load_env_map(str(tmp_path / "sky.hdr"))
    want = rgbe[..., :3] * np.ldexp(1.0, rgbe[..., 3].astype(int) - 136)[..., None]
    np.testing.assert_allclose(got, want, rtol=1e-6)
    assert (np.abs(got - img) <= img.max(axis=2, keepdims=True) / 64).all()  # 8-bit shared-exponent mantissas
    from PIL import Image
    px = (rng.random((5, 9, 3)) * 255).astype(np.uint8)
    Image.fromarray(px).save(str(tmp_path / "sky.png"))
    np.testing.assert_allclose(load_env_map(str(tmp_path / "sky.png")), px / 255.0, rtol=1e-6)
    cfg, world, _ = load_scene('[render]\nbackground = { type = "env_map", file = "sky.png", intensity = 2.0 }\n',
                               base_dir=str(tmp_path))
    assert cfg.background == abi.BG_ENVMAP and cfg.bg_intensity == 2.0 and world.env_map.shape == (5, 9, 3)


def test_unsupported_features_are_named():
    text = """
[render]
firefly_filter = 4.0

[[torus]]
center = [0.0, 0.0, 0.0]
major_radius = 1.0
minor_radius = 0.2
material = { type = "lambertian", color = [0.5, 0.5, 0.5] }

[[sphere]]
center = [0.0, 0.0, 0.0]
radius = 1.0
bump_strength = 0.5
material = { type = "marble", color = [0.5, 0.5, 0.5] }
"""
    with pytest.raises(UnsupportedSceneError) as e:
        load_scene(text)
    items = e.value.items
    for want in ("[torus]", "render.firefly_filter", "bump_strength", "'marble'"):
        assert any(want in it for it in items), (want, items)


def test_panorama_camera_is_read():
    cfg, world, _ = load_scene('[camera]\nlook_from = [0.0, 1.0, 0.0]\npanorama = true\n')
    assert world.camera.panorama is True
    cfg, world, _ = load_scene('[camera]\nlook_from = [0.0, 1.0, 0.0]\n')
    assert world.camera.panorama is False


# The reference project's example scene directory (examples/scenes of a Luminara checkout),
# named by LUM_REFERENCE_SCENES; the test is skipped when it is unset.
REF_SCENES = os.environ.get("LUM_REFERENCE_SCENES", "")


@pytest.mark.skipif(not REF_SCENES or not os.path.isdir(REF_SCENES),
                    reason="LUM_REFERENCE_SCENES (the reference's examples/scenes) not set")
def test_reference_example_scenes_load_or_are_rejected_by_name():
    loaded = []
    for f in sorted(glob.glob(os.path.join(REF_SCENES, "*.toml"))):
        try:
            cfg, world, post = load_scene_file(f)
        except UnsupportedSceneError as e:
            assert e.items
            continue
        loaded.append(os.path.basename(f))
        assert world.n_prims() > 0 and cfg.width > 0
        img, _ = O.OracleScene(world).render(
            S.RenderConfig(width=8, height=6, samples_per_pixel=1, max_depth=3, background=cfg.background,
                           bg_color=cfg.bg_color, bg_color2=cfg.bg_color2, bg_dir=cfg.bg_dir,
                           bg_intensity=cfg.bg_intensity), mode=O.MODE_KEYED)
        assert np.isfinite(img).all()
    print("loaded:", loaded)
    assert {"cornell.toml", "distortion.toml", "pbr_showcase.toml", "prism.toml", "retro.toml",
            "toon.toml"} <= set(loaded), loaded
