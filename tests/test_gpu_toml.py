"""GPU renders of scenes loaded from TOML text match the keyed oracle (same tolerance as the
other keyed parity tests: >= 97% of pixels within 2e-3 * (1 + |ref|), means within 0.5%).

The checker plane sits half a checker cell below y = 0: the reference's 3D checker
(src/texture.rs:38-50) takes floor(p.y / scale), so on a plane at a multiple of the scale the
cell parity follows the sign of each hit point's rounding error, which f32 and f64 vertices
do not share."""
import pytest

import luminara_b200 as L
from tests.test_gpu_render import keyed_compare
from tests.test_toml_scene import BOX_ROOM

pytestmark = pytest.mark.gpu

LIGHTS_AND_SPHERES = """
[render]
width = 48
height = 32
samples = 16
max_depth = 8
background = { type = "gradient", bottom = [0.05, 0.05, 0.1], top = [0.2, 0.3, 0.5] }

[camera]
look_from = [0.0, 2.0, 8.0]
look_at = [0.0, 0.5, 0.0]
vfov = 35.0
aperture = 0.05
focus_dist = 8.0

[[plane]]
point = [0.0, -0.35, 0.0]
normal = [0.0, 1.0, 0.0]
material = { type = "checker", color1 = [0.9, 0.9, 0.9], color2 = [0.2, 0.2, 0.2], scale = 0.7 }

[[sphere]]
center = [-1.5, 0.8, 0.0]
radius = 0.8
material = { type = "pbr", color = [0.9, 0.6, 0.3], roughness = 0.35, metallic = 0.8 }

[[sphere]]
center = [0.0, 0.8, 0.5]
radius = 0.8
material = { type = "dielectric", refraction_index = 1.5, tint = [0.9, 1.0, 0.95], roughness = 0.05 }

[[sphere]]
center = [1.6, 0.6, 0.0]
radius = 0.6
material = { type = "mirror" }

[[light]]
position = [0.0, 4.0, 2.0]
radius = 0.3
intensity = 20.0

[[disk]]
center = [2.5, 3.0, -1.0]
normal = [0.0, -1.0, 0.2]
radius = 0.7
material = { type = "blackbody", temperature = 3500.0, intensity = 6.0 }

[[quad]]
q = [-3.0, 3.5, -2.0]
u = [1.5, 0.0, 0.0]
v = [0.0, 0.0, 1.5]
material = { type = "emissive", color = [0.8, 0.9, 1.0], intensity = 5.0 }
"""


def test_box_room_toml_matches_keyed_oracle():
    cfg, world, _ = L.load_scene(BOX_ROOM)
    cfg.width, cfg.height, cfg.samples_per_pixel = 64, 48, 16
    world.camera.aspect_ratio = 64 / 48
    keyed_compare(world, cfg)


def test_lights_and_spheres_toml_matches_keyed_oracle():
    cfg, world, _ = L.load_scene(LIGHTS_AND_SPHERES)
    assert len(world.lights) == 3
    keyed_compare(world, cfg)
