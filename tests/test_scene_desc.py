"""The Python front end's scene description (World.desc): the object and material records it
hands to lum_scene_create are built column by column as numpy records; they must be, byte for
byte, the records the field-by-field ctypes construction gives (Material.to_c, one LumObject
per object), for every workload and for every material and texture feature.  CPU only."""
import ctypes as C

import numpy as np
import pytest

from luminara_b200 import abi
from luminara_b200 import scene as S
from luminara_b200 import workloads as W


def _reference_records(world):
    """Objects and materials as one ctypes record per object / material, field by field."""
    for o in world.objects:
        world.material_index(o.material)
    objs, n_xf = [], 0
    for o in world.objects:
        lo = abi.LumObject()
        lo.kind = o.kind
        lo.material = world.material_index(o.material)
        lo.transform = -1
        p = list(map(float, o.params)) + [0.0] * (12 - len(o.params))
        lo.p[:] = p[:12]
        if o.xforms:
            lo.transform = n_xf
            n_xf += 1
        objs.append(lo)
    mats = [m.to_c(world.material_index) for m in world.materials]
    ob = bytes((abi.LumObject * len(objs))(*objs)) if objs else b""
    mb = bytes((abi.LumMaterial * len(mats))(*mats)) if mats else b""
    return ob, mb


def _desc_records(world):
    d = world.desc()
    n_o, n_m = d.c.n_objects, d.c.n_materials
    ob = C.string_at(C.addressof(d._objects), n_o * C.sizeof(abi.LumObject))
    mb = C.string_at(C.addressof(d._materials), n_m * C.sizeof(abi.LumMaterial))
    return ob, mb


def _feature_world():
    w = S.World()
    chk = S.Lambertian(texture=S.Checker((0.1, 0.2, 0.3), (0.9, 0.8, 0.7), scale=3.5))
    solid = S.Emissive((1.0, 0.5, 0.25), intensity=4.0, texture=S.SolidColor((0.3, 0.6, 0.9)))
    sub = S.Subsurface((0.8, 0.6, 0.5), 0.2, (0.9, 0.3, 0.2))
    blend = S.Blend(S.Metal((0.9, 0.9, 0.9), 0.1), S.Dielectric(1.33, tint=(0.9, 1.0, 0.95), roughness=0.2), 0.3)
    mats = [chk, solid, sub, blend, S.Iridescent((0.5, 0.5, 0.5), 300.0, 1.4, 0.1), S.Toon((1, 0, 0), 4, 0.5),
            S.Anisotropic((0.4, 0.4, 0.4), 0.1, 0.5, 1), S.Clearcoat((0.2, 0.3, 0.4), 0.8, 1.5),
            S.Velvet((0.5, 0.1, 0.1), 0.7), S.Translucent((0.6, 0.6, 0.2), 0.5, 0.3), S.Microfacet((0.7, 0.7, 0.7)),
            S.Isotropic((0.5, 0.5, 0.5)), S.Transparent()]
    for k, m in enumerate(mats):
        w.add(S.Sphere((k, 0.0, 0.0), 0.4, m))
    w.add(S.Translate(S.RotateY(S.Quad((0, 0, 0), (1, 0, 0), (0, 1, 0), chk), 30.0), (0.0, 2.0, 0.0)))
    w.add(S.MovingSphere((0, 3, 0), (0, 3.5, 0), 0.5, solid))
    w.add(S.Disk((0, 5, 0), (0, -1, 0), 0.7, sub))
    w.add(S.Triangle((0, 0, 1), (1, 0, 1), (0, 1, 1), blend))
    return w


@pytest.mark.parametrize("name", sorted(W.CONFIGS))
def test_workload_desc_matches_field_by_field(name):
    kw = {"level": 3} if name == "dense_mesh" else {}
    world, _ = W.CONFIGS[name](**kw)
    if world._bulk:
        pytest.skip("bulk objects are passed through as records")
    assert _desc_records(world) == _reference_records(world)


def test_feature_world_desc_matches_field_by_field():
    world = _feature_world()
    ob, mb = _desc_records(world)
    rob, rmb = _reference_records(world)
    assert ob == rob
    assert mb == rmb
    # the Blend's children are the records named by its sub indices
    d = world.desc()
    m = np.frombuffer(mb, dtype=S.MATERIAL_DTYPE)
    blends = np.nonzero(m["kind"] == abi.MAT_BLEND)[0]
    assert len(blends) == 1 and set(m["sub"][blends[0]]) <= set(range(d.c.n_materials))


def test_batched_worlds_desc_match_field_by_field():
    for world, _ in W.batched(n_scenes=6, res_choices=(64,), seed=5):
        if world._bulk:
            continue
        assert _desc_records(world) == _reference_records(world)
