"""CPU checks of the C ABI: the library loads, exports every declared entry point, its
structs match the header, and argument errors are reported before any device work."""
import ctypes as C
import os
import re
import subprocess

import pytest

import luminara_b200 as L
from luminara_b200 import abi
from luminara_b200 import scene as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "luminara_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:lum_status|int32_t|const char\*)\s+(lum_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = declared_functions()
    assert "lum_render" in names and "lum_scene_create" in names
    for n in names:
        assert hasattr(lib, n), f"missing export {n}"
    assert lib.lum_abi_version() == abi.LUM_ABI_VERSION


def test_struct_layouts_match_header(tmp_path):
    structs = list(abi.STRUCT_SIZES)
    prog = tmp_path / "sizes.c"
    prog.write_text('#include <stdio.h>\n#include "luminara_gpu.h"\nint main(void){\n' +
                    "".join(f'printf("{s} %zu\\n", sizeof({s}));\n' for s in structs) + "return 0;}\n")
    exe = tmp_path / "sizes"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    for line in out.strip().splitlines():
        name, size = line.split()
        assert abi.STRUCT_SIZES[name] == int(size), name


def test_null_arguments_rejected():
    lib = L.lib()
    h = C.c_void_p()
    assert lib.lum_scene_create(None, C.byref(h)) == abi.LUM_ERR_INVALID_ARGUMENT
    assert b"null" in lib.lum_last_error()
    assert lib.lum_render(None, None, None, None) == abi.LUM_ERR_INVALID_ARGUMENT
    assert lib.lum_intersect(None, None, 1, None) == abi.LUM_ERR_INVALID_ARGUMENT
    assert lib.lum_scene_destroy(None) == abi.LUM_OK


def test_bad_material_rejected():
    w = S.World()
    w.add(S.Sphere((0, 0, 0), 1.0, S.Lambertian((0.5, 0.5, 0.5))))
    d = w.desc()
    d.c.objects[0].material = 5            # out of range
    h = C.c_void_p()
    assert L.lib().lum_scene_create(d.ref(), C.byref(h)) == abi.LUM_ERR_INVALID_ARGUMENT
    assert b"material" in L.lib().lum_last_error()


def test_unknown_object_kind_rejected():
    w = S.World()
    w.add(S.Sphere((0, 0, 0), 1.0, S.Lambertian((0.5, 0.5, 0.5))))
    d = w.desc()
    d.c.objects[0].kind = 99
    h = C.c_void_p()
    assert L.lib().lum_scene_create(d.ref(), C.byref(h)) == abi.LUM_ERR_INVALID_ARGUMENT


def test_transformed_fog_unsupported():
    w = S.World()
    w.add(S.Translate(S.ConstantMedium(S.Sphere((0, 0, 0), 1.0, None), 0.5, (1, 1, 1)), (1, 0, 0)))
    d = w.desc()
    h = C.c_void_p()
    assert L.lib().lum_scene_create(d.ref(), C.byref(h)) == abi.LUM_ERR_UNSUPPORTED


def _create_status(world):
    d = world.desc()
    h = C.c_void_p()
    rc = L.lib().lum_scene_create(d.ref(), C.byref(h))
    return rc, L.lib().lum_last_error()


def _one(prim):
    w = S.World()
    w.add(S.Sphere((0, 0, -3), 0.5, S.Lambertian((0.5, 0.5, 0.5))))
    w.add(prim)
    return w


@pytest.mark.parametrize("bad", [
    lambda m: S.Sphere((float("nan"), 0, 0), 1.0, m),
    lambda m: S.Sphere((0, 0, 0), float("inf"), m),
    lambda m: S.MovingSphere((0, 0, 0), (0, float("nan"), 0), 1.0, m),
    lambda m: S.Quad((0, 0, 0), (1, 0, float("inf")), (0, 1, 0), m),
    lambda m: S.XzRect(0, 1, 0, float("nan"), 2, m),
    lambda m: S.Triangle((0, 0, 0), (1, 0, 0), (0, 1e39, 0), m),          # beyond the f32 range
    lambda m: S.Disk((0, 0, 0), (0, float("nan"), 0), 1.0, m),
    lambda m: S.Plane((0, 0, 0), (0, 1, float("-inf")), m),
    lambda m: S.make_box((0, 0, 0), (1, float("nan"), 1), m),
    lambda m: S.ConstantMedium(S.Sphere((0, 0, 0), 1.0, None), float("nan"), (1, 1, 1)),
    lambda m: S.Translate(S.Sphere((0, 0, 0), 1.0, m), (0, float("inf"), 0)),
    lambda m: S.Scale(S.Sphere((1e30, 0, 0), 1.0, m), 1e10),                # finite inputs, f32 overflow
])
def test_non_finite_geometry_rejected_before_device_work(bad):
    """Non-finite parameters never reach the BVH builder (whose bin index would convert a NaN
    to an integer) or the device: LUM_ERR_INVALID_ARGUMENT names the object.  The reference's
    loader only ever sees finite TOML numbers (scene.rs:846)."""
    rc, msg = _create_status(_one(bad(S.Lambertian((0.5, 0.5, 0.5)))))
    assert rc == abi.LUM_ERR_INVALID_ARGUMENT, msg
    assert b"object 1" in msg or b"transform" in msg


@pytest.mark.parametrize("bad,word", [
    (lambda m: S.Quad((0, 0, 0), (1, 0, 0), (2, 0, 0), m), b"degenerate quad"),
    (lambda m: S.XyRect(0, 0, 0, 1, 2, m), b"degenerate rect"),
    (lambda m: S.Disk((0, 0, 0), (0, 1, 0), 0.0, m), b"degenerate disk"),
    (lambda m: S.ConstantMedium(S.Sphere((0, 0, 0), 1.0, None), -0.5, (1, 1, 1)), b"density"),
])
def test_degenerate_geometry_rejected(bad, word):
    rc, msg = _create_status(_one(bad(S.Lambertian((0.5, 0.5, 0.5)))))
    assert rc == abi.LUM_ERR_INVALID_ARGUMENT, msg
    assert word in msg and b"object 1" in msg


def test_non_finite_mesh_material_light_camera_rejected():
    import numpy as np

    w = S.World()
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, float("nan")]], float)
    w.add_mesh(S.Mesh(pos, np.array([[0, 1, 2]], np.uint32), S.Lambertian((0.5, 0.5, 0.5))))
    rc, msg = _create_status(w)
    assert rc == abi.LUM_ERR_INVALID_ARGUMENT and b"mesh 0 vertex 2" in msg, msg

    w = _one(S.Sphere((0, 1, 0), 1.0, S.Metal((0.5, float("nan"), 0.5), 0.1)))
    rc, msg = _create_status(w)
    assert rc == abi.LUM_ERR_INVALID_ARGUMENT and b"material" in msg, msg

    w = _one(S.Sphere((0, 1, 0), 1.0, S.Lambertian((0.5, 0.5, 0.5))))
    w.add_light(S.LightInfo.Sphere((0, 5, 0), float("inf"), (4, 4, 4)))
    rc, msg = _create_status(w)
    assert rc == abi.LUM_ERR_INVALID_ARGUMENT and b"light 0" in msg, msg

    w = _one(S.Sphere((0, 1, 0), 1.0, S.Lambertian((0.5, 0.5, 0.5))))
    w.camera.look_from = (0, 0, float("nan"))
    rc, msg = _create_status(w)
    assert rc == abi.LUM_ERR_INVALID_ARGUMENT and b"camera" in msg, msg


def test_valid_edge_geometry_passes_validation():
    """Finite edge cases the reference renders are not rejected: a box flat along one axis (its
    four zero-area sides are left out), a sphere of negative radius (inward normals), a fog of
    density 0 and a degenerate mesh triangle.  On a machine without a GPU the call then fails at
    the first CUDA call, not in validation."""
    import numpy as np

    w = S.World()
    m = S.Lambertian((0.5, 0.5, 0.5))
    w.add(S.make_box((0, 0, 0), (1, 0, 1), m))
    w.add(S.Sphere((0, 0, 0), -1.0, m))
    w.add(S.ConstantMedium(S.Sphere((0, 0, 0), 1.0, None), 0.0, (1, 1, 1)))
    w.add_mesh(S.Mesh(np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0]], float), np.array([[0, 1, 2]], np.uint32), m))
    rc, msg = _create_status(w)
    assert rc != abi.LUM_ERR_INVALID_ARGUMENT, msg
    if rc == abi.LUM_OK:
        return
    assert rc in (abi.LUM_ERR_NO_DEVICE, abi.LUM_ERR_CUDA), msg
