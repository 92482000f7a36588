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


def test_panorama_unsupported_and_bad_material_rejected():
    w = S.World()
    w.add(S.Sphere((0, 0, 0), 1.0, S.Lambertian((0.5, 0.5, 0.5))))
    w.camera.panorama = True
    with pytest.raises(L.LuminaraError) as e:
        L.GpuScene(w)
    assert e.value.status == abi.LUM_ERR_UNSUPPORTED
    w.camera.panorama = False
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
