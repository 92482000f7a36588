"""TOML scene front end: the reference's scene files -> World + RenderConfig.

Restates `scene::load_scene` (src/scene.rs:846-1645) and `build_material`
(src/scene.rs:1709-2048) for the primitives, materials and backgrounds the device path
renders, so `examples/scenes/*.toml` files feed the drop-in directly:

    cfg, world, post = load_scene_file("cornell.toml")
    img, stats = luminara_b200.GpuScene(world).render(cfg)

What is kept from the reference, on purpose:
  * defaults: RenderConfig (src/render.rs:423-450), CameraConfig (src/camera.rs:32-45, aspect
    = width / height), material option defaults (fuzz 0, roughness 0.5, metallic 0,
    intensity 1, checker scale 1, [[light]] colour 1 / intensity 10 / radius 0.1);
  * object order (spheres, moving spheres, planes, lights, fog, disks, triangles, quads,
    meshes, boxes, rect_xy, rect_xz, rect_yz), which fixes primitive ids;
  * light harvesting for NEE: emissive or blackbody spheres (at their untransformed centre),
    [[light]] entries, emissive or blackbody disks (unit normal) and quads (normal
    unit(u x v)), and emissive rect_xz (normal -y); emissive rect_xy / rect_yz and boxes are
    not harvested, exactly as in the reference;
  * transform order: sphere RotateX, RotateY, RotateZ, Translate, Scale; box Scale, RotateX,
    RotateY, RotateZ, Translate.

Post-processing settings (tone_map, gamma, bloom, ...) are returned in `post` untouched: they
act on the finished image, after the sample loop.  Anything the device path does not
render (other primitives, procedural/image textures, bump/normal maps, non-uniform box scale)
raises UnsupportedSceneError naming every such item, instead of rendering a different scene.
"""
from __future__ import annotations

import math
import os
import tomllib
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import abi
from . import scene as S

# RenderSettings keys the sample loop reads; every other [render] key is post-processing.
_PATH_KEYS = {"width", "height", "samples", "max_depth", "seed", "exposure", "pixel_filter", "background",
              "adaptive", "adaptive_threshold"}
# [render] keys whose feature is in the sample loop but not built here.
_UNBUILT_RENDER_KEYS = {"firefly_filter", "lens_distortion", "chromatic_aberration"}
_SUPPORTED_TABLES = {"render", "camera", "sphere", "moving_sphere", "plane", "light", "fog", "disk", "triangle",
                     "quad", "mesh", "box", "rect_xy", "rect_xz", "rect_yz"}


class UnsupportedSceneError(ValueError):
    """The scene uses features outside the device path; `items` lists them."""

    def __init__(self, items: List[str]):
        self.items = items
        super().__init__("scene uses features this renderer does not implement: " + "; ".join(items))


def blackbody_to_rgb(temperature: float) -> Tuple[float, float, float]:
    """Colour of a black body at `temperature` K (src/scene.rs:1679-1707): the piecewise
    log/power fit of Tanner Helland ("How to Convert Temperature (K) to RGB", 2012) to CIE
    1964 blackbody colours, temperature clamped to [1000, 40000] K, channels in [0, 1]."""
    t = min(max(temperature, 1000.0), 40000.0) / 100.0
    if t <= 66.0:
        r = 1.0
        g = min(max(99.4708025861 * math.log(t) - 161.1195681661, 0.0), 255.0) / 255.0
    else:
        r = min(max(329.698727446 * (t - 60.0) ** -0.1332047592 / 255.0, 0.0), 1.0)
        g = min(max(288.1221695283 * (t - 60.0) ** -0.0755148492 / 255.0, 0.0), 1.0)
    if t >= 66.0:
        b = 1.0
    elif t <= 19.0:
        b = 0.0
    else:
        b = min(max(138.5177312231 * math.log(t - 10.0) - 305.0447927307, 0.0), 255.0) / 255.0
    return (r, g, b)


def _v3(a) -> Tuple[float, float, float]:
    return (float(a[0]), float(a[1]), float(a[2]))


def _unit(a) -> Tuple[float, float, float]:
    v = np.asarray(a, dtype=np.float64)
    return _v3(v / np.linalg.norm(v))


class _Loader:
    def __init__(self, base_dir: str):
        self.base_dir = base_dir
        self.unsupported: List[str] = []
        self.env_map: Optional[np.ndarray] = None

    def bad(self, what: str):
        if what not in self.unsupported:
            self.unsupported.append(what)

    # ------------------------------------------------------------------ materials
    def material(self, desc: dict, where: str) -> Optional[S.Material]:
        """build_material (src/scene.rs:1709-2048) for the in-scope material types."""
        t = desc.get("type", "")
        c = desc.get("color")
        if t in ("Lambertian", "lambertian", "matte"):
            return S.Lambertian(_v3(c))
        if t in ("Metal", "metal"):
            return S.Metal(_v3(c), float(desc.get("fuzz", 0.0)))
        if t in ("Dielectric", "dielectric"):
            tint = desc.get("tint")
            return S.Dielectric(float(desc["refraction_index"]), _v3(tint) if tint is not None else (1.0, 1.0, 1.0),
                                roughness=float(desc.get("roughness", 0.0)),
                                dispersion=float(desc.get("dispersion", 0.0)))
        if t in ("Emissive", "emissive"):
            if desc.get("texture") is not None:
                self.bad(f"{where}: emissive image texture")
                return None
            return S.Emissive(_v3(c), float(desc.get("intensity", 1.0)))
        if t in ("Microfacet", "microfacet", "pbr"):
            if desc.get("texture") is not None:
                self.bad(f"{where}: microfacet image texture")
                return None
            return S.Microfacet(_v3(c), roughness=float(desc.get("roughness", 0.5)),
                                metallic=float(desc.get("metallic", 0.0)))
        if t in ("Checker", "checker"):
            return S.Lambertian(texture=S.Checker(_v3(desc["color1"]), _v3(desc["color2"]),
                                                  float(desc.get("scale", 1.0))))
        if t in ("Mirror", "mirror"):
            return S.Metal((0.95, 0.95, 0.95), 0.0)
        if t in ("Glass", "glass"):
            return S.Dielectric(1.5)
        if t in ("Blackbody", "blackbody"):
            return S.Emissive(blackbody_to_rgb(float(desc["temperature"])), float(desc.get("intensity", 1.0)))
        # the other materials, with build_material's defaults (src/scene.rs:1823-1832, 1991-2047)
        if t in ("Toon", "toon", "cel"):
            return S.Toon(_v3(c), int(desc.get("bands", 3)), float(desc.get("specular", 0.5)))
        if t in ("Anisotropic", "anisotropic", "brushed"):
            return S.Anisotropic(_v3(c), float(desc.get("roughness_u", 0.1)), float(desc.get("roughness_v", 0.5)),
                                 int(desc.get("tangent_axis", 1)))
        if t in ("Clearcoat", "clearcoat"):
            return S.Clearcoat(_v3(c), float(desc.get("coat_gloss", 0.8)), float(desc.get("coat_ior", 1.5)))
        if t in ("Velvet", "velvet"):
            return S.Velvet(_v3(c), float(desc.get("sheen", 1.0)))
        if t in ("Iridescent", "iridescent"):
            return S.Iridescent(_v3(c if c is not None else (0.9, 0.9, 0.9)), float(desc.get("thickness", 400.0)),
                                float(desc.get("film_ior", 1.4)), float(desc.get("roughness", 0.05)))
        if t in ("Translucent", "translucent"):
            return S.Translucent(_v3(c), float(desc.get("translucency", 0.5)), float(desc.get("scatter_width", 0.8)))
        if t in ("Subsurface", "subsurface", "sss"):
            return S.Subsurface(_v3(c), float(desc.get("mean_free_path", 0.5)),
                                _v3(desc.get("scatter_color", (0.8, 0.5, 0.5))))
        if t in ("BlendMat", "blend"):
            a = self.material(desc["material_a"], where + ".material_a")
            b = self.material(desc["material_b"], where + ".material_b")
            if a is None or b is None:
                return None
            return S.Blend(a, b, float(desc.get("ratio", 0.5)))
        if t in ("Opacity", "opacity", "alpha"):
            inner = self.material(desc["material"], where + ".material")
            if inner is None:
                return None
            return S.Blend(inner, S.Transparent(), min(max(float(desc["opacity"]), 0.0), 1.0))
        self.bad(f"{where}: material type '{t}'")
        return None

    @staticmethod
    def emission(desc: dict, blackbody: bool = True) -> Optional[Tuple[float, float, float]]:
        """Emission of an emissive (or blackbody) material description, for light harvesting."""
        t = desc.get("type", "")
        if t in ("Emissive", "emissive"):
            k = float(desc.get("intensity", 1.0))
            return tuple(float(x) * k for x in desc["color"])
        if blackbody and t in ("Blackbody", "blackbody"):
            k = float(desc.get("intensity", 1.0))
            return tuple(x * k for x in blackbody_to_rgb(float(desc["temperature"])))
        return None

    # ------------------------------------------------------------------ meshes
    def mesh(self, m: dict, mat: S.Material) -> List[S.Mesh]:
        """load_obj / load_ply (src/obj.rs:18-150, 154-241): positions scaled then offset, fan
        triangulation, smooth normals where all three face vertices name one."""
        path = m["file"]
        if not os.path.isabs(path) and not os.path.exists(path):
            path = os.path.join(self.base_dir, path)
        scale = float(m.get("scale", 1.0))
        offset = np.asarray(m.get("offset", (0.0, 0.0, 0.0)), dtype=np.float64)
        with open(path) as f:
            text = f.read()
        if path.endswith(".ply"):
            tris, norms = _load_ply(text, scale, offset)
        else:
            tris, norms = _load_obj(text, scale, offset)
        # consecutive runs of flat / smooth triangles become one Mesh each (order kept)
        out: List[S.Mesh] = []
        i = 0
        while i < len(tris):
            smooth = norms[i] is not None
            j = i
            while j < len(tris) and (norms[j] is not None) == smooth:
                j += 1
            pos = np.array(tris[i:j], dtype=np.float64).reshape(-1, 3)
            idx = np.arange(len(pos), dtype=np.uint32).reshape(-1, 3)
            nrm = np.array(norms[i:j], dtype=np.float64).reshape(-1, 3) if smooth else None
            out.append(S.Mesh(positions=pos, indices=idx, material=mat, normals=nrm))
            i = j
        return out

    # ------------------------------------------------------------------ scene
    def load(self, doc: dict) -> Tuple[S.RenderConfig, S.World, Dict]:
        for k in doc:
            if k not in _SUPPORTED_TABLES:
                n = len(doc[k]) if isinstance(doc[k], list) else 1
                self.bad(f"{n} x [{k}]")
        cfg = S.RenderConfig()
        post: Dict = {}
        r = doc.get("render", {})
        for k, v in r.items():
            if k in _UNBUILT_RENDER_KEYS:
                if v not in (False, 0, 0.0, None):
                    self.bad(f"render.{k}")
            elif k not in _PATH_KEYS:
                post[k] = v
        cfg.width = int(r.get("width", cfg.width))
        cfg.height = int(r.get("height", cfg.height))
        cfg.samples_per_pixel = int(r.get("samples", cfg.samples_per_pixel))
        cfg.max_depth = int(r.get("max_depth", cfg.max_depth))
        cfg.seed = int(r.get("seed", cfg.seed))
        cfg.exposure = float(r.get("exposure", cfg.exposure))
        cfg.adaptive = bool(r.get("adaptive", cfg.adaptive))                    # scene.rs:914-919
        cfg.adaptive_threshold = float(r.get("adaptive_threshold", cfg.adaptive_threshold))
        pf = r.get("pixel_filter")
        if pf is not None:
            cfg.pixel_filter = {"triangle": abi.FILTER_TRIANGLE, "tent": abi.FILTER_TRIANGLE,
                                "gaussian": abi.FILTER_GAUSSIAN, "gauss": abi.FILTER_GAUSSIAN,
                                "mitchell": abi.FILTER_MITCHELL}.get(pf, abi.FILTER_BOX)
        if "background" in r:
            self.background(r["background"], cfg)

        world = S.World()
        world.env_map = self.env_map
        cam = S.CameraConfig(aspect_ratio=cfg.width / cfg.height)
        c = doc.get("camera", {})
        if "look_from" in c:
            cam.look_from = _v3(c["look_from"])
        if "look_at" in c:
            cam.look_at = _v3(c["look_at"])
        if "vup" in c:
            cam.vup = _v3(c["vup"])
        cam.vfov_degrees = float(c.get("vfov", cam.vfov_degrees))
        cam.aperture = float(c.get("aperture", cam.aperture))
        cam.focus_dist = float(c.get("focus_dist", cam.focus_dist))
        cam.panorama = c.get("panorama") is True                        # scene.rs:1170-1172
        world.camera = cam

        def add(obj, mat, light=None):
            if mat is None:
                return
            world.add(obj)
            if light is not None:
                world.add_light(light, material=mat)

        for i, s in enumerate(doc.get("sphere", [])):
            where = f"sphere[{i}]"
            for k in ("bump_strength", "normal_map"):
                if k in s:
                    self.bad(f"{where}.{k}")
            mat = self.material(s["material"], where)
            e = self.emission(s["material"])
            light = S.LightInfo.Sphere(_v3(s["center"]), float(s["radius"]), e) if e is not None else None
            obj = S.Sphere(_v3(s["center"]), float(s["radius"]), mat)
            if "rotate_x" in s:
                obj = S.RotateX(obj, float(s["rotate_x"]))
            if "rotate_y" in s:
                obj = S.RotateY(obj, float(s["rotate_y"]))
            if "rotate_z" in s:
                obj = S.RotateZ(obj, float(s["rotate_z"]))
            if "translate" in s:
                obj = S.Translate(obj, _v3(s["translate"]))
            if "scale" in s:
                obj = S.Scale(obj, float(s["scale"]))
            add(obj, mat, light)
        for i, s in enumerate(doc.get("moving_sphere", [])):
            mat = self.material(s["material"], f"moving_sphere[{i}]")
            add(S.MovingSphere(_v3(s["center0"]), _v3(s["center1"]), float(s["radius"]), mat), mat)
        for i, p in enumerate(doc.get("plane", [])):
            mat = self.material(p["material"], f"plane[{i}]")
            add(S.Plane(_v3(p["point"]), _v3(p["normal"]), mat), mat)
        for l in doc.get("light", []):
            color = _v3(l.get("color", (1.0, 1.0, 1.0)))
            k = float(l.get("intensity", 10.0))
            rad = float(l.get("radius", 0.1))
            mat = S.Emissive(color, k)
            add(S.Sphere(_v3(l["position"]), rad, mat), mat,
                S.LightInfo.Sphere(_v3(l["position"]), rad, tuple(x * k for x in color)))
        for f in doc.get("fog", []):
            world.add(S.ConstantMedium(S.Sphere(_v3(f["center"]), float(f["radius"]), S.Lambertian((0.0, 0.0, 0.0))),
                                       float(f["density"]), _v3(f["color"])))
        for i, d in enumerate(doc.get("disk", [])):
            mat = self.material(d["material"], f"disk[{i}]")
            e = self.emission(d["material"])
            light = (S.LightInfo.Disk(_v3(d["center"]), _unit(d["normal"]), float(d["radius"]), e)
                     if e is not None else None)
            add(S.Disk(_v3(d["center"]), _v3(d["normal"]), float(d["radius"]), mat), mat, light)
        for i, t in enumerate(doc.get("triangle", [])):
            mat = self.material(t["material"], f"triangle[{i}]")
            add(S.Triangle(_v3(t["v0"]), _v3(t["v1"]), _v3(t["v2"]), mat), mat)
        for i, q in enumerate(doc.get("quad", [])):
            where = f"quad[{i}]"
            if "normal_map" in q:
                self.bad(f"{where}.normal_map")
            mat = self.material(q["material"], where)
            e = self.emission(q["material"])
            light = (S.LightInfo.Rect(_v3(q["q"]), _v3(q["u"]), _v3(q["v"]), _unit(np.cross(q["u"], q["v"])), e)
                     if e is not None else None)
            add(S.Quad(_v3(q["q"]), _v3(q["u"]), _v3(q["v"]), mat), mat, light)
        for i, m in enumerate(doc.get("mesh", [])):
            mat = self.material(m["material"], f"mesh[{i}]")
            if mat is not None:
                for mesh in self.mesh(m, mat):
                    world.add_mesh(mesh)
        for i, b in enumerate(doc.get("box", [])):
            where = f"box[{i}]"
            if "scale_xyz" in b:
                self.bad(f"{where}.scale_xyz")
            mat = self.material(b["material"], where)
            obj = S.make_box(_v3(b["min"]), _v3(b["max"]), mat)
            if "scale" in b:
                obj = S.Scale(obj, float(b["scale"]))
            if "rotate_x" in b:
                obj = S.RotateX(obj, float(b["rotate_x"]))
            if "rotate_y" in b:
                obj = S.RotateY(obj, float(b["rotate_y"]))
            if "rotate_z" in b:
                obj = S.RotateZ(obj, float(b["rotate_z"]))
            if "translate" in b:
                obj = S.Translate(obj, _v3(b["translate"]))
            add(obj, mat)
        for i, rr in enumerate(doc.get("rect_xy", [])):
            mat = self.material(rr["material"], f"rect_xy[{i}]")
            add(S.XyRect(rr["x"][0], rr["x"][1], rr["y"][0], rr["y"][1], rr["k"], mat), mat)
        for i, rr in enumerate(doc.get("rect_xz", [])):
            mat = self.material(rr["material"], f"rect_xz[{i}]")
            e = self.emission(rr["material"], blackbody=False)
            light = None
            if e is not None:
                x0, x1, z0, z1, k = rr["x"][0], rr["x"][1], rr["z"][0], rr["z"][1], rr["k"]
                light = S.LightInfo.Rect((x0, k, z0), (x1 - x0, 0.0, 0.0), (0.0, 0.0, z1 - z0), (0.0, -1.0, 0.0), e)
            add(S.XzRect(rr["x"][0], rr["x"][1], rr["z"][0], rr["z"][1], rr["k"], mat), mat, light)
        for i, rr in enumerate(doc.get("rect_yz", [])):
            mat = self.material(rr["material"], f"rect_yz[{i}]")
            add(S.YzRect(rr["y"][0], rr["y"][1], rr["z"][0], rr["z"][1], rr["k"], mat), mat)
        if self.unsupported:
            raise UnsupportedSceneError(self.unsupported)
        return cfg, world, post

    def background(self, bg: dict, cfg: S.RenderConfig) -> None:
        """BackgroundDesc -> Background (src/scene.rs:1140-1175)."""
        t = bg.get("type", "")
        if t in ("Sky", "sky"):
            cfg.background = abi.BG_SKY
        elif t in ("Solid", "solid"):
            cfg.background, cfg.bg_color = abi.BG_SOLID, _v3(bg["color"])
        elif t in ("Black", "black"):
            cfg.background, cfg.bg_color = abi.BG_SOLID, (0.0, 0.0, 0.0)
        elif t in ("Gradient", "gradient"):
            cfg.background, cfg.bg_color, cfg.bg_color2 = abi.BG_GRADIENT, _v3(bg["bottom"]), _v3(bg["top"])
        elif t in ("Sunset", "sunset"):
            cfg.background = abi.BG_SUN
            cfg.bg_dir, cfg.bg_color, cfg.bg_intensity, cfg.bg_color2 = (0.3, 0.15, -1.0), (1.0, 0.6, 0.2), 30.0, \
                (0.8, 0.4, 0.2)
        elif t in ("Sun", "sun"):
            cfg.background = abi.BG_SUN
            cfg.bg_dir = _v3(bg["direction"])
            cfg.bg_color = _v3(bg.get("sun_color", (1.0, 0.95, 0.85)))
            cfg.bg_intensity = float(bg.get("intensity", 20.0))
            cfg.bg_color2 = _v3(bg.get("sky_color", (0.5, 0.7, 1.0)))
        elif t in ("Starfield", "starfield"):                                   # src/scene.rs:1133-1138
            cfg.background = abi.BG_STARFIELD
            cfg.bg_star_density = float(bg.get("star_density", 1.0))
            cfg.bg_star_brightness = float(bg.get("star_brightness", 5.0))
        elif t in ("EnvMap", "env_map"):                                        # src/scene.rs:1139-1141
            path = bg["file"]
            if not os.path.isabs(path):
                path = os.path.join(self.base_dir, path)
            cfg.background = abi.BG_ENVMAP
            cfg.bg_intensity = float(bg.get("intensity", 1.0))
            self.env_map = load_env_map(path)
        else:
            self.bad(f"render.background type '{t}'")


def _read_radiance_hdr(path: str) -> np.ndarray:
    """Radiance RGBE (.hdr / .pic): header, resolution line, flat or run-length-encoded scanlines;
    each pixel (r, g, b, e) is (r, g, b) * 2^(e - 136), e = 0 black."""
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while True:                                                 # header lines up to a blank line
        end = data.index(b"\n", pos)
        line = data[pos:end].strip()
        pos = end + 1
        if not line:
            break
    end = data.index(b"\n", pos)
    res = data[pos:end].split()
    pos = end + 1
    if len(res) != 4 or res[0] not in (b"-Y", b"+Y") or res[2] != b"+X":
        raise ValueError(f"{path}: unsupported Radiance orientation {res}")
    h, w = int(res[1]), int(res[3])
    buf = np.frombuffer(data, dtype=np.uint8)
    out = np.zeros((h, w, 4), dtype=np.uint8)
    for y in range(h):
        if 8 <= w < 32768 and buf[pos] == 2 and buf[pos + 1] == 2 and (int(buf[pos + 2]) << 8 | int(buf[pos + 3])) == w:
            pos += 4
            for c in range(4):                                  # new-style RLE, one channel at a time
                x = 0
                while x < w:
                    n = int(buf[pos])
                    pos += 1
                    if n > 128:
                        out[y, x:x + n - 128, c] = buf[pos]
                        pos += 1
                        x += n - 128
                    else:
                        out[y, x:x + n, c] = buf[pos:pos + n]
                        pos += n
                        x += n
        else:
            out[y] = buf[pos:pos + 4 * w].reshape(w, 4)
            pos += 4 * w
    if res[0] == b"+Y":
        out = out[::-1]
    e = out[..., 3].astype(np.int32)
    scale = np.where(e > 0, np.ldexp(1.0, e - 136), 0.0)
    return (out[..., :3].astype(np.float64) * scale[..., None]).astype(np.float32)


def load_env_map(path: str) -> np.ndarray:
    """Background::load_env_map (src/render.rs:3589-3602): the image as linear float RGB, top
    row first -- Radiance .hdr as stored, 8/16-bit images divided by 255 / 65535 (no sRGB
    decoding, as image's to_rgb32f)."""
    if path.lower().endswith((".hdr", ".pic")):
        return _read_radiance_hdr(path)
    from PIL import Image
    with Image.open(path) as im:
        if im.mode in ("I;16", "I;16B", "I;16L", "I"):
            return np.repeat((np.asarray(im, dtype=np.float64) / 65535.0)[..., None], 3, axis=2).astype(np.float32)
        a = np.asarray(im.convert("RGB"), dtype=np.float32) / 255.0
    return np.ascontiguousarray(a)


def _load_obj(text: str, scale: float, offset: np.ndarray):
    verts, normals, faces = [], [], []
    for ln, line in enumerate(text.splitlines()):
        line = line.strip()
        if not line or line.startswith("#"):
            continue
        parts = line.split()
        if parts[0] == "v":
            if len(parts) < 4:
                raise ValueError(f"Line {ln + 1}: vertex needs 3 coordinates")
            verts.append(np.array([float(x) for x in parts[1:4]]) * scale + offset)
        elif parts[0] == "vn":
            if len(parts) < 4:
                raise ValueError(f"Line {ln + 1}: normal needs 3 components")
            n = np.array([float(x) for x in parts[1:4]])
            normals.append(n / np.linalg.norm(n))
        elif parts[0] == "f":
            fv = []
            for p in parts[1:]:
                seg = p.split("/")
                fv.append((int(seg[0]), int(seg[2]) if len(seg) >= 3 and seg[2] else None))
            if len(fv) < 3:
                raise ValueError(f"Line {ln + 1}: face needs at least 3 vertices")
            for i in range(1, len(fv) - 1):                                  # fan
                faces.append((fv[0], fv[i], fv[i + 1]))
    tris, norms = [], []
    for f in faces:
        try:
            tris.append([verts[p - 1] for p, _ in f])
        except IndexError:
            raise ValueError(f"Vertex index {max(p for p, _ in f)} out of range")
        ns = [n for _, n in f]
        if all(n is not None and 1 <= n <= len(normals) for n in ns):
            norms.append([normals[n - 1] for n in ns])
        else:
            norms.append(None)
    return tris, norms


def _load_ply(text: str, scale: float, offset: np.ndarray):
    lines = iter(text.splitlines())
    if next(lines, "").strip() != "ply":
        raise ValueError("Not a PLY file (missing 'ply' magic)")
    nv = nf = 0
    for line in lines:
        parts = line.split()
        if line.strip() == "end_header":
            break
        if len(parts) >= 3 and parts[0] == "element":
            if parts[1] == "vertex":
                nv = int(parts[2])
            elif parts[1] == "face":
                nf = int(parts[2])
    else:
        raise ValueError("PLY header not terminated (missing 'end_header')")
    verts = [np.array([float(x) for x in next(lines).split()[:3]]) * scale + offset for _ in range(nv)]
    tris = []
    for _ in range(nf):
        parts = next(lines).split()
        n = int(parts[0])
        idx = [int(x) for x in parts[1:n + 1]]
        for j in range(1, len(idx) - 1):
            tris.append([verts[idx[0]], verts[idx[j]], verts[idx[j + 1]]])
    return tris, [None] * len(tris)


def load_scene(toml_str: str, base_dir: str = ".") -> Tuple[S.RenderConfig, S.World, Dict]:
    """Parses a scene file's text: (RenderConfig, World with camera and NEE lights, post-processing
    settings).  Raises UnsupportedSceneError for features outside the device path."""
    doc = tomllib.loads(toml_str)
    return _Loader(base_dir).load(doc)


def load_scene_file(path: str) -> Tuple[S.RenderConfig, S.World, Dict]:
    with open(path, "rb") as f:
        doc = tomllib.load(f)
    return _Loader(os.path.dirname(os.path.abspath(path))).load(doc)


# [render] settings of the LDR colour chain (lum_render_ldr / lum_tonemap_device).
_TONE_NAMES = {"aces": abi.TONEMAP_ACES, "reinhard": abi.TONEMAP_REINHARD, "filmic": abi.TONEMAP_FILMIC,
               "uncharted2": abi.TONEMAP_FILMIC, "none": abi.TONEMAP_NONE}
_CHAIN_KEYS = {"tone_map", "auto_exposure", "gamma", "dither", "posterize", "vignette", "saturation",
               "white_balance", "hue_shift", "grade_shadows", "grade_highlights", "brightness", "contrast", "sepia",
               "tint", "color_balance"}


def tonemap_config(post: Dict) -> S.ToneMapConfig:
    """The colour-chain settings of a scene file's [render] table (`post` from load_scene) as a
    ToneMapConfig (unknown tone_map names select ACES, as in src/render.rs:1130-1137).  Any other
    active post-processing setting (bloom, denoise, blur, stylisation passes, ...) raises
    UnsupportedSceneError: the chain would otherwise produce a different image."""
    tm = S.ToneMapConfig()
    bad = []
    for k, v in post.items():
        if k in _CHAIN_KEYS:
            if k == "tone_map":
                tm.tone_map = _TONE_NAMES.get(str(v), abi.TONEMAP_ACES)
            elif k in ("grade_shadows", "grade_highlights", "tint", "color_balance"):
                setattr(tm, k, _v3(v))
            elif k in ("auto_exposure", "dither"):
                setattr(tm, k, bool(v))
            elif k == "posterize":
                tm.posterize = int(v)
            else:
                setattr(tm, k, float(v))
        elif not (v in (False, 0, 0.0, "", None) or (k == "solarize" and float(v) < 0.0)):
            bad.append(f"render.{k}")
    if bad:
        raise UnsupportedSceneError(bad)
    return tm
