"""Scene construction mirroring the reference's Rust types.

Reference names are kept: ``Sphere``, ``MovingSphere``, ``Quad``, ``XyRect``/``XzRect``/
``YzRect``, ``Triangle``, ``Disk``, ``Plane``, ``make_box``, ``Translate``, ``RotateX/Y/Z``,
``Scale``, ``ConstantMedium``, materials ``Lambertian``/``Metal``/``Dielectric``/``Emissive``/
``Microfacet``/``Isotropic``, textures ``SolidColor``/``Checker``, ``LightInfo`` and
``CameraConfig`` (src/sphere.rs, quad.rs, rect.rs, triangle.rs, disk.rs, plane.rs,
transform.rs, constant_medium.rs, material.rs, texture.rs, render.rs:16-39, camera.rs:17-41).

A :class:`World` collects objects the way ``HittableList`` does and is flattened into a
``lum_scene_desc`` (include/luminara_gpu.h); the GPU library and the CPU oracle both consume
that description.  Objects that the reference wraps in transforms become one description
object with a transform record (boxes) or a transformed primitive.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import abi

Vec = Sequence[float]


# --------------------------------------------------------------------------------------
# Textures and materials
# --------------------------------------------------------------------------------------
@dataclass
class SolidColor:
    color: Vec


@dataclass
class Checker:
    even: Vec
    odd: Vec
    scale: float = 1.0


@dataclass
class Material:
    kind: int
    color: Vec = (0.0, 0.0, 0.0)
    texture: object = None
    fuzz: float = 0.0
    ior: float = 1.5
    roughness: float = 0.0
    metallic: float = 0.0
    intensity: float = 1.0
    dispersion: float = 0.0
    tint: Vec = (1.0, 1.0, 1.0)
    color2: Optional[Vec] = None      # Subsurface scatter_color
    extra: Sequence[float] = (0.0, 0.0, 0.0, 0.0)
    children: Optional[Sequence["Material"]] = None   # Blend: (mat_a, mat_b)

    def to_c(self, index_of=None) -> abi.LumMaterial:
        """index_of(material) -> material index; needed by Blend for its children."""
        m = abi.LumMaterial()
        m.kind = self.kind
        m.texture = abi.TEX_SOLID
        m.color[:] = list(map(float, self.color))
        m.tex_scale = 1.0
        tex = self.texture
        if isinstance(tex, SolidColor):
            m.color[:] = list(map(float, tex.color))
        elif isinstance(tex, Checker):
            m.texture = abi.TEX_CHECKER
            m.color[:] = list(map(float, tex.even))
            m.color2[:] = list(map(float, tex.odd))
            m.tex_scale = float(tex.scale)
        m.fuzz = float(self.fuzz)
        m.ior = float(self.ior)
        m.roughness = float(self.roughness)
        m.metallic = float(self.metallic)
        m.intensity = float(self.intensity)
        m.dispersion = float(self.dispersion)
        m.tint[:] = list(map(float, self.tint))
        if self.color2 is not None:
            m.color2[:] = list(map(float, self.color2))
        m.extra[:] = [float(x) for x in tuple(self.extra) + (0.0,) * (4 - len(self.extra))]
        if self.children is not None:
            m.sub[:] = [index_of(c) for c in self.children]
        return m


def Lambertian(albedo: Vec = (0.5, 0.5, 0.5), texture=None) -> Material:
    return Material(abi.MAT_LAMBERTIAN, color=albedo, texture=texture)


def Metal(albedo: Vec, fuzz: float = 0.0) -> Material:
    return Material(abi.MAT_METAL, color=albedo, fuzz=fuzz)


def Dielectric(refraction_index: float, tint: Vec = (1.0, 1.0, 1.0), roughness: float = 0.0,
               dispersion: float = 0.0) -> Material:
    return Material(abi.MAT_DIELECTRIC, ior=refraction_index, tint=tint, roughness=roughness,
                    dispersion=dispersion)


def Emissive(color: Vec, intensity: float = 1.0, texture=None) -> Material:
    return Material(abi.MAT_EMISSIVE, color=color, intensity=intensity, texture=texture)


def Microfacet(albedo: Vec, roughness: float = 0.5, metallic: float = 0.0, texture=None) -> Material:
    return Material(abi.MAT_MICROFACET, color=albedo, roughness=roughness, metallic=metallic, texture=texture)


def Isotropic(albedo: Vec) -> Material:
    return Material(abi.MAT_ISOTROPIC, color=albedo)


# The other reference materials (material.rs:396-865); clamps are applied by the library.
def Blend(mat_a: Material, mat_b: Material, ratio: float) -> Material:
    return Material(abi.MAT_BLEND, extra=(ratio,), children=(mat_a, mat_b))


def Transparent() -> Material:
    return Material(abi.MAT_TRANSPARENT)


def Iridescent(base_color: Vec, thickness: float, film_ior: float, roughness: float) -> Material:
    return Material(abi.MAT_IRIDESCENT, color=base_color, extra=(thickness,), ior=film_ior, roughness=roughness)


def Toon(color: Vec, bands: int, specular: float) -> Material:
    return Material(abi.MAT_TOON, color=color, extra=(bands, specular))


def Anisotropic(color: Vec, roughness_u: float, roughness_v: float, tangent_axis: int) -> Material:
    return Material(abi.MAT_ANISOTROPIC, color=color, extra=(roughness_u, roughness_v, tangent_axis))


def Clearcoat(base_color: Vec, coat_gloss: float, coat_ior: float) -> Material:
    return Material(abi.MAT_CLEARCOAT, color=base_color, extra=(coat_gloss,), ior=coat_ior)


def Velvet(color: Vec, sheen: float) -> Material:
    return Material(abi.MAT_VELVET, color=color, extra=(sheen,))


def Translucent(color: Vec, translucency: float, scatter_width: float) -> Material:
    return Material(abi.MAT_TRANSLUCENT, color=color, extra=(translucency, scatter_width))


def Subsurface(color: Vec, mean_free_path: float, scatter_color: Vec) -> Material:
    return Material(abi.MAT_SUBSURFACE, color=color, extra=(mean_free_path,), color2=scatter_color)


# --------------------------------------------------------------------------------------
# Geometry
# --------------------------------------------------------------------------------------
@dataclass
class Prim:
    kind: int
    params: List[float]
    material: Optional[Material]
    xforms: List[tuple] = field(default_factory=list)


def Sphere(center: Vec, radius: float, material: Material) -> Prim:
    return Prim(abi.OBJ_SPHERE, [*center, radius], material)


def MovingSphere(center0: Vec, center1: Vec, radius: float, material: Material) -> Prim:
    return Prim(abi.OBJ_MOVING_SPHERE, [*center0, *center1, radius], material)


def Quad(q: Vec, u: Vec, v: Vec, material: Material) -> Prim:
    return Prim(abi.OBJ_QUAD, [*q, *u, *v], material)


def XyRect(x0, x1, y0, y1, k, material) -> Prim:
    return Prim(abi.OBJ_RECT_XY, [x0, x1, y0, y1, k], material)


def XzRect(x0, x1, z0, z1, k, material) -> Prim:
    return Prim(abi.OBJ_RECT_XZ, [x0, x1, z0, z1, k], material)


def YzRect(y0, y1, z0, z1, k, material) -> Prim:
    return Prim(abi.OBJ_RECT_YZ, [y0, y1, z0, z1, k], material)


def Triangle(v0: Vec, v1: Vec, v2: Vec, material: Material) -> Prim:
    return Prim(abi.OBJ_TRIANGLE, [*v0, *v1, *v2], material)


def Disk(center: Vec, normal: Vec, radius: float, material: Material) -> Prim:
    return Prim(abi.OBJ_DISK, [*center, *normal, radius], material)


def Plane(point: Vec, normal: Vec, material: Material) -> Prim:
    return Prim(abi.OBJ_PLANE, [*point, *normal], material)


def make_box(p_min: Vec, p_max: Vec, material: Material) -> Prim:
    """Six axis rects (src/rect.rs:128-141) kept together so transforms wrap them as one
    composite object, as src/scene.rs:1561-1600 does."""
    return Prim(abi.OBJ_BOX, [*p_min, *p_max], material)


def ConstantMedium(boundary: Prim, density: float, color: Vec) -> Prim:
    """Fog inside a sphere or box boundary (src/constant_medium.rs:9-74)."""
    if boundary.kind == abi.OBJ_SPHERE:
        return Prim(abi.OBJ_FOG_SPHERE, [*boundary.params[:4], density], Isotropic(color))
    if boundary.kind == abi.OBJ_BOX:
        return Prim(abi.OBJ_FOG_BOX, [*boundary.params[:6], density], Isotropic(color))
    raise ValueError("ConstantMedium boundary must be a Sphere or make_box")


def _wrap(obj: Prim, op: int, arg) -> Prim:
    return Prim(obj.kind, obj.params, obj.material, obj.xforms + [(op, arg)])


def Translate(obj: Prim, offset: Vec) -> Prim:
    return _wrap(obj, abi.XF_TRANSLATE, tuple(offset))


def RotateX(obj: Prim, degrees: float) -> Prim:
    return _wrap(obj, abi.XF_ROTATE_X, (degrees, 0.0, 0.0))


def RotateY(obj: Prim, degrees: float) -> Prim:
    return _wrap(obj, abi.XF_ROTATE_Y, (degrees, 0.0, 0.0))


def RotateZ(obj: Prim, degrees: float) -> Prim:
    return _wrap(obj, abi.XF_ROTATE_Z, (degrees, 0.0, 0.0))


def Scale(obj: Prim, factor: float) -> Prim:
    return _wrap(obj, abi.XF_SCALE, (factor, 0.0, 0.0))


@dataclass
class Mesh:
    """Triangle mesh (MeshTriangle, src/obj.rs:250-320): one primitive per triangle."""
    positions: np.ndarray            # (V,3) float64
    indices: np.ndarray              # (T,3) uint32
    material: Optional[Material] = None
    tri_material: Optional[np.ndarray] = None   # (T,) indices into World.materials
    normals: Optional[np.ndarray] = None        # (V,3)


# --------------------------------------------------------------------------------------
# Lights and camera
# --------------------------------------------------------------------------------------
@dataclass
class LightInfo:
    kind: int
    p0: Vec = (0.0, 0.0, 0.0)
    u: Vec = (0.0, 0.0, 0.0)
    v: Vec = (0.0, 0.0, 0.0)
    normal: Vec = (0.0, 1.0, 0.0)
    radius: float = 0.0
    emission: Vec = (0.0, 0.0, 0.0)

    @staticmethod
    def Sphere(center: Vec, radius: float, emission: Vec) -> "LightInfo":
        return LightInfo(abi.LIGHT_SPHERE, p0=center, radius=radius, emission=emission)

    @staticmethod
    def Rect(origin: Vec, u: Vec, v: Vec, normal: Vec, emission: Vec) -> "LightInfo":
        return LightInfo(abi.LIGHT_RECT, p0=origin, u=u, v=v, normal=normal, emission=emission)

    @staticmethod
    def Disk(center: Vec, normal: Vec, radius: float, emission: Vec) -> "LightInfo":
        return LightInfo(abi.LIGHT_DISK, p0=center, normal=normal, radius=radius, emission=emission)

    def to_c(self) -> abi.LumLight:
        l = abi.LumLight()
        l.kind = self.kind
        l.p0[:] = list(map(float, self.p0))
        l.u[:] = list(map(float, self.u))
        l.v[:] = list(map(float, self.v))
        l.normal[:] = list(map(float, self.normal))
        l.radius = float(self.radius)
        l.emission[:] = list(map(float, self.emission))
        return l


@dataclass
class CameraConfig:
    """camera.rs:17-41 defaults."""
    look_from: Vec = (0.0, 1.0, 3.0)
    look_at: Vec = (0.0, 0.0, 0.0)
    vup: Vec = (0.0, 1.0, 0.0)
    vfov_degrees: float = 40.0
    aspect_ratio: float = 16.0 / 9.0
    aperture: float = 0.0
    focus_dist: float = 1.0
    panorama: bool = False

    def to_c(self) -> abi.LumCamera:
        c = abi.LumCamera()
        c.look_from[:] = list(map(float, self.look_from))
        c.look_at[:] = list(map(float, self.look_at))
        c.vup[:] = list(map(float, self.vup))
        c.vfov_degrees = float(self.vfov_degrees)
        c.aspect_ratio = float(self.aspect_ratio)
        c.aperture = float(self.aperture)
        c.focus_dist = float(self.focus_dist)
        c.panorama = 1 if self.panorama else 0
        return c


@dataclass
class RenderConfig:
    """The RenderConfig fields the sample loop reads (render.rs:239-431 defaults)."""
    width: int = 800
    height: int = 450
    samples_per_pixel: int = 100
    max_depth: int = 50
    seed: int = 31337
    background: int = abi.BG_SKY
    bg_color: Vec = (0.0, 0.0, 0.0)
    bg_color2: Vec = (0.0, 0.0, 0.0)
    bg_dir: Vec = (0.0, 1.0, 0.0)
    bg_intensity: float = 0.0
    pixel_filter: int = abi.FILTER_BOX
    exposure: float = 1.0
    crop: Optional[Sequence[int]] = None
    sample_begin: int = 0
    sample_count: int = 0
    adaptive: bool = False
    adaptive_threshold: float = 0.03
    time_limit: float = 0.0
    bg_star_density: float = 0.0      # BG_STARFIELD
    bg_star_brightness: float = 0.0

    def to_c(self) -> abi.LumRenderParams:
        p = abi.LumRenderParams()
        p.width = int(self.width)
        p.height = int(self.height)
        p.samples_per_pixel = int(self.samples_per_pixel)
        p.max_depth = int(self.max_depth)
        p.seed = int(self.seed) & 0xFFFFFFFFFFFFFFFF
        p.background = int(self.background)
        p.pixel_filter = int(self.pixel_filter)
        p.bg_color[:] = list(map(float, self.bg_color))
        p.bg_color2[:] = list(map(float, self.bg_color2))
        p.bg_dir[:] = list(map(float, self.bg_dir))
        p.bg_intensity = float(self.bg_intensity)
        p.exposure = float(self.exposure)
        if self.crop is not None:
            p.has_crop = 1
            p.crop[:] = [int(x) for x in self.crop]
        p.sample_begin = int(self.sample_begin)
        p.sample_count = int(self.sample_count)
        p.adaptive = 1 if self.adaptive else 0
        p.adaptive_threshold = float(self.adaptive_threshold)
        p.time_limit = float(self.time_limit)
        p.bg_star_density = float(self.bg_star_density)
        p.bg_star_brightness = float(self.bg_star_brightness)
        return p

    def out_shape(self):
        w = max(self.width, 1)
        h = max(self.height, 1)
        if self.crop is not None:
            w = min(self.crop[2], w)
            h = min(self.crop[3], h)
        return (h, w, 3)


@dataclass
class ToneMapConfig:
    """The RenderConfig fields of the LDR colour chain (src/render.rs:423-510 defaults)."""
    tone_map: int = abi.TONEMAP_ACES
    auto_exposure: bool = False
    exposure: float = 1.0          # used by tonemap_device; render_ldr takes the render's exposure
    gamma: float = 0.0
    dither: bool = False
    posterize: int = 0
    vignette: float = 0.0
    saturation: float = 1.0
    white_balance: float = 0.0
    hue_shift: float = 0.0
    grade_shadows: Vec = (1.0, 1.0, 1.0)
    grade_highlights: Vec = (1.0, 1.0, 1.0)
    brightness: float = 0.0
    contrast: float = 1.0
    sepia: float = 0.0
    tint: Vec = (1.0, 1.0, 1.0)
    color_balance: Vec = (1.0, 1.0, 1.0)

    def to_c(self) -> abi.LumTonemapParams:
        t = abi.LumTonemapParams()
        for f in ("tone_map", "posterize"):
            setattr(t, f, int(getattr(self, f)))
        for f in ("auto_exposure", "dither"):
            setattr(t, f, 1 if getattr(self, f) else 0)
        for f in ("exposure", "gamma", "vignette", "saturation", "white_balance", "hue_shift", "brightness",
                  "contrast", "sepia"):
            setattr(t, f, float(getattr(self, f)))
        for f in ("grade_shadows", "grade_highlights", "tint", "color_balance"):
            getattr(t, f)[:] = [float(x) for x in getattr(self, f)]
        return t

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f in self.__dataclass_fields__}


# --------------------------------------------------------------------------------------
# World -> lum_scene_desc
# --------------------------------------------------------------------------------------
OBJECT_DTYPE = np.dtype([("kind", "<i4"), ("material", "<i4"), ("transform", "<i4"), ("reserved", "<i4"),
                         ("p", "<f8", 12)])
MATERIAL_DTYPE = np.dtype([("kind", "<i4"), ("texture", "<i4"), ("color", "<f8", 3), ("color2", "<f8", 3),
                           ("tex_scale", "<f8"), ("fuzz", "<f8"), ("ior", "<f8"), ("roughness", "<f8"),
                           ("metallic", "<f8"), ("intensity", "<f8"), ("dispersion", "<f8"), ("tint", "<f8", 3),
                           ("sub", "<i4", 2), ("extra", "<f8", 4)])


def material_array(n: int) -> np.ndarray:
    """n zeroed lum_material records (tint (1,1,1), checker scale 1)."""
    m = np.zeros(n, dtype=MATERIAL_DTYPE)
    m["tint"] = 1.0
    m["tex_scale"] = 1.0
    return m


class World:
    """An ordered object list (HittableList) plus NEE lights and camera.

    ``add`` keeps insertion order, which fixes primitive ids: one id per object (six for a
    box), then mesh triangles in mesh order.  ``add_bulk`` appends many untransformed objects
    at once from structured arrays laid out as lum_object / lum_material.
    """

    def __init__(self):
        self.objects: List[Prim] = []
        self.meshes: List[Mesh] = []
        self.lights: List[LightInfo] = []
        self.materials: List[Material] = []
        self._mat_index = {}
        self._bulk = []          # (insert position in objects, object array, material array)
        self.light_materials: List[Optional[Material]] = []
        self.env_map: Optional[np.ndarray] = None      # (H, W, 3) float32 map of BG_ENVMAP
        self.camera = CameraConfig()

    def add_bulk(self, objects: np.ndarray, materials: np.ndarray) -> int:
        """Appends objects (OBJECT_DTYPE, material = index into `materials`, transform -1)."""
        first = self.n_prims()
        self._bulk.append((len(self.objects), np.ascontiguousarray(objects, dtype=OBJECT_DTYPE),
                           np.ascontiguousarray(materials, dtype=MATERIAL_DTYPE)))
        return first

    def material_index(self, m: Optional[Material]) -> int:
        if m is None:
            return -1
        key = id(m)
        if key not in self._mat_index:
            for c in (m.children or ()):          # Blend children get indices too
                self.material_index(c)
            self._mat_index[key] = len(self.materials)
            self.materials.append(m)
        return self._mat_index[key]

    def add(self, obj: Prim) -> int:
        """Adds an object; returns its first primitive id."""
        first = self.n_prims()
        self.objects.append(obj)
        self.material_index(obj.material)
        return first

    def add_mesh(self, mesh: Mesh) -> int:
        first = self.n_prims()
        self.meshes.append(mesh)
        if mesh.material is not None:
            self.material_index(mesh.material)
        return first

    def add_light(self, light: LightInfo, material: Optional[Material] = None) -> None:
        """Adds an NEE light; `material` is the emissive material whose emission it carries
        (used by the adjoint to route light-emission gradients)."""
        self.lights.append(light)
        self.light_materials.append(material)

    def light_material_indices(self):
        return [self.material_index(m) if m is not None else -1 for m in self.light_materials]

    def n_prims(self) -> int:
        n = sum(6 if o.kind == abi.OBJ_BOX else 1 for o in self.objects)
        n += sum(int(((b["kind"] == abi.OBJ_BOX) * 5 + 1).sum()) for _, b, _ in self._bulk)
        return n + sum(int(m.indices.shape[0]) for m in self.meshes)

    def desc(self) -> "SceneDesc":
        return SceneDesc(self)


_ZEROS = tuple((0.0,) * k for k in range(13))


def _object_array(objs, materials, transforms) -> np.ndarray:
    """The objects as OBJECT_DTYPE records, filled column by column."""
    n = len(objs)
    a = np.zeros(n, dtype=OBJECT_DTYPE)
    if not n:
        return a
    flat = []
    for o in objs:
        p = o.params
        if len(p) > 12:
            p = p[:12]
        flat.extend(p)
        flat.extend(_ZEROS[12 - len(p)])
    a["kind"] = [o.kind for o in objs]
    a["material"] = materials
    a["transform"] = transforms
    a["p"] = np.array(flat, dtype=np.float64).reshape(n, 12)
    return a


def _material_array(mats, index_of) -> np.ndarray:
    """The materials as MATERIAL_DTYPE records: the fields Material.to_c sets, filled column by
    column."""
    n = len(mats)
    a = material_array(n)
    if not n:
        return a
    texture, color, color2, scale = [], [], [], []
    for m in mats:
        t, c, c2, sc = abi.TEX_SOLID, m.color, (0.0, 0.0, 0.0), 1.0
        tex = m.texture
        if isinstance(tex, SolidColor):
            c = tex.color
        elif isinstance(tex, Checker):
            t, c, c2, sc = abi.TEX_CHECKER, tex.even, tex.odd, tex.scale
        if m.color2 is not None:
            c2 = m.color2
        texture.append(t)
        color.extend(c)
        color2.extend(c2)
        scale.append(sc)
    a["kind"] = [m.kind for m in mats]
    a["texture"] = texture
    a["color"] = np.array(color, dtype=np.float64).reshape(n, 3)
    a["color2"] = np.array(color2, dtype=np.float64).reshape(n, 3)
    a["tex_scale"] = scale
    for f in ("fuzz", "ior", "roughness", "metallic", "intensity", "dispersion"):
        a[f] = [getattr(m, f) for m in mats]
    a["tint"] = np.array([x for m in mats for x in m.tint], dtype=np.float64).reshape(n, 3)
    ex = []
    for m in mats:
        e = tuple(m.extra)[:4]
        ex.extend(e)
        ex.extend(_ZEROS[4 - len(e)])
    a["extra"] = np.array(ex, dtype=np.float64).reshape(n, 4)
    for k, m in enumerate(mats):
        if m.children is not None:
            a["sub"][k] = [index_of(c) for c in m.children]
    return a


class SceneDesc:
    """Owns the arrays behind one lum_scene_desc.  Objects and materials are built as numpy
    records laid out as lum_object / lum_material (one row per object or material) and handed
    to the C ABI in place."""

    def __init__(self, world: World):
        xforms = []
        for o in world.objects:
            world.material_index(o.material)
        mat_of, tr_of = [], []
        for o in world.objects:
            tr = -1
            if o.xforms:
                if len(o.xforms) > abi.MAX_XF_OPS:
                    raise ValueError("too many transform ops")
                t = abi.LumTransform()
                t.n_ops = len(o.xforms)
                for i, (op, arg) in enumerate(o.xforms):
                    t.op[i] = op
                    t.arg[i][:] = list(map(float, arg))
                tr = len(xforms)
                xforms.append(t)
            mat_of.append(world.material_index(o.material))
            tr_of.append(tr)
        obj_np = _object_array(world.objects, mat_of, tr_of)
        n_mat_regular = len(world.materials)
        if world._bulk:
            # interleave the bulk chunks at their insertion positions; their material indices
            # follow the regular materials
            parts, mats_np, last, mat_base = [], [], 0, n_mat_regular
            for pos, bobj, bmat in world._bulk:
                parts.append(obj_np[last:pos])
                chunk = bobj.copy()
                chunk["material"] += mat_base
                chunk["transform"] = -1
                parts.append(chunk)
                mats_np.append(bmat)
                mat_base += len(bmat)
                last = pos
            parts.append(obj_np[last:])
            obj_np = np.concatenate(parts)
            self._bulk_mats = np.concatenate(mats_np)
        else:
            self._bulk_mats = None
        n_objects = len(obj_np)
        self._obj_np = np.ascontiguousarray(obj_np if n_objects else np.zeros(1, dtype=OBJECT_DTYPE))
        self._objects = (abi.LumObject * len(self._obj_np)).from_buffer(self._obj_np)
        self._xforms = (abi.LumTransform * max(len(xforms), 1))(*xforms)
        self._keep = []
        meshes = []
        for m in world.meshes:
            pos = np.ascontiguousarray(m.positions, dtype=np.float64)
            idx = np.ascontiguousarray(m.indices, dtype=np.uint32)
            lm = abi.LumMesh()
            lm.positions = pos.ctypes.data_as(C.POINTER(C.c_double))
            lm.n_vertices = pos.shape[0]
            lm.indices = idx.ctypes.data_as(C.POINTER(C.c_uint32))
            lm.n_triangles = idx.shape[0]
            self._keep += [pos, idx]
            if m.normals is not None:
                nrm = np.ascontiguousarray(m.normals, dtype=np.float64)
                lm.normals = nrm.ctypes.data_as(C.POINTER(C.c_double))
                self._keep.append(nrm)
            if m.tri_material is not None:
                tm = np.ascontiguousarray(m.tri_material, dtype=np.int32)
                lm.tri_material = tm.ctypes.data_as(C.POINTER(C.c_int32))
                self._keep.append(tm)
            lm.material = world.material_index(m.material)
            meshes.append(lm)
        self._meshes = (abi.LumMesh * max(len(meshes), 1))(*meshes)
        mat_np = _material_array(world.materials, world.material_index)
        if self._bulk_mats is not None:
            mat_np = np.concatenate([mat_np, self._bulk_mats])
        n_materials = len(mat_np)
        self._mat_np = np.ascontiguousarray(mat_np if n_materials else np.zeros(1, dtype=MATERIAL_DTYPE))
        self._materials = (abi.LumMaterial * len(self._mat_np)).from_buffer(self._mat_np)
        lights = [l.to_c() for l in world.lights]
        self._lights = (abi.LumLight * max(len(lights), 1))(*lights)
        d = abi.LumSceneDesc()
        d.objects = self._objects
        d.n_objects = n_objects
        d.meshes = self._meshes
        d.n_meshes = len(meshes)
        d.materials = self._materials
        d.n_materials = n_materials
        d.transforms = self._xforms
        d.n_transforms = len(xforms)
        d.lights = self._lights
        d.n_lights = len(lights)
        d.camera = world.camera.to_c()
        self.c = d
        self.n_prims = world.n_prims()
        self.n_materials = n_materials

    def ref(self):
        return C.byref(self.c)
