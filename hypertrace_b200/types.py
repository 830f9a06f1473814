"""Scene types: a Python mirror of the reference's entity types, for any scene.

The reference describes a scene by a Rust type (objects/src/*, types/src/*) whose derive
macros give every entity a byte layout and an OpenCL source template. This module mirrors
those types one for one. Each entity type knows

  - ``cxx()``: its C++ type expression over the templates of
    hypertrace_b200/csrc/ht_generic.cuh (what ``htc_program_build`` compiles with NVRTC),
  - ``lay(W)``: its serialized (size, alignment) for a usize of W bytes (and f64 fields of
    ``f64_bytes(W)`` bytes: 8 when the scene is written with double_support, else 4), by the rules of
    type-macros/src/entity.rs:7-200 (fields in order, each at a multiple of its alignment;
    alignment = lcm of the fields'; size rounded up to it; an enum is a usize index with the
    payload at the enum's alignment; a Vec is a usize count with the elements at their
    alignment, types/src/containers/vector.rs:19-57),
  - ``write(buf, off, value, W)``: the bytes ``EntityBuffer::new`` uploads
    (processing/src/buffer.rs:14-29; f64 fields as f32 when double_support is off, as f64
    when it is on, types/src/primitive/scalar.rs:175-215; 3-vectors padded to 4 components,
    types/src/primitive/vector.rs:74-106; a primitive vector or matrix is aligned to its own
    size, types/src/primitive/matrix.rs:171-209). Colors and the gradient power are f32 in
    the reference and stay 4 bytes either way.

Values are plain Python data: floats, 3-/4-sequences, 2x2 complex arrays (Moebius),
``(outer, inner)`` tuples (Chain), dicts keyed by field name (structs), ``(variant index,
value)`` tuples (enums) and lists (Vec). ``serialize(scene_type, value, address_width)``
returns the scene bytes; ``hy_tiled_type`` and ``eu_gradient_type`` are the types of the
reference's ``hy`` and ``eu`` examples (main/examples/hy.rs, main/examples/eu.rs), which the
library also serves as built-in recipes (HTC_RECIPE_HY_TILED, HTC_RECIPE_EU_GRADIENT).
"""
from __future__ import annotations

import math
import struct
from typing import List, Sequence, Tuple

import numpy as np


def upm(x: int, a: int) -> int:
    return (x + a - 1) // a * a


def lcm(a: int, b: int) -> int:
    return a // math.gcd(a, b) * b


def _usize_bytes(x: int, W: int) -> bytes:
    return struct.pack("<I" if W == 4 else "<Q", int(x))


class Cfg(int):
    """The layout parameter every entity method takes: an int (the usize size in bytes, 4 or
    8) that also carries the size of an f64 field (4, or 8 with double_support)."""

    def __new__(cls, usize: int, f64: int = 4):
        obj = super().__new__(cls, usize)
        obj.f64 = f64
        return obj


def f64_bytes(W) -> int:
    """Bytes of an f64 field under layout parameter W (a plain int means double_support off)."""
    return getattr(W, "f64", 4)


def _pack_reals(buf, off, W, values) -> None:
    struct.pack_into("<%d%s" % (len(values), "d" if f64_bytes(W) == 8 else "f"), buf, off, *[float(v) for v in values])


class Entity:
    """An entity type."""
    dynamic = False

    def cxx(self) -> str:
        raise NotImplementedError

    def lay(self, W: int) -> Tuple[int, int]:
        raise NotImplementedError

    def size_of(self, value, W: int) -> int:
        return self.lay(W)[0]

    def write(self, buf: bytearray, off: int, value, W: int) -> None:
        raise NotImplementedError

    def __repr__(self) -> str:
        return self.cxx()


# ----------------------------------------------------------------------------- primitives

class Unit(Entity):
    """A zero-sized entity: unit structs (shapes, Lambertian, ...) and PhantomData."""

    def __init__(self, name: str = "Zst"):
        self.name = name

    def cxx(self):
        return self.name

    def lay(self, W):
        return (0, 1)

    def write(self, buf, off, value, W):
        pass


class F32(Entity):
    """An f32 field (the gradient background's power)."""

    def cxx(self):
        return "F32"

    def lay(self, W):
        return (4, 4)

    def write(self, buf, off, value, W):
        struct.pack_into("<f", buf, off, float(value))


class F64(Entity):
    """An f64 field (fov, portions, refractive index, tiling sizes): 4 bytes as f32, or 8."""

    def cxx(self):
        return "F32"

    def lay(self, W):
        f = f64_bytes(W)
        return (f, f)

    def write(self, buf, off, value, W):
        _pack_reals(buf, off, W, [value])


class Vec3(Entity):
    """Vector<f32, 3> (colors): 16 bytes, aligned to 16."""

    def cxx(self):
        return "R3"

    def lay(self, W):
        return (16, 16)

    def write(self, buf, off, value, W):
        v = [float(x) for x in value]
        struct.pack_into("<fff", buf, off, v[0], v[1], v[2])


class Vec3F64(Entity):
    """Vector<f64, 3> (directions, shifts): 4 reals, aligned to their size."""

    def cxx(self):
        return "R3"

    def lay(self, W):
        f = f64_bytes(W)
        return (4 * f, 4 * f)

    def write(self, buf, off, value, W):
        _pack_reals(buf, off, W, [float(x) for x in value][:3])


class Quat(Entity):
    """Quaternion<f64> (rotations): 4 reals, aligned to their size."""

    def cxx(self):
        return "Quat"

    def lay(self, W):
        f = f64_bytes(W)
        return (4 * f, 4 * f)

    def write(self, buf, off, value, W):
        _pack_reals(buf, off, W, [float(x) for x in value])


class Array(Entity):
    """[T; N] (types/src/containers/array.rs)."""

    def __init__(self, elem: Entity, n: int):
        self.elem, self.n = elem, n

    def cxx(self):
        raise TypeError("arrays appear only as fields")

    def lay(self, W):
        s, a = self.elem.lay(W)
        return (s * self.n, a)

    def write(self, buf, off, value, W):
        if len(value) != self.n:
            raise ValueError(f"array of {self.n} elements expected, got {len(value)}")
        s = self.elem.lay(W)[0]
        for i, v in enumerate(value):
            self.elem.write(buf, off + i * s, v, W)


class Struct(Entity):
    """A struct of named fields (derive(Entity) on a struct)."""

    def __init__(self, cxx: str, fields: Sequence[Tuple[str, Entity]]):
        self._cxx = cxx
        self.fields = list(fields)
        self.dynamic = bool(self.fields) and self.fields[-1][1].dynamic

    def cxx(self):
        return self._cxx

    def align(self, W):
        a = 1
        for _, f in self.fields:
            a = lcm(a, f.lay(W)[1])
        return a

    def offsets(self, W) -> List[int]:
        o, out = 0, []
        for _, f in self.fields:
            s, a = f.lay(W)
            o = upm(o, a)
            out.append(o)
            o += s
        return out

    def lay(self, W):
        o = 0
        for _, f in self.fields:
            s, a = f.lay(W)
            o = upm(o, a) + s
        al = self.align(W)
        return (upm(o, al), al)

    def size_of(self, value, W):
        if not self.dynamic:
            return self.lay(W)[0]
        offs = self.offsets(W)
        name, last = self.fields[-1]
        return upm(offs[-1] + last.size_of(self._field(value, name), W), self.align(W))

    @staticmethod
    def _field(value, name):
        if isinstance(value, dict):
            return value.get(name)
        return getattr(value, name)

    def write(self, buf, off, value, W):
        for (name, f), o in zip(self.fields, self.offsets(W)):
            f.write(buf, off + o, self._field(value, name), W)


class Enum(Entity):
    """An enum of single-field variants: usize index, then the payload at the enum's
    alignment (type-macros/src/entity.rs:14-27,160-181,319-344)."""

    def __init__(self, cxx: str, variants: Sequence[Tuple[str, Entity]]):
        self._cxx = cxx
        self.variants = list(variants)

    def cxx(self):
        return self._cxx

    def align(self, W):
        a = W
        for _, v in self.variants:
            a = lcm(a, v.lay(W)[1])
        return a

    def lay(self, W):
        s = 0
        for _, v in self.variants:
            vs, va = v.lay(W)
            s = max(s, upm(W, va) + vs)
        al = self.align(W)
        return (upm(s, al), al)

    def index(self, key) -> int:
        if isinstance(key, int):
            return key
        return [n for n, _ in self.variants].index(key)

    def write(self, buf, off, value, W):
        key, inner = value
        i = self.index(key)
        buf[off:off + W] = _usize_bytes(i, W)
        self.variants[i][1].write(buf, off + upm(W, self.align(W)), inner, W)


class Vector(Entity):
    """Vec<T> (types/src/containers/vector.rs:19-57): usize count, elements at T's
    alignment and static size."""
    dynamic = True

    def __init__(self, cxx_prefix: str, geo: str, elem: Entity):
        self.prefix, self.geo, self.elem = cxx_prefix, geo, elem

    def cxx(self):
        return f"{self.prefix}<{self.geo}, {self.elem.cxx()}>"

    def lay(self, W):
        ea = self.elem.lay(W)[1]
        return (upm(W, ea), lcm(W, ea))

    def size_of(self, value, W):
        es = self.elem.lay(W)[0]
        head, al = self.lay(W)
        return upm(head + len(value) * es, al)

    def write(self, buf, off, value, W):
        buf[off:off + W] = _usize_bytes(len(value), W)
        head = self.lay(W)[0]
        es = self.elem.lay(W)[0]
        for i, v in enumerate(value):
            self.elem.write(buf, off + head + i * es, v, W)


# ----------------------------------------------------------------------------- maps

class Moebius(Entity):
    """Moebius<Complex<f64>> as comp2x2 (types/src/primitive/matrix.rs:171-209); value: a 2x2
    complex array [[a, b], [c, d]]."""
    geo = "Hy"

    def cxx(self):
        return "Moebius"

    def lay(self, W):
        f = f64_bytes(W)
        return (8 * f, 8 * f)

    def write(self, buf, off, value, W):
        m = np.asarray(value, dtype=np.complex128)
        vals = [m[0, 0], m[0, 1], m[1, 0], m[1, 1]]
        _pack_reals(buf, off, W, [float(x) for z in vals for x in (z.real, z.imag)])


class Shift3(Entity):
    geo = "Eu"

    def cxx(self):
        return "Shift3"

    def lay(self, W):
        return Vec3F64().lay(W)

    def write(self, buf, off, value, W):
        Vec3F64().write(buf, off, value, W)


class Rotation3(Entity):
    """Rotation3 as a quaternion (real, i, j, k)."""
    geo = "Eu"

    def cxx(self):
        return "Rotation3"

    def lay(self, W):
        return Quat().lay(W)

    def write(self, buf, off, value, W):
        Quat().write(buf, off, value, W)


class Linear3(Entity):
    """Linear<f64, 3> as real3x3 = 16 floats, rows padded with 0 and a last row (0, 0, 0, 1)
    (types/src/primitive/matrix.rs:117-165); value: a 3x3 array."""
    geo = "Eu"

    def cxx(self):
        return "Linear3"

    def lay(self, W):
        f = f64_bytes(W)
        return (16 * f, 16 * f)

    def write(self, buf, off, value, W):
        m = np.asarray(value, dtype=np.float64).reshape(3, 3)
        vals = [float(m[i, j]) for i in range(3) for j in range(3)]
        flat = vals[0:3] + [0.0] + vals[3:6] + [0.0] + vals[6:9] + [0.0] + [0.0, 0.0, 0.0, 1.0]
        _pack_reals(buf, off, W, flat)


class Chain(Entity):
    """Chain<A, B>: outer A after inner B (types/src/map.rs:172-235); value: (a, b)."""
    geo = "Eu"

    def __init__(self, outer: Entity, inner: Entity, name: str = ""):
        self.outer, self.inner, self.name = outer, inner, name

    def cxx(self):
        return self.name or f"Chain<{self.outer.cxx()}, {self.inner.cxx()}>"

    def lay(self, W):
        (sa, aa), (sb, ab) = self.outer.lay(W), self.inner.lay(W)
        al = lcm(aa, ab)
        return (upm(upm(sa, ab) + sb, al), al)

    def write(self, buf, off, value, W):
        a, b = value
        self.outer.write(buf, off, a, W)
        self.inner.write(buf, off + upm(self.outer.lay(W)[0], self.inner.lay(W)[1]), b, W)


def Homogenous3() -> Chain:
    """Chain<Shift3, Rotation3>; value: (shift xyz, rotation quaternion)."""
    return Chain(Shift3(), Rotation3(), "Homogenous3")


# ----------------------------------------------------------------------------- views

def PointView(geo: str) -> Struct:
    """PointView<G>{fov, phantom} (objects/src/view/point.rs:11-14); value: {"fov": f}."""
    return Struct(f"PointView<{geo}>", [("fov", F64()), ("phantom", Unit())])


def MappedView(geo: str, view: Entity, map_: Entity) -> Struct:
    """Mapped<G, V, M>{geometry, map, inner} (objects/src/mapped.rs:5-11)."""
    return Struct(f"MappedView<{geo}, {view.cxx()}, {map_.cxx()}>",
                  [("geometry", Unit()), ("map", map_), ("inner", view)])


# ----------------------------------------------------------------------------- shapes

def PlaneHy() -> Unit:
    return Unit("PlaneHy")


def Horosphere() -> Unit:
    return Unit("Horosphere")


def PlaneEu() -> Unit:
    return Unit("PlaneEu")


def Sphere() -> Unit:
    return Unit("Sphere")


def Cube() -> Unit:
    return Unit("Cube")


def ShapeVec(geo: str, shape: Entity) -> Vector:
    return Vector("ShapeVec", geo, shape)


def MappedShape(geo: str, shape: Entity, map_: Entity) -> Struct:
    return Struct(f"MappedShape<{geo}, {shape.cxx()}, {map_.cxx()}>",
                  [("geometry", Unit()), ("map", map_), ("inner", shape)])


def ShapeChoice(geo: str, *variants: Tuple[str, Entity]) -> Enum:
    """shape_choice! (objects/src/shape/choice.rs); variants: (name, shape) pairs."""
    return Enum(f"ShapeChoice<{geo}, {', '.join(v.cxx() for _, v in variants)}>", variants)


# ----------------------------------------------------------------------------- materials

def Lambertian() -> Unit:
    return Unit("Lambertian")


def Specular() -> Unit:
    return Unit("Specular")


def Absorbing() -> Unit:
    return Unit("Absorbing")


def Transparent() -> Unit:
    return Unit("Transparent")


def Refractive() -> Struct:
    """{index} (objects/src/material/refractive.rs)."""
    return Struct("Refractive", [("index", F64())])


def Colored(inner: Entity) -> Struct:
    """{color, inner} (objects/src/material/modifier.rs:13-18)."""
    return Struct(f"Colored<{inner.cxx()}>", [("color", Vec3()), ("inner", inner)])


def Emissive(inner: Entity) -> Struct:
    """{emission, inner} (objects/src/material/modifier.rs:46-51)."""
    return Struct(f"Emissive<{inner.cxx()}>", [("emission", Vec3()), ("inner", inner)])


def Component(material: Entity) -> Struct:
    """{material, portion} (objects/src/material/mixture.rs:4-9)."""
    return Struct(f"Component<{material.cxx()}>", [("material", material), ("portion", F64())])


def Mixture(*components: Tuple[str, Entity]) -> Struct:
    """mixture! (objects/src/material/mixture.rs:27-60); components: (name, material)."""
    comps = [(n, Component(m)) for n, m in components]
    return Struct(f"Mixture<{', '.join(c.cxx() for _, c in comps)}>", comps)


# ----------------------------------------------------------------------------- objects

def Covered(geo: str, shape: Entity, material: Entity) -> Struct:
    """Covered<G, S, M>{geometry, material, shape} (objects/src/object/covered.rs:12-18)."""
    return Struct(f"Covered<{geo}, {shape.cxx()}, {material.cxx()}>",
                  [("geometry", Unit()), ("material", material), ("shape", shape)])


def MappedObject(geo: str, obj: Entity, map_: Entity) -> Struct:
    return Struct(f"MappedObject<{geo}, {obj.cxx()}, {map_.cxx()}>",
                  [("geometry", Unit()), ("map", map_), ("inner", obj)])


def ObjectVec(geo: str, obj: Entity) -> Vector:
    return Vector("ObjectVec", geo, obj)


def ObjectChoice(geo: str, *variants: Tuple[str, Entity]) -> Enum:
    """object_choice! (objects/src/object/choice.rs)."""
    return Enum(f"ObjectChoice<{geo}, {', '.join(v.cxx() for _, v in variants)}>", variants)


_PLANE_TILINGS = {"Uniform": "PlaneUniform", "Pentagonal": "PlanePentagonal", "Pentastar": "PlanePentastar"}
_HORO_TILINGS = {"Uniform": "HoroUniform", "Square": "HoroSquare", "Hexagonal": "HoroHexagonal"}


def _tiled(kind: str, material: Entity, tiling: str, n: int) -> Struct:
    return Struct(f"{kind}<{material.cxx()}, {tiling}, {n}>",
                  [("tiling", Unit()), ("materials", Array(material, n)), ("border_material", material),
                   ("cell_size", F64()), ("border_width", F64())])


def TiledPlane(material: Entity, tiling: str, n: int) -> Struct:
    """TiledPlane<M, K, N> (objects/src/object/tiled_plane.rs:35-42); tiling one of
    Uniform, Pentagonal, Pentastar."""
    return _tiled("TiledPlane", material, _PLANE_TILINGS[tiling], n)


def TiledHorosphere(material: Entity, tiling: str, n: int) -> Struct:
    """TiledHorosphere<M, K, N> (objects/src/object/tiled_horosphere.rs:35-42); tiling one
    of Uniform, Square, Hexagonal."""
    return _tiled("TiledHorosphere", material, _HORO_TILINGS[tiling], n)


# ----------------------------------------------------------------------------- backgrounds

def ConstBg() -> Struct:
    return Struct("ConstBg", [("color", Vec3())])


def GradBg() -> Struct:
    """{direction, colors[2], power} (objects/src/background/basic.rs:54-58)."""
    return Struct("GradBg", [("direction", Vec3F64()), ("colors", Array(Vec3(), 2)), ("power", F32())])


# ----------------------------------------------------------------------------- scene

def SceneImpl(geo: str, view: Entity, obj: Entity, background: Entity) -> Struct:
    """SceneImpl<G, V, T, B, H>{geometry, view, background, object} (objects/src/scene.rs:19-28);
    H is the program's light-hop count."""
    return Struct(f"SceneImpl<{geo}, {view.cxx()}, {obj.cxx()}, {background.cxx()}>",
                  [("geometry", Unit()), ("view", view), ("background", background), ("object", obj)])


def layout(address_width: int = 32, double_support: bool = False) -> Cfg:
    """The layout parameter of a types::Config (types/src/config.rs:38-43)."""
    if address_width not in (32, 64):
        raise ValueError("address_width must be 32 or 64")
    return Cfg(4 if address_width == 32 else 8, 8 if double_support else 4)


def serialize(scene_type: Entity, value, address_width: int = 32, double_support: bool = False) -> bytes:
    W = layout(address_width, double_support)
    buf = bytearray(scene_type.size_of(value, W))
    scene_type.write(buf, 0, value, W)
    return bytes(buf)


def static_size(scene_type: Entity, address_width: int = 32, double_support: bool = False) -> int:
    """Bytes of the scene without its dynamic part (htc_program_static_size)."""
    W = layout(address_width, double_support)
    if isinstance(scene_type, Struct) and scene_type.dynamic:
        offs = scene_type.offsets(W)
        return offs[-1] + scene_type.fields[-1][1].lay(W)[0]
    return scene_type.lay(W)[0]


# ----------------------------------------------------------------------------- named types

def hearth_material() -> Struct:
    """Mixture{diffuse: Colored<Lambertian>, specular: Specular, luminous: Emissive<Absorbing>}
    (main/examples/hearth.rs:19-25)."""
    return Mixture(("diffuse", Colored(Lambertian())), ("specular", Specular()),
                   ("luminous", Emissive(Absorbing())))


def hearth_type() -> Struct:
    """The hyperbolic recipe HTC_RECIPE_HY as a generic scene type."""
    obj = MappedObject("Hy", Covered("Hy", ShapeChoice("Hy", ("Plane", PlaneHy()), ("Horosphere", Horosphere())),
                                     hearth_material()), Moebius())
    return SceneImpl("Hy", MappedView("Hy", PointView("Hy"), Moebius()), ObjectVec("Hy", obj), ConstBg())


def euclid_type() -> Struct:
    """The Euclidean recipe HTC_RECIPE_EU as a generic scene type."""
    obj = MappedObject("Eu", Covered("Eu", ShapeChoice("Eu", ("Plane", PlaneEu()), ("Sphere", Sphere())),
                                     hearth_material()), Homogenous3())
    return SceneImpl("Eu", MappedView("Eu", PointView("Eu"), Homogenous3()), ObjectVec("Eu", obj), ConstBg())


def hy_tiled_material() -> Struct:
    """Emissive<Mixture{diffuse: Colored<Lambertian>, specular: Specular, transparent:
    Transparent}> (main/examples/hy.rs:35-62)."""
    return Emissive(Mixture(("diffuse", Colored(Lambertian())), ("specular", Specular()),
                            ("transparent", Transparent())))


def hy_tiled_type() -> Struct:
    """The scene type of main/examples/hy.rs (HTC_RECIPE_HY_TILED)."""
    m = hy_tiled_material()
    choice = ObjectChoice("Hy", ("PlaneStar", TiledPlane(m, "Pentastar", 2)),
                          ("PlanePenta", TiledPlane(m, "Pentagonal", 2)),
                          ("HoroHexa", TiledHorosphere(m, "Hexagonal", 3)),
                          ("HoroSquare", TiledHorosphere(m, "Square", 4)))
    return SceneImpl("Hy", MappedView("Hy", PointView("Hy"), Moebius()),
                     ObjectVec("Hy", MappedObject("Hy", choice, Moebius())), ConstBg())


def eu_gradient_material() -> Struct:
    """Mixture{diffuse: Colored<Lambertian>, specular: Specular, refractive:
    Colored<Refractive>} (main/examples/eu.rs:38-44)."""
    return Mixture(("diffuse", Colored(Lambertian())), ("specular", Specular()),
                   ("refractive", Colored(Refractive())))


def eu_gradient_type() -> Struct:
    """The scene type of main/examples/eu.rs (HTC_RECIPE_EU_GRADIENT)."""
    shape = ShapeChoice("Eu", ("Plane", PlaneEu()), ("Sphere", Sphere()), ("Cube", Cube()))
    obj = MappedObject("Eu", Covered("Eu", shape, eu_gradient_material()), Shift3())
    return SceneImpl("Eu", MappedView("Eu", PointView("Eu"), Homogenous3()), ObjectVec("Eu", obj), GradBg())


# ----------------------------------------------------------------------------- values

def _map_value(m):
    """scene.Hom3 -> (shift, rotation); a Moebius array passes through."""
    if hasattr(m, "shift"):
        return (np.asarray(m.shift, dtype=np.float64), np.asarray(m.rot, dtype=np.float64))
    return np.asarray(m)


def hearth_value(scene) -> dict:
    """Value of hearth_type() / euclid_type() for a scene.Scene of recipe HTC_RECIPE_HY / EU
    (the same bytes as scene.serialize)."""
    def mat(m):
        return {"diffuse": {"material": {"color": m.diffuse_color, "inner": None}, "portion": m.diffuse},
                "specular": {"material": None, "portion": m.specular},
                "luminous": {"material": {"emission": m.emission, "inner": None}, "portion": m.luminous}}
    objs = [{"map": _map_value(o.map), "inner": {"material": mat(o.material), "shape": (int(o.shape), None)}}
            for o in scene.objects]
    return {"view": {"map": _map_value(scene.camera), "inner": {"fov": scene.fov}},
            "background": {"color": scene.background}, "object": objs}


# ----------------------------------------------------------------------------- example scenes

def _unpack_color(rgb: int) -> np.ndarray:
    """unpack_color + make_color of main/examples/hy.rs:27-33 (sRGB byte -> linear, power 2.2)."""
    v = np.array([(rgb >> 16) & 0xFF, (rgb >> 8) & 0xFF, rgb & 0xFF], dtype=np.float32) / np.float32(255.0)
    return np.power(v, np.float32(2.2)).astype(np.float32)


def _hy_material(diffuse, specularity: float, transparency: float, emission=None) -> dict:
    """make_material of main/examples/hy.rs:43-62."""
    return {"emission": (0.0, 0.0, 0.0) if emission is None else emission,
            "inner": {"diffuse": {"material": {"color": diffuse, "inner": None},
                                  "portion": 1.0 - specularity - transparency},
                      "specular": {"material": None, "portion": specularity},
                      "transparent": {"material": None, "portion": transparency}}}


def hy_example_camera() -> np.ndarray:
    """The controller's initial map in main/examples/hy.rs:143-148:
    rotate_z(5 pi / 6) . rotate_x(2 pi / 5) . shift_z(2)."""
    from . import scene as S
    return S.mo_chain(S.mo_chain(S.mo_zrotate(5 * np.pi / 6), S.mo_xrotate(2 * np.pi / 5)), S.mo_zshift(2.0))


def hy_example_value(camera=None, fov: float = 1.0) -> dict:
    """The scene of main/examples/hy.rs:103-139 (value of hy_tiled_type())."""
    from . import scene as S
    border = _hy_material(_unpack_color(0xE4E4E4), 0.0, 0.0, np.ones(3, dtype=np.float32))
    m = lambda rgb, s, t: _hy_material(_unpack_color(rgb), s, t)
    ident = S.mo_identity()
    shift2 = np.array([[1.0, np.sqrt(2.0)], [0.0, 1.0]], dtype=np.complex128)
    objs = [
        {"map": ident, "inner": ("HoroHexa", {"materials": [m(0xFE0000, .1, .1), m(0xFFAA01, .1, .1), m(0x35ADAE, .1, .1)],
                                              "border_material": border, "cell_size": 0.5, "border_width": 0.02})},
        {"map": S.mo_chain(shift2, S.mo_xrotate(np.pi)),
         "inner": ("HoroSquare", {"materials": [m(0xFE7401, .1, .1), m(0xFE0000, .1, .1), m(0xFFAA01, .1, .1),
                                                m(0xFED601, .1, .1)],
                                  "border_material": border, "cell_size": 0.5, "border_width": 0.02})},
        {"map": ident, "inner": ("PlaneStar", {"materials": [m(0xFE7401, .1, 0.0), m(0x35ADAE, .1, 0.0)],
                                               "border_material": border, "cell_size": float("nan"),
                                               "border_width": 0.01})},
        {"map": np.array([[1.0, 2.0j], [0.0, 1.0]], dtype=np.complex128),
         "inner": ("PlanePenta", {"materials": [m(0xFE0000, .1, 0.0), m(0xFED601, .1, 0.0)],
                                  "border_material": border, "cell_size": float("nan"), "border_width": 0.02})},
    ]
    cam = hy_example_camera() if camera is None else camera
    return {"view": {"map": cam, "inner": {"fov": fov}}, "background": {"color": _unpack_color(0xEEEEEE)},
            "object": objs}


def eu_example_value(camera=None, fov: float = 1.0) -> dict:
    """The scene of main/examples/eu.rs:71-122 (value of eu_gradient_type()); the camera is
    the controller's initial map, a shift by (0, 0.5, 2) (eu.rs:134-140)."""
    def mix(dc, dp, sp, rc, ri, rp):
        return {"diffuse": {"material": {"color": dc, "inner": None}, "portion": dp},
                "specular": {"material": None, "portion": sp},
                "refractive": {"material": {"color": rc, "inner": {"index": ri}}, "portion": rp}}
    objs = [
        {"map": (0.0, 1.0, 0.0), "inner": {"material": mix((1.0, 0.2, 0.2), 0.0, 0.1, (1.0, 1.0, 0.2), 1.2, 0.9),
                                           "shape": ("Sphere", None)}},
        {"map": (0.0, -1.0, 0.0), "inner": {"material": mix((0.2, 0.8, 0.8), 1.0, 0.0, (1.0, 1.0, 1.0), 1.0, 0.0),
                                            "shape": ("Cube", None)}},
        {"map": (0.0, 0.0, -1.0), "inner": {"material": mix((1.0, 1.0, 1.0), 0.9, 0.1, (1.0, 1.0, 1.0), 1.0, 0.0),
                                            "shape": ("Plane", None)}},
    ]
    cam = ((0.0, 0.5, 2.0), (1.0, 0.0, 0.0, 0.0)) if camera is None else camera
    return {"view": {"map": cam, "inner": {"fov": fov}},
            "background": {"direction": (0.0, 1.0, 0.0), "colors": [(1.0, 1.0, 1.0), (0.0, 0.0, 0.0)], "power": 2.4},
            "object": objs}


def hy_tiled_random_value(seed: int, n_objects: int = 8, max_distance: float = 2.0) -> dict:
    """A random scene of hy_tiled_type(): n tiled objects of random variants, random maps
    (translation <= max_distance), random materials and camera."""
    from . import scene as S
    rng = np.random.default_rng(seed)

    def mat(emissive: bool = False):
        s, t = float(rng.uniform(0, 0.4)), float(rng.uniform(0, 0.4))
        em = tuple(rng.uniform(0.5, 3.0, 3)) if emissive else None
        return _hy_material(tuple(rng.uniform(0.1, 0.9, 3)), s, t, em)
    counts = {"PlaneStar": 2, "PlanePenta": 2, "HoroHexa": 3, "HoroSquare": 4}
    names = list(counts)
    objs = []
    for _ in range(n_objects):
        v = names[int(rng.integers(4))]
        body = {"materials": [mat() for _ in range(counts[v])], "border_material": mat(emissive=bool(rng.integers(2))),
                "cell_size": float(rng.uniform(0.2, 1.0)) if v.startswith("Horo") else float("nan"),
                "border_width": float(rng.uniform(0.005, 0.05))}
        objs.append({"map": S.random_moebius(rng, max_distance), "inner": (v, body)})
    return {"view": {"map": S.random_moebius(rng, 1.0), "inner": {"fov": float(rng.uniform(0.6, 1.5))}},
            "background": {"color": tuple(rng.uniform(0.2, 1.0, 3))}, "object": objs}


def eu_gradient_random_value(seed: int, n_objects: int = 8) -> dict:
    """A random scene of eu_gradient_type(): planes, spheres and cubes shifted around the
    origin, random mixtures (refractive indices in [1, 2]), a random camera in front."""
    from . import scene as S
    rng = np.random.default_rng(seed)
    objs = []
    for i in range(n_objects):
        shape = ("Plane", "Sphere", "Cube")[0 if i == 0 else int(rng.integers(1, 3))]
        p = rng.dirichlet([1.0, 1.0, 1.0])
        objs.append({"map": (0.0, 0.0, -1.5) if i == 0 else tuple(rng.uniform(-3, 3, 2)) + (float(rng.uniform(-1, 2)),),
                     "inner": {"material": {
                         "diffuse": {"material": {"color": tuple(rng.uniform(0.1, 0.9, 3)), "inner": None}, "portion": float(p[0])},
                         "specular": {"material": None, "portion": float(p[1])},
                         "refractive": {"material": {"color": tuple(rng.uniform(0.5, 1.0, 3)),
                                                     "inner": {"index": float(rng.uniform(1.0, 2.0))}},
                                        "portion": float(p[2])}},
                         "shape": (shape, None)}})
    q = S.quat_axis_angle([1.0, 0.0, 0.0], float(rng.uniform(-0.3, 0.3)))
    cam = ((float(rng.uniform(-1, 1)), float(rng.uniform(-1, 1)), float(rng.uniform(5, 8))), tuple(q))
    d = rng.normal(size=3)
    return {"view": {"map": cam, "inner": {"fov": float(rng.uniform(0.6, 1.5))}},
            "background": {"direction": tuple(d / np.linalg.norm(d)),
                           "colors": [tuple(rng.uniform(0.5, 1.5, 3)), tuple(rng.uniform(0.0, 0.3, 3))],
                           "power": float(rng.uniform(0.5, 4.0))},
            "object": objs}


def eu_compound_type() -> Struct:
    """A Euclidean scene type that no example builds, for the containers and maps the examples
    leave out: one mapped object (map Chain<Linear3, Shift3>) covered with the eu.rs mixture,
    whose shape is a vector of mapped shapes (maps Chain<Shift3, Linear3>) choosing plane /
    sphere / cube; gradient background."""
    shape = ShapeChoice("Eu", ("Plane", PlaneEu()), ("Sphere", Sphere()), ("Cube", Cube()))
    shapes = ShapeVec("Eu", MappedShape("Eu", shape, Chain(Shift3(), Linear3())))
    obj = MappedObject("Eu", Covered("Eu", shapes, eu_gradient_material()), Chain(Linear3(), Shift3()))
    return SceneImpl("Eu", MappedView("Eu", PointView("Eu"), Homogenous3()), obj, GradBg())


def _random_linear(rng: np.random.Generator, lo: float = 0.5, hi: float = 1.5, max_angle: float = np.pi) -> np.ndarray:
    """Rotation (angle <= max_angle) x shear x scale in [lo, hi]."""
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    a = float(rng.uniform(-max_angle, max_angle))
    k = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    q = np.eye(3) + np.sin(a) * k + (1 - np.cos(a)) * (k @ k)
    shear = np.eye(3) + np.triu(rng.uniform(-0.3, 0.3, (3, 3)), 1)
    return q @ shear @ np.diag(rng.uniform(lo, hi, 3))


def eu_compound_random_value(seed: int, n_shapes: int = 6) -> dict:
    """A random scene of eu_compound_type(): a ground plane and spheres / cubes under random
    linear maps (scale, shear, rotation), one random mixture, a camera in front."""
    from . import scene as S
    rng = np.random.default_rng(seed)
    shapes = [{"map": ((0.0, 0.0, -1.5), np.eye(3)), "inner": ("Plane", None)}]
    for _ in range(n_shapes - 1):
        shapes.append({"map": (tuple(rng.uniform(-2.5, 2.5, 2)) + (float(rng.uniform(-0.5, 1.5)),),
                               _random_linear(rng)),
                       "inner": (("Sphere", "Cube")[int(rng.integers(2))], None)})
    p = rng.dirichlet([1.0, 1.0, 1.0])
    material = {"diffuse": {"material": {"color": tuple(rng.uniform(0.2, 0.9, 3)), "inner": None}, "portion": float(p[0])},
                "specular": {"material": None, "portion": float(p[1])},
                "refractive": {"material": {"color": tuple(rng.uniform(0.5, 1.0, 3)),
                                            "inner": {"index": float(rng.uniform(1.1, 1.8))}},
                               "portion": float(p[2])}}
    obj = {"map": (_random_linear(rng, 0.8, 1.2, 0.3), tuple(rng.uniform(-0.3, 0.3, 3))),
           "inner": {"material": material, "shape": shapes}}
    q = S.quat_axis_angle([1.0, 0.0, 0.0], float(rng.uniform(-0.2, 0.2)))
    cam = ((float(rng.uniform(-0.5, 0.5)), float(rng.uniform(-0.5, 0.5)), float(rng.uniform(6, 8))), tuple(q))
    d = rng.normal(size=3)
    return {"view": {"map": cam, "inner": {"fov": float(rng.uniform(0.7, 1.3))}},
            "background": {"direction": tuple(d / np.linalg.norm(d)),
                           "colors": [tuple(rng.uniform(0.5, 1.5, 3)), tuple(rng.uniform(0.0, 0.3, 3))],
                           "power": float(rng.uniform(0.5, 4.0))},
            "object": obj}
