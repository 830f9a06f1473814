"""Scene description, byte-exact serializer and synthetic workload generators.

The serialized bytes are what the reference's `EntityBuffer::new` uploads
(processing/src/buffer.rs:14-29 -> types/src/io.rs:185-230): every field aligned to its
own alignment, every struct padded to the lcm of its fields' alignments
(type-macros/src/entity.rs:7-186), 3-vectors padded to 4 components
(types/src/primitive/vector.rs:95-106), ``f64`` written as ``f32`` when
``double_support`` is false (types/src/primitive/scalar.rs:198-207), ``usize`` 4 or 8
bytes by address width (scalar.rs:101-165), enums as ``{usize index; union}``
(type-macros/src/source.rs:171-178), ``Vec`` as ``{usize size; T elements[]}``
(types/src/containers/vector.rs:19-57, kernel/ocl/container/vector.inl:8-13).

Two scene recipes are served (the ``hearth`` recipe, main/examples/hearth.rs:27-41, and
its Euclidean counterpart, main/examples/eu.rs:30-44 with ``Homogenous3`` maps):

    SceneImpl<G, Mapped<PointView, Map>,
              Vec<Mapped<Covered<Choice{Plane, Horosphere|Sphere},
                                 Mixture{diffuse: Colored<Lambertian>,
                                         specular: Specular,
                                         luminous: Emissive<Absorbing>}>, Map>>,
              ConstBg, H>

Byte layout (offsets in bytes; identical for address width 32 and 64 because every
``usize`` sits in a slot padded to >= 8):

    hyperbolic scene  : view.map Moebius [0,32) ; view.fov f32 @32 ; background rgb @64 ;
                        objects.size usize @96 ; object[i] @128 + 128*i
    euclidean scene   : view.map Homogenous3 [0,32) ; view.fov @32 ; background rgb @48 ;
                        objects.size @64 ; object[i] @80 + 128*i
    object record     : map [0,32) ; diffuse.color @32 ; diffuse.portion @48 ;
                        specular.portion @64 ; luminous.emission @80 ;
                        luminous.portion @96 ; shape.index @112 ; (record = 128 bytes)
    Moebius           : a, b, c, d complex (re, im) f32, row-major (types/src/primitive/matrix.rs:247-262)
    Homogenous3       : shift xyz (+pad) [0,16) ; rotation quaternion (real, i, j, k) [16,32)
"""
from __future__ import annotations

import dataclasses
import struct
from typing import List, Optional, Sequence

import numpy as np

RECIPE_HY = 1
RECIPE_EU = 2

SHAPE_PLANE = 0
SHAPE_HOROSPHERE = 1  # hyperbolic recipe
SHAPE_SPHERE = 1      # euclidean recipe

OBJ_STRIDE = 128
HY_OBJECTS_OFFSET = 128
EU_OBJECTS_OFFSET = 80


# ----------------------------------------------------------------------------- maps (f64)
# Host-side map composition is FP64, like the reference host (vecmat/ccgeom in f64,
# narrowed to f32 at serialization: types/src/primitive/scalar.rs:198-207).

def mo_identity() -> np.ndarray:
    return np.array([[1, 0], [0, 1]], dtype=np.complex128)


def mo_chain(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Composition a∘b (kernel/ocl/transform/moebius.cc:58-60: c22_dot)."""
    return a @ b


def mo_normalize(m: np.ndarray) -> np.ndarray:
    """Scale to det = 1 (kernel/ocl/algebra/matrix_complex.cc:50-52)."""
    det = m[0, 0] * m[1, 1] - m[0, 1] * m[1, 0]
    return m / np.sqrt(det)


def mo_zshift(l: float) -> np.ndarray:
    """Translation along the j axis (kernel/ocl/geometry/hyperbolic.cc:35-39)."""
    e = np.exp(l / 2)
    return np.array([[e, 0], [0, 1 / e]], dtype=np.complex128)


def mo_xshift(l: float) -> np.ndarray:
    """kernel/ocl/geometry/hyperbolic.cc:40-44"""
    c, s = np.cosh(l / 2), np.sinh(l / 2)
    return np.array([[c, s], [s, c]], dtype=np.complex128)


def mo_yshift(l: float) -> np.ndarray:
    """kernel/ocl/geometry/hyperbolic.cc:45-49"""
    c, s = np.cosh(l / 2), np.sinh(l / 2)
    return np.array([[c, 1j * s], [-1j * s, c]], dtype=np.complex128)


def mo_zrotate(phi: float) -> np.ndarray:
    """kernel/ocl/geometry/hyperbolic.cc:51-54"""
    c, s = np.cos(phi / 2), np.sin(phi / 2)
    return np.array([[c + 1j * s, 0], [0, c - 1j * s]], dtype=np.complex128)


def mo_xrotate(theta: float) -> np.ndarray:
    """kernel/ocl/geometry/hyperbolic.cc:55-58"""
    c, s = np.cos(theta / 2), np.sin(theta / 2)
    return np.array([[c, 1j * s], [1j * s, c]], dtype=np.complex128)


def mo_yrotate(theta: float) -> np.ndarray:
    """kernel/ocl/geometry/hyperbolic.cc:59-62"""
    c, s = np.cos(theta / 2), np.sin(theta / 2)
    return np.array([[c, -s], [s, c]], dtype=np.complex128)


def _qmul(a, b):
    return np.array([
        a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3],
        a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
        a[0] * b[2] + a[2] * b[0] - a[1] * b[3] + a[3] * b[1],
        a[0] * b[3] + a[3] * b[0] + a[1] * b[2] - a[2] * b[1],
    ])


def mo_apply(m: np.ndarray, p) -> np.ndarray:
    """(a p + b)(c p + d)^-1 on a quaternion point (kernel/ocl/transform/moebius.cc:20-25), f64."""
    p = np.asarray(p, dtype=np.float64)

    def cq(c, q):
        return np.array([c.real * q[0] - c.imag * q[1], c.real * q[1] + c.imag * q[0],
                         c.real * q[2] - c.imag * q[3], c.real * q[3] + c.imag * q[2]])
    a, b, c, d = m[0, 0], m[0, 1], m[1, 0], m[1, 1]
    num = cq(a, p) + np.array([b.real, b.imag, 0, 0])
    den = cq(c, p) + np.array([d.real, d.imag, 0, 0])
    inv = np.array([den[0], -den[1], -den[2], -den[3]]) / np.dot(den, den)
    return _qmul(num, inv)


def hy_distance(a, b) -> float:
    """kernel/ocl/geometry/hyperbolic.cc:20-23, f64."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    x = 1 + np.dot(a - b, a - b) / (2 * a[2] * b[2])
    return float(np.log(x + np.sqrt(max(x * x - 1, 0.0))))


J = np.array([0.0, 0.0, 1.0, 0.0])


def quat_axis_angle(axis, angle: float) -> np.ndarray:
    """Rotation3 quaternion (real, i, j, k) (kernel/ocl/transform/rotation.cc rot3_from_axis)."""
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.linalg.norm(axis)
    return np.concatenate([[np.cos(angle / 2)], np.sin(angle / 2) * axis])


@dataclasses.dataclass
class Hom3:
    """Homogenous3 = Chain<Shift3, Rotation3>: p -> R p + shift (transform/chain.inl:36-39)."""
    shift: np.ndarray
    rot: np.ndarray  # quaternion (real, i, j, k)

    @staticmethod
    def identity() -> "Hom3":
        return Hom3(np.zeros(3), np.array([1.0, 0.0, 0.0, 0.0]))


# ----------------------------------------------------------------------------- materials

@dataclasses.dataclass
class Mixture:
    """Mixture{diffuse: Colored<Lambertian>, specular: Specular, luminous: Emissive<Absorbing>}."""
    diffuse_color: Sequence[float] = (0.0, 0.0, 0.0)
    diffuse: float = 0.0
    specular: float = 0.0
    emission: Sequence[float] = (0.0, 0.0, 0.0)
    luminous: float = 0.0

    @staticmethod
    def lambertian(color) -> "Mixture":
        return Mixture(diffuse_color=tuple(color), diffuse=1.0)

    @staticmethod
    def mirror() -> "Mixture":
        return Mixture(specular=1.0)

    @staticmethod
    def emitter(radiance) -> "Mixture":
        return Mixture(emission=tuple(radiance), luminous=1.0)


@dataclasses.dataclass
class SceneObject:
    map: object          # 2x2 complex ndarray (hyperbolic) or Hom3 (euclidean)
    shape: int           # SHAPE_PLANE or SHAPE_HOROSPHERE / SHAPE_SPHERE
    material: Mixture


@dataclasses.dataclass
class Scene:
    recipe: int
    camera: object                   # Moebius (2x2 complex) or Hom3
    fov: float
    background: Sequence[float]
    objects: List[SceneObject]
    hops: int

    @property
    def n_objects(self) -> int:
        return len(self.objects)

    def to_bytes(self, address_width: int = 32) -> bytes:
        return serialize(self, address_width)


# ----------------------------------------------------------------------------- serializer

def _f32(x) -> bytes:
    return struct.pack("<f", float(x))


def _usize(x: int, aw: int) -> bytes:
    return struct.pack("<I" if aw == 32 else "<Q", int(x))


def _moebius_bytes(m: np.ndarray) -> bytes:
    out = b""
    for (i, j) in ((0, 0), (0, 1), (1, 0), (1, 1)):
        out += _f32(m[i, j].real) + _f32(m[i, j].imag)
    return out


def _hom3_bytes(h: Hom3) -> bytes:
    return (_f32(h.shift[0]) + _f32(h.shift[1]) + _f32(h.shift[2]) + b"\0" * 4
            + b"".join(_f32(v) for v in h.rot))


def _object_bytes(o: SceneObject, recipe: int, aw: int) -> bytes:
    buf = bytearray(OBJ_STRIDE)
    buf[0:32] = _moebius_bytes(o.map) if recipe == RECIPE_HY else _hom3_bytes(o.map)
    m = o.material
    buf[32:44] = b"".join(_f32(c) for c in m.diffuse_color)
    buf[48:52] = _f32(m.diffuse)
    buf[64:68] = _f32(m.specular)
    buf[80:92] = b"".join(_f32(c) for c in m.emission)
    buf[96:100] = _f32(m.luminous)
    idx = _usize(o.shape, aw)
    buf[112:112 + len(idx)] = idx
    return bytes(buf)


def scene_size(recipe: int, n_objects: int) -> int:
    base = HY_OBJECTS_OFFSET if recipe == RECIPE_HY else EU_OBJECTS_OFFSET
    return base + OBJ_STRIDE * n_objects


def serialize(scene: Scene, address_width: int = 32) -> bytes:
    """Scene -> the bytes `EntityBuffer::new` would upload (config: little-endian,
    double_support = false, address width 32 or 64)."""
    if address_width not in (32, 64):
        raise ValueError("address_width must be 32 or 64")
    aw = address_width
    buf = bytearray(scene_size(scene.recipe, len(scene.objects)))
    if scene.recipe == RECIPE_HY:
        buf[0:32] = _moebius_bytes(scene.camera)
        buf[32:36] = _f32(scene.fov)
        buf[64:76] = b"".join(_f32(c) for c in scene.background)
        n = _usize(len(scene.objects), aw)
        buf[96:96 + len(n)] = n
        off = HY_OBJECTS_OFFSET
    elif scene.recipe == RECIPE_EU:
        buf[0:32] = _hom3_bytes(scene.camera)
        buf[32:36] = _f32(scene.fov)
        buf[48:60] = b"".join(_f32(c) for c in scene.background)
        n = _usize(len(scene.objects), aw)
        buf[64:64 + len(n)] = n
        off = EU_OBJECTS_OFFSET
    else:
        raise ValueError(f"unknown recipe {scene.recipe}")
    for i, o in enumerate(scene.objects):
        buf[off + OBJ_STRIDE * i: off + OBJ_STRIDE * (i + 1)] = _object_bytes(o, scene.recipe, aw)
    return bytes(buf)


# ----------------------------------------------------------------------------- seeds

def pixel_seeds(global_seed: int, n_pixels: int, offset: int = 0) -> np.ndarray:
    """Per-pixel initial RNG states: seed_i = fmix32(global_seed ^ fmix32(i + offset)).

    The reference fills its seed buffer from a host `SmallRng` stream
    (processing/src/canvas.rs:193-195); the kernel only consumes the buffer, so both the
    oracle and the CUDA path take these harness seeds (MurmurHash3's fmix32 finaliser).
    """
    def fmix(h):
        h = h.astype(np.uint64)
        h ^= h >> np.uint64(16)
        h = (h * np.uint64(0x85EBCA6B)) & np.uint64(0xFFFFFFFF)
        h ^= h >> np.uint64(13)
        h = (h * np.uint64(0xC2B2AE35)) & np.uint64(0xFFFFFFFF)
        h ^= h >> np.uint64(16)
        return h
    i = np.arange(offset, offset + n_pixels, dtype=np.uint64)
    return fmix(np.uint64(global_seed & 0xFFFFFFFF) ^ fmix(i)).astype(np.uint32)


# ----------------------------------------------------------------------------- generators

def _material_for(kind: int, rng: np.random.Generator) -> Mixture:
    if kind == 0:
        return Mixture.lambertian(rng.uniform(0.2, 0.9, 3))
    if kind == 1:
        return Mixture.mirror()
    return Mixture.emitter(rng.uniform(1.0, 5.0, 3))


def _material_kinds(n: int, rng: np.random.Generator) -> np.ndarray:
    """50 % Lambertian, 30 % mirror, 20 % emissive, assigned by object index after a
    seeded shuffle."""
    kinds = np.zeros(n, dtype=np.int64)
    n_mirror = int(round(0.3 * n))
    n_emit = int(round(0.2 * n))
    kinds[:n_emit] = 2
    kinds[n_emit:n_emit + n_mirror] = 1
    rng.shuffle(kinds)
    return kinds


def random_moebius(rng: np.random.Generator, max_distance: float) -> np.ndarray:
    """2x2 complex matrix with N(0,1) entries normalised to det = 1, rejected until its
    translation distance d(m·j, j) is at most `max_distance`."""
    while True:
        m = rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))
        det = m[0, 0] * m[1, 1] - m[0, 1] * m[1, 0]
        if abs(det) < 1e-3:
            continue
        m = mo_normalize(m)
        if hy_distance(mo_apply(m, J), J) <= max_distance:
            return m


def hyperbolic_scene(n_planes: int, n_horospheres: int, max_distance: float, hops: int,
                     seed: int, camera: Optional[np.ndarray] = None,
                     background=(0.3, 0.4, 0.6), fov: float = 1.0) -> Scene:
    rng = np.random.default_rng(seed)
    n = n_planes + n_horospheres
    shapes = np.array([SHAPE_PLANE] * n_planes + [SHAPE_HOROSPHERE] * n_horospheres)
    rng.shuffle(shapes)
    kinds = _material_kinds(n, rng)
    objs = [SceneObject(random_moebius(rng, max_distance), int(shapes[i]), _material_for(int(kinds[i]), rng))
            for i in range(n)]
    return Scene(RECIPE_HY, mo_identity() if camera is None else camera, fov,
                 tuple(background), objs, hops)


def euclidean_scene(n_spheres: int, hops: int, seed: int, camera: Optional[Hom3] = None,
                    background=(0.3, 0.4, 0.6), fov: float = 1.0) -> Scene:
    """Unit spheres (the reference's sphere is unit radius, shape/eu/sphere.cc:3-29, and
    Homogenous3 has no scale) centred in U[-4,4] x U[-4,4] x U[3,10], plus the ground plane
    y = -1. Camera at the origin looking +z: the reference camera looks along -z
    (view/point/impl.inl:23), so the camera map is a rotation by pi about y."""
    rng = np.random.default_rng(seed)
    kinds = _material_kinds(n_spheres, rng)
    objs = []
    for i in range(n_spheres):
        c = np.array([rng.uniform(-4, 4), rng.uniform(-4, 4), rng.uniform(3, 10)])
        objs.append(SceneObject(Hom3(c, np.array([1.0, 0.0, 0.0, 0.0])), SHAPE_SPHERE,
                                _material_for(int(kinds[i]), rng)))
    # Local plane z = 0 (normal (0,0,-1)) rotated so local +z maps to world +y, then y = -1.
    ground = Hom3(np.array([0.0, -1.0, 0.0]), quat_axis_angle([1, 0, 0], -np.pi / 2))
    objs.append(SceneObject(ground, SHAPE_PLANE, Mixture.lambertian((0.6, 0.6, 0.6))))
    cam = camera if camera is not None else Hom3(np.zeros(3), quat_axis_angle([0, 1, 0], np.pi))
    return Scene(RECIPE_EU, cam, fov, tuple(background), objs, hops)


@dataclasses.dataclass
class Workload:
    """One named synthetic workload: a scene plus image size and samples per pixel."""
    name: str
    scene: Scene
    width: int
    height: int
    spp: int
    global_seed: int


def config0(seed: int = 0x5EED0000) -> Workload:
    """Euclidean 320x240, 8 spheres + ground plane, H=4, 16 passes x 1 spp."""
    return Workload("euclidean-320x240-8spheres-h4", euclidean_scene(8, 4, seed), 320, 240, 16, seed)


def config1(seed: int = 0x5EED0001) -> Workload:
    """Hyperbolic 800x600, 12 geodesic planes + 6 horospheres, translation <= 3, H=6, 64 spp."""
    return Workload("hyperbolic-800x600-18obj-h6", hyperbolic_scene(12, 6, 3.0, 6, seed), 800, 600, 64, seed)


def config2(seed: int = 0x5EED0002) -> Workload:
    """Hyperbolic 1920x1080, 200 objects (60 % horospheres, 40 % planes), translation <= 6,
    H=8, 256 spp."""
    return Workload("hyperbolic-1920x1080-200obj-h8", hyperbolic_scene(80, 120, 6.0, 8, seed),
                    1920, 1080, 256, seed)
