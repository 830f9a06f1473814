"""Scene byte ABI: the serializer writes what the reference's types::io writer would.

Mirrors processing/src/tests/ocl.rs (struct size / offset probes) for the two recipes,
using the sizes the reference's Entity derive computes (type-macros/src/entity.rs).
"""
import struct

import numpy as np
import pytest

from hypertrace_b200 import scene as S


def _f(b, off):
    return struct.unpack_from("<f", b, off)[0]


def _u(b, off):
    return struct.unpack_from("<I", b, off)[0]


def test_sizes():
    assert S.scene_size(S.RECIPE_HY, 0) == 128
    assert S.scene_size(S.RECIPE_HY, 200) == 128 + 200 * 128
    assert S.scene_size(S.RECIPE_EU, 9) == 80 + 9 * 128
    for aw in (32, 64):
        assert len(S.config1().scene.to_bytes(aw)) == S.scene_size(S.RECIPE_HY, 18)
        assert len(S.config0().scene.to_bytes(aw)) == S.scene_size(S.RECIPE_EU, 9)


def test_alignment_multiples():
    # Vec<Mapped<..Moebius>> aligns to 32 (comp2x2 = real8), the euclidean one to 16.
    for n in range(5):
        assert S.scene_size(S.RECIPE_HY, n) % 32 == 0
        assert S.scene_size(S.RECIPE_EU, n) % 16 == 0


@pytest.mark.parametrize("aw", [32, 64])
def test_hyperbolic_offsets(aw):
    sc = S.config1().scene
    b = sc.to_bytes(aw)
    cam = sc.camera
    assert _f(b, 0) == np.float32(cam[0, 0].real) and _f(b, 24) == np.float32(cam[1, 1].real)
    assert _f(b, 32) == np.float32(sc.fov)
    assert [_f(b, 64 + 4 * i) for i in range(3)] == [np.float32(c) for c in sc.background]
    assert _u(b, 96) == sc.n_objects
    if aw == 64:
        assert _u(b, 100) == 0
    for i, o in enumerate(sc.objects):
        base = 128 + 128 * i
        m = o.map
        assert _f(b, base + 8) == np.float32(m[0, 1].real) and _f(b, base + 12) == np.float32(m[0, 1].imag)
        assert _f(b, base + 48) == np.float32(o.material.diffuse)
        assert _f(b, base + 64) == np.float32(o.material.specular)
        assert _f(b, base + 96) == np.float32(o.material.luminous)
        assert [_f(b, base + 80 + 4 * k) for k in range(3)] == [np.float32(c) for c in o.material.emission]
        assert _u(b, base + 112) == o.shape


def test_euclidean_offsets():
    sc = S.config0().scene
    b = sc.to_bytes()
    assert [_f(b, 16 + 4 * i) for i in range(4)] == [np.float32(v) for v in sc.camera.rot]
    assert _f(b, 32) == np.float32(sc.fov)
    assert [_f(b, 48 + 4 * i) for i in range(3)] == [np.float32(c) for c in sc.background]
    assert _u(b, 64) == sc.n_objects
    o = sc.objects[0]
    assert [_f(b, 80 + 4 * i) for i in range(3)] == [np.float32(v) for v in o.map.shift]
    assert _u(b, 80 + 112) == o.shape


def test_padding_is_zero():
    b = S.config1().scene.to_bytes()
    # padding after the view (36..64), after background (76..96), inside object records
    assert b[36:64] == bytes(28) and b[76:96] == bytes(20)
    assert b[128 + 44:128 + 48] == bytes(4) and b[128 + 116:128 + 128] == bytes(12)


def test_moebius_generators_det_one():
    rng = np.random.default_rng(0)
    for _ in range(50):
        m = S.random_moebius(rng, 3.0)
        det = m[0, 0] * m[1, 1] - m[0, 1] * m[1, 0]
        assert abs(det - 1) < 1e-12
        assert S.hy_distance(S.mo_apply(m, S.J), S.J) <= 3.0 + 1e-9


def test_hyperbolic_distance_invariance():
    """f64 host maps: an isometry preserves distance (kernel/ocl/geometry/hyperbolic.cc:128-147)."""
    rng = np.random.default_rng(1)
    for _ in range(100):
        a = np.array([*rng.normal(size=2), np.exp(rng.normal()), 0])
        b = np.array([*rng.normal(size=2), np.exp(rng.normal()), 0])
        m = S.mo_identity()
        for _ in range(8):
            k = rng.integers(3)
            m = S.mo_chain(m, [S.mo_yrotate(2 * np.pi * rng.uniform()), S.mo_zrotate(2 * np.pi * rng.uniform()),
                               S.mo_zshift(rng.normal())][k])
        assert abs(S.hy_distance(a, b) - S.hy_distance(S.mo_apply(m, a), S.mo_apply(m, b))) < 1e-9


def test_seeds_deterministic():
    a = S.pixel_seeds(5, 1000)
    b = S.pixel_seeds(5, 1000)
    assert a.dtype == np.uint32 and np.array_equal(a, b)
    assert len(np.unique(a)) > 990
    assert np.array_equal(S.pixel_seeds(5, 10, offset=100), S.pixel_seeds(5, 110)[100:])


def test_workload_shapes():
    c2 = S.config2()
    assert (c2.width, c2.height, c2.spp, c2.scene.hops) == (1920, 1080, 256, 8)
    shapes = [o.shape for o in c2.scene.objects]
    assert len(shapes) == 200 and shapes.count(S.SHAPE_HOROSPHERE) == 120
    c1 = S.config1()
    assert [o.shape for o in c1.scene.objects].count(S.SHAPE_PLANE) == 12
