"""Property tests of the device primitives, after the reference's own unit tests.

The reference tests its kernel library with property tests (no golden vectors):
transform/moebius.cc:97-137 (chaining), geometry/hyperbolic.cc:128-205 (distance invariance
under isometries), shape/hy/plane.cc:49-71 and horosphere.cc:47-69 (hits lie on the shape,
unit directions and normals), shape/eu/sphere.cc:41-64, random.cc:127-247 (samplers),
material/lambertian.cc:28-69, specular.cc:21-45, refractive and transparent materials.
The same properties are checked here on the CUDA implementations (evaluated by
tests/cuda/libht_selftest.so), and where the reference's own code is built (oracle/_ref)
its outputs are compared bit for bit with the device's.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cuda", "libht_selftest.so")
EPS = 1e-6
N = 4096
CONF = 3.0 / np.sqrt(N)

EV = dict(MO_APPLY=0, MO_CHAIN=1, RAY_MAP=2, HY_DIST=3, PLANE_HY=4, HOROSPHERE=5, HEMI=6, LAMBERT=7,
          SPECULAR=8, REFRACTIVE=9, SPHERE=10, CUBE=11, PLANE_EU=12, RNG=13)
OUT = dict(MO_APPLY=4, MO_CHAIN=8, RAY_MAP=8, HY_DIST=2, PLANE_HY=13, HOROSPHERE=13, HEMI=3, LAMBERT=4,
           SPECULAR=4, REFRACTIVE=4, SPHERE=7, CUBE=7, PLANE_EU=7, RNG=4)


@pytest.fixture(scope="module")
def ev(built):
    lib = ctypes.CDLL(LIB)
    fn = lib.ht_selftest_eval
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                   ctypes.c_void_p]

    def run(kind, inp, seeds=None):
        inp = np.ascontiguousarray(inp, dtype=np.float32)
        n, stride = inp.shape
        out = np.zeros((n, OUT[kind]), dtype=np.float32)
        sd = None if seeds is None else np.ascontiguousarray(seeds, dtype=np.uint32).copy()
        rc = fn(EV[kind], n, inp.ctypes.data, stride, out.ctypes.data, OUT[kind],
                None if sd is None else sd.ctypes.data)
        assert rc == 0
        return out if sd is None else (out, sd)
    return run


def rand_moebius(rng, n):
    """det-1 maps from N(0,1) complex entries (c22_normalize, matrix_complex.cc:50-52), as 8 floats."""
    m = rng.normal(size=(n, 2, 2)) + 1j * rng.normal(size=(n, 2, 2))
    det = m[:, 0, 0] * m[:, 1, 1] - m[:, 0, 1] * m[:, 1, 0]
    m = m / np.sqrt(det)[:, None, None]
    flat = np.stack([m[:, 0, 0], m[:, 0, 1], m[:, 1, 0], m[:, 1, 1]], axis=1)
    return np.stack([flat.real, flat.imag], axis=2).reshape(n, 8).astype(np.float32)


def rand_hypos(rng, n):
    """Points of the half-space (TestRngHyPos::normal: xy normal, z = exp(normal))."""
    return np.stack([rng.normal(size=n), rng.normal(size=n), np.exp(rng.normal(size=n)), np.zeros(n)], 1)


def rand_unit(rng, n, dims=3):
    v = rng.normal(size=(n, dims))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def qmul_np(a, b):
    return np.stack([a[:, 0] * b[:, 0] - a[:, 1] * b[:, 1] - a[:, 2] * b[:, 2] - a[:, 3] * b[:, 3],
                     a[:, 0] * b[:, 1] + a[:, 1] * b[:, 0] + a[:, 2] * b[:, 3] - a[:, 3] * b[:, 2],
                     a[:, 0] * b[:, 2] + a[:, 2] * b[:, 0] - a[:, 1] * b[:, 3] + a[:, 3] * b[:, 1],
                     a[:, 0] * b[:, 3] + a[:, 3] * b[:, 0] + a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1]], 1)


def hy_dist_np(a, b):
    x = 1 + np.sum((a - b) ** 2, axis=1) / (2 * a[:, 2] * b[:, 2])
    return np.arccosh(x)


def test_moebius_chaining(ev):   # transform/moebius.cc:97-106
    rng = np.random.default_rng(1)
    inp = np.concatenate([rand_moebius(rng, N), rand_moebius(rng, N), rand_hypos(rng, N)], 1)
    out = ev("MO_CHAIN", inp)
    a, b = out[:, :4].astype(np.float64), out[:, 4:].astype(np.float64)
    scale = np.maximum(np.linalg.norm(b, axis=1), 1.0)
    assert np.all(np.linalg.norm(a - b, axis=1) <= 1e-3 * scale)
    assert np.all(np.abs(out[:, 3]) <= 1e-3 * scale) and np.all(out[:, 2] > 0)   # stays in the half-space


def test_moebius_inverse_round_trip(ev):   # mo_inverse = adjugate for det-1 maps
    rng = np.random.default_rng(2)
    m = rand_moebius(rng, N)
    p = rand_hypos(rng, N)
    q = ev("MO_APPLY", np.concatenate([m, p], 1))
    inv = m.copy().reshape(N, 4, 2)
    inv[:, [0, 3]] = m.reshape(N, 4, 2)[:, [3, 0]]
    inv[:, [1, 2]] = -m.reshape(N, 4, 2)[:, [1, 2]]
    back = ev("MO_APPLY", np.concatenate([inv.reshape(N, 8), q], 1))
    ok = np.linalg.norm(back - p, axis=1) <= 1e-3 * np.maximum(np.linalg.norm(p, axis=1), 1) * np.maximum(np.linalg.norm(q, axis=1), 1)
    assert ok.mean() > 0.999


def test_distance_invariance(ev):   # geometry/hyperbolic.cc:146-164
    rng = np.random.default_rng(3)
    a, b = rand_hypos(rng, N), rand_hypos(rng, N)
    out = ev("HY_DIST", np.concatenate([a, b, rand_moebius(rng, N)], 1)).astype(np.float64)
    ref = hy_dist_np(a, b)
    assert np.allclose(out[:, 0], ref, rtol=1e-4, atol=1e-3)
    assert np.median(np.abs(out[:, 1] - out[:, 0]) / np.maximum(out[:, 0], 1e-3)) < 1e-4
    assert np.mean(np.abs(out[:, 1] - out[:, 0]) <= 1e-2 * np.maximum(out[:, 0], 1)) > 0.99


def test_ray_map_unit_and_matches_reference(ev):
    rng = np.random.default_rng(4)
    m, p = rand_moebius(rng, N), rand_hypos(rng, N)
    v = np.concatenate([rand_unit(rng, N), np.zeros((N, 1))], 1)
    out = ev("RAY_MAP", np.concatenate([m, p, v], 1))
    assert np.allclose(np.linalg.norm(out[:, 4:], axis=1), 1, atol=1e-5)
    assert np.all(out[:, 2] > 0)
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    lib = ctypes.CDLL(os.path.join(oracle.REF_DIR, "libhtref_f32.so"))
    fn = lib.htref_ray_hy_map
    fn.argtypes = [ctypes.c_void_p] * 4
    same = 0
    for i in range(512):
        mm = np.ascontiguousarray(m[i], dtype=np.float32)
        pp = np.ascontiguousarray(p[i].astype(np.float32), dtype=np.float64)
        vv = np.ascontiguousarray(v[i].astype(np.float32), dtype=np.float64)
        o = np.zeros(8)
        fn(mm.ctypes.data, pp.ctypes.data, vv.ctypes.data, o.ctypes.data)
        same += np.array_equal(o.astype(np.float32), out[i])
    assert same == 512, f"{512 - same} of 512 ray maps differ from the reference's"


def test_plane_hy_detect(ev):   # shape/hy/plane.cc:49-71
    rng = np.random.default_rng(5)
    d = np.concatenate([rand_unit(rng, N), np.zeros((N, 1))], 1)
    out = ev("PLANE_HY", np.concatenate([rand_hypos(rng, N), d, np.zeros((N, 1))], 1)).astype(np.float64)
    hit = out[:, 0] > -EPS
    assert hit.sum() > N // 10
    start, direction, normal = out[hit, 1:5], out[hit, 5:9], out[hit, 9:13]
    assert np.allclose(np.linalg.norm(start, axis=1), 1, atol=1e-4)
    assert np.allclose(np.linalg.norm(direction, axis=1), 1, atol=1e-4)
    assert np.allclose(normal, -start, atol=1e-6)
    repeat = ev("PLANE_HY", np.concatenate([rand_hypos(rng, N), d, np.ones((N, 1))], 1))
    assert np.all(repeat[:, 0] == -1)   # a plane is never hit twice in a row


def test_horosphere_detect(ev):   # shape/hy/horosphere.cc:47-69
    rng = np.random.default_rng(6)
    p = rand_hypos(rng, N)
    d = np.concatenate([rand_unit(rng, N), np.zeros((N, 1))], 1)
    out = ev("HOROSPHERE", np.concatenate([p, d, np.zeros((N, 1))], 1)).astype(np.float64)
    hit = out[:, 0] > -EPS
    above = p[:, 2] > 1 + EPS
    assert np.all(hit[above])
    assert np.allclose(out[above, 9:13], [0, 0, -1, 0])
    assert np.allclose(out[hit, 3], 1, atol=1e-6)
    assert np.allclose(np.linalg.norm(out[hit, 5:9], axis=1), 1, atol=1e-4)


def test_hemisphere_cosine(ev):   # random.cc:136-160
    seeds = np.arange(N, dtype=np.uint32) * 2654435761 + 12345
    out, _ = ev("HEMI", np.zeros((N, 1)), seeds)
    out = out.astype(np.float64)
    assert np.allclose(np.linalg.norm(out, axis=1), 1, atol=1e-5)
    assert np.all(out[:, 2] > -EPS)
    assert np.abs(out[:, :2].mean(0)).max() < 2 * CONF
    assert abs(out[:, 2].mean() - 2.0 / 3.0) < 2 * CONF   # E[cos] of a cosine-weighted hemisphere
    if oracle.ref_available():
        lib = ctypes.CDLL(os.path.join(oracle.REF_DIR, "libhtref_f32.so"))
        fn = lib.htref_hemisphere_cosine
        fn.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
        ref = np.zeros((1024, 3))
        for i in range(1024):
            st = ctypes.c_uint32()
            fn(int(seeds[i]), 1, ref[i].ctypes.data, ctypes.byref(st))
        ref, dev = ref.astype(np.float32), out[:1024].astype(np.float32)
        # z is a square root on both sides: exact. x and y carry cos/sin, which the device rounds
        # once from FP64 and the host libm (cosf/sinf, not correctly rounded) rounds within 0.56 ulp;
        # times sin_theta, one ulp there is at most two in the product.
        assert np.array_equal(ref[:, 2], dev[:, 2])
        gap = np.abs(ref[:, :2] - dev[:, :2])
        assert np.all(gap <= 2 * np.spacing(np.maximum(np.abs(ref[:, :2]), np.abs(dev[:, :2]))))
        assert np.mean(np.all(ref == dev, axis=1)) > 0.95


def test_rng_stream_matches_reference(ev):   # random.cc:8-14
    seeds = np.arange(N, dtype=np.uint32) * 747796405 + 2891336453
    out, state = ev("RNG", np.zeros((N, 1)), seeds)
    s = seeds.astype(np.uint64)
    for k in range(4):
        s = (1103515245 * s + 12345) & 0xFFFFFFFF
        assert np.array_equal(out[:, k], s.astype(np.float32) / np.float32(2 ** 32))
    assert np.array_equal(state, s.astype(np.uint32))


def test_lambertian(ev):   # material/lambertian.cc:28-69
    rng = np.random.default_rng(7)
    n = np.tile(rand_unit(rng, 1), (N, 1))
    d = rand_unit(rng, N)
    d[np.sum(d * n, 1) > 0] *= -1
    seeds = rng.integers(0, 2 ** 32, N, dtype=np.uint64).astype(np.uint32)
    out, _ = ev("LAMBERT", np.concatenate([n, d], 1), seeds)
    o = out[:, :3].astype(np.float64)
    assert np.all(out[:, 3] == 1)
    assert np.allclose(np.linalg.norm(o, axis=1), 1, atol=1e-5)
    assert np.all(np.sum(o * n, 1) > 0)   # leaves on the side the light came from
    assert abs(np.sum(o * n, 1).mean() - 2.0 / 3.0) < 2 * CONF


def test_specular(ev):   # material/specular.cc:21-45
    rng = np.random.default_rng(8)
    n, d = rand_unit(rng, N), rand_unit(rng, N)
    d[np.sum(d * n, 1) > 0] *= -1
    out = ev("SPECULAR", np.concatenate([n, d], 1)).astype(np.float64)
    o = out[:, :3]
    assert np.all(out[:, 3] == 1)
    assert np.allclose(np.sum(o * n, 1), -np.sum(d * n, 1), atol=1e-5)
    assert np.allclose(o - np.sum(o * n, 1, keepdims=True) * n, d - np.sum(d * n, 1, keepdims=True) * n, atol=1e-5)


def test_refractive(ev):   # material/refractive.cc:4-22: Snell's law, total internal reflection
    rng = np.random.default_rng(9)
    n, d = rand_unit(rng, N), rand_unit(rng, N)
    index = rng.uniform(1.1, 2.0, N)
    out = ev("REFRACTIVE", np.concatenate([n, d, index[:, None]], 1)).astype(np.float64)
    o = out[:, :3]
    a = np.sum(d * n, 1)
    k = np.where(a < -EPS, 1 / index, index)
    x = (a * a - 1) * k * k + 1
    refr = x > EPS
    assert np.all(out[:, 3] == 1)
    dt, ot = d - a[:, None] * n, o - np.sum(o * n, 1, keepdims=True) * n
    assert np.allclose(ot[refr], (k[:, None] * dt)[refr], atol=1e-5)   # tangential part scales by k
    assert np.allclose(np.linalg.norm(o[refr], axis=1), 1, atol=1e-4)
    assert np.allclose(np.sum(o * n, 1)[refr] * np.sign(a[refr]), np.sqrt(x[refr]), atol=1e-4)
    assert np.allclose(np.sum(o * n, 1)[~refr], -a[~refr], atol=1e-5)   # reflected


@pytest.mark.parametrize("shape", ["SPHERE", "CUBE", "PLANE_EU"])
def test_euclidean_shapes(ev, shape):   # shape/eu/sphere.cc:41-64, cube.cc, plane.cc
    rng = np.random.default_rng(10)
    p = rng.normal(size=(N, 3)) * 1.5
    d = rand_unit(rng, N)
    out = ev(shape, np.concatenate([p, d, np.zeros((N, 1))], 1)).astype(np.float64)
    hit = out[:, 0] > -EPS
    assert hit.sum() > N // 10
    h, nrm, t = out[hit, 1:4], out[hit, 4:7], out[hit, 0]
    assert np.allclose(h, p[hit] + t[:, None] * d[hit], atol=1e-4 * np.maximum(1, np.abs(t))[:, None])
    if shape == "SPHERE":
        assert np.allclose(np.linalg.norm(h, axis=1), 1, atol=1e-5) and np.allclose(nrm, h)
    elif shape == "CUBE":
        assert np.allclose(np.abs(h).max(1), 1, atol=1e-4)
        inside = np.abs(p[hit]).max(1) < 1   # a ray from inside leaves through a face, normal outward
        assert np.allclose(np.abs(nrm).sum(1), 1)
        assert np.all(np.sum(nrm * d[hit], 1)[~inside] <= 0) and np.all(np.sum(nrm * d[hit], 1)[inside] >= 0)
    else:
        assert np.allclose(h[:, 2], 0) and np.allclose(nrm, [0, 0, -1])
