"""Pins the CPU restatement (oracle/htoracle.c) to the reference.

1. Golden fixtures (tests/golden/, generated from the reference's own kernel sources
   compiled as host C++ by tests/golden/make_golden.py): the restatement must reproduce
   canvas and seeds bit for bit, for f32 and for the f64 build.
2. Live comparison against oracle/_ref on fresh random scenes, when it is built.
"""
import glob
import os

import numpy as np
import pytest

from hypertrace_b200 import scene as S
from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz")) if not p.endswith("rng_stream.npz"))


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
@pytest.mark.parametrize("precision", [32, 64])
def test_port_reproduces_golden(built, path, precision):
    f = np.load(path)
    out = oracle.render(f["scene"].tobytes(), int(f["recipe"]), int(f["hops"]), int(f["width"]),
                        int(f["height"]), f["pixels"], f["seeds_in"], passes=int(f["passes"]),
                        flags=oracle.JITTER_YX, threads=4, precision=precision)
    key = "" if precision == 32 else "_f64"
    assert np.array_equal(out.seeds, f["seeds_out" + key])
    assert np.array_equal(out.canvas.view(np.uint32), f["canvas_out" + key].view(np.uint32))
    if precision == 32:
        assert [out.stats[k] for k in ("samples", "hops", "object_tests", "hits")] == list(f["stats"])


def test_rng_stream_golden(built):
    f = np.load(os.path.join(GOLDEN, "rng_stream.npz"))
    vals, state = oracle.rng_uniforms(int(f["seed"]), len(f["uniforms"]))
    assert np.array_equal(vals, f["uniforms"])
    assert state == int(f["state"])


def test_rng_known_answer(built):
    # LCG s' = 1103515245 s + 12345 (mod 2^32), u = (float)s' / 2^32 (random.cc:8-14)
    vals, state = oracle.rng_uniforms(0, 3)
    s = 0
    expect = []
    for _ in range(3):
        s = (1103515245 * s + 12345) & 0xFFFFFFFF
        expect.append(float(np.float32(s) / np.float32(2 ** 32)))
    assert list(vals) == expect
    assert state == s


def test_jitter_order_matters(built):
    """The two draw orders give different radiance but consume the same draws."""
    wl = S.config0()
    pix = np.arange(0, 320 * 240, 97, dtype=np.uint32)
    seeds = S.pixel_seeds(wl.global_seed, 320 * 240)[pix]
    a = oracle.render(wl.scene.to_bytes(), wl.scene.recipe, wl.scene.hops, 320, 240, pix, seeds, flags=0)
    b = oracle.render(wl.scene.to_bytes(), wl.scene.recipe, wl.scene.hops, 320, 240, pix, seeds,
                      flags=oracle.JITTER_YX)
    assert not np.array_equal(a.canvas, b.canvas)


def test_address_width_64_same_result(built):
    wl = S.config1()
    pix = np.arange(0, 800 * 600, 401, dtype=np.uint32)
    seeds = S.pixel_seeds(wl.global_seed, 800 * 600)[pix]
    a = oracle.render(wl.scene.to_bytes(32), 1, 6, 800, 600, pix, seeds, address_width=32)
    b = oracle.render(wl.scene.to_bytes(64), 1, 6, 800, 600, pix, seeds, address_width=64)
    assert np.array_equal(a.seeds, b.seeds)
    assert np.array_equal(a.canvas, b.canvas)


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", [101, 202, 303])
@pytest.mark.parametrize("recipe", [S.RECIPE_HY, S.RECIPE_EU])
def test_port_matches_reference_live(built, seed, recipe):
    rng = np.random.default_rng(seed)
    if recipe == S.RECIPE_HY:
        sc = S.hyperbolic_scene(int(rng.integers(1, 10)), int(rng.integers(0, 10)), float(rng.uniform(1, 6)),
                                int(rng.integers(1, 9)), seed)
    else:
        sc = S.euclidean_scene(int(rng.integers(1, 12)), int(rng.integers(1, 6)), seed)
    W, H = 64, 48
    pix = np.arange(W * H, dtype=np.uint32)
    seeds = S.pixel_seeds(seed, W * H)
    data = sc.to_bytes()
    for precision in (32, 64):
        ref = oracle.render(data, recipe, sc.hops, W, H, pix, seeds, passes=2, impl="reference",
                            precision=precision, threads=4)
        port = oracle.render(data, recipe, sc.hops, W, H, pix, seeds, passes=2, flags=oracle.JITTER_YX,
                             precision=precision, threads=4)
        assert np.array_equal(ref.seeds, port.seeds)
        assert np.array_equal(ref.canvas.view(np.uint32), port.canvas.view(np.uint32))
        assert ref.stats == port.stats


def test_bad_scene_rejected(built):
    wl = S.config1()
    data = bytearray(wl.scene.to_bytes())
    with pytest.raises(RuntimeError):
        oracle.render(bytes(data[:100]), 1, 6, 8, 8, [0], [1])
    data[96:100] = (1000).to_bytes(4, "little")
    with pytest.raises(RuntimeError):
        oracle.render(bytes(data), 1, 6, 8, 8, [0], [1])
    good = bytearray(wl.scene.to_bytes())
    good[128 + 112:128 + 116] = (7).to_bytes(4, "little")  # shape index out of range
    with pytest.raises(RuntimeError):
        oracle.render(bytes(good), 1, 6, 8, 8, [0], [1])
