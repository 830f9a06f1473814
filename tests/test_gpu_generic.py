"""GPU: the generic scene programs (hypertrace_b200/csrc/ht_generic.cuh).

  * the built-in recipes for the reference's hy and eu example types
    (HTC_RECIPE_HY_TILED, HTC_RECIPE_EU_GRADIENT) against the golden fixtures of the
    reference's own kernel code and against the C port on random scenes of those types;
  * programs compiled at run time with NVRTC (htc_program_build) from the Python type
    mirror: the hearth / Euclidean types reproduce the hand-written kernels bit for bit,
    the example types reproduce the built-in recipes, a type served by no recipe (an extra
    one-variant object choice) reproduces the equivalent recipe;
  * errors: a type that does not compile, a scene smaller than its type, an object count
    beyond the buffer.
The comparison bar is the one of test_gpu_parity.py, with one difference for the gradient
background (background/gradient.cc:3-13): it raises a float to a float power, which the
reference's host build evaluates with glibc's powf (not correctly rounded: errors up to about
0.8 ulp) and the CUDA path as the FP64 power rounded once. The two differ by one ulp on a few
per cent of the background hits, so on scenes with that background the radiance is compared
with the 1e-4 tolerance everywhere but is bit-identical only on >= GRADIENT_MIN_EXACT of the
pixels (RNG streams stay bit-exact: the power decides no branch).
"""
import os

import numpy as np
import pytest
import torch

from hypertrace_b200 import _lib
from hypertrace_b200 import processing as P
from hypertrace_b200 import scene as S
from hypertrace_b200 import types as T
from oracle import oracle

from test_gpu_parity import _compare

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GRADIENT_MIN_EXACT = 0.95
# Random scenes of these types run more hops (5-6) than the golden cases; a path diverges
# when any of its hops takes a branch on a last-ulp transcendental difference, so the bound on
# diverged pixels scales with hops x passes (0.2 % at the fixtures' 2-3 hops x 2-3 passes).
RANDOM_MAX_MISMATCH = 0.005


def _run(render, data, W, H, seeds, passes, persistent=True, stats=None):
    ctx = render.context
    scene = torch.from_numpy(np.frombuffer(data, dtype=np.uint8).copy()).to(ctx.device)
    canvas = torch.zeros(W * H * 4, dtype=torch.float32, device=ctx.device)
    sd = torch.from_numpy(np.asarray(seeds, dtype=np.uint32).view(np.int32).copy()).to(ctx.device)
    st = None if stats is None else stats.data_ptr()
    if persistent:
        _lib.call("htc_render_passes", render.handle, W, H, scene.data_ptr(), scene.numel(), canvas.data_ptr(),
                  sd.data_ptr(), passes, st, ctx.stream())
    else:
        for _ in range(passes):
            _lib.call("htc_render_ex", render.handle, W, H, scene.data_ptr(), scene.numel(), canvas.data_ptr(),
                      sd.data_ptr(), st, ctx.stream())
    _lib.call("htc_program_check", render.handle, ctx.stream())
    return canvas.cpu().numpy().reshape(-1, 4).copy(), sd.cpu().numpy().view(np.uint32).copy()


@pytest.mark.parametrize("name", ["hy_tiled_800x600", "eu_gradient_800x600"])
@pytest.mark.parametrize("persistent", [False, True])
def test_example_recipes_match_golden(built, name, persistent):
    f = np.load(os.path.join(GOLDEN, name + ".npz"))
    W, H, passes, pix = int(f["width"]), int(f["height"]), int(f["passes"]), f["pixels"]
    ctx = P.Context(0)
    r = P.Render(ctx, int(f["recipe"]), int(f["hops"]), _lib.HTC_FLAG_JITTER_YX)
    seeds = np.zeros(W * H, dtype=np.uint32)
    seeds[pix] = f["seeds_in"]
    stats = torch.zeros(8, dtype=torch.int64, device=ctx.device)
    cv, sd = _run(r, f["scene"].tobytes(), W, H, seeds, passes, persistent, stats)

    class Ref:
        canvas = f["canvas_out"]
        seeds = f["seeds_out"]
    _compare(cv[pix], sd[pix], Ref, f"golden {name} persistent={persistent}",
             min_exact=GRADIENT_MIN_EXACT if name.startswith("eu_gradient") else 1.0 - 0.002)
    assert np.array_equal(sd[pix], f["seeds_out"])
    assert int(stats[0]) == W * H * passes


@pytest.mark.parametrize("seed", [5, 6])
@pytest.mark.parametrize("recipe", [_lib.HTC_RECIPE_HY_TILED, _lib.HTC_RECIPE_EU_GRADIENT])
def test_example_recipes_match_port_random(built, seed, recipe):
    if recipe == _lib.HTC_RECIPE_HY_TILED:
        ty, val, hops = T.hy_tiled_type(), T.hy_tiled_random_value(seed, 10), 5
    else:
        ty, val, hops = T.eu_gradient_type(), T.eu_gradient_random_value(seed, 9), 6
    W, H, passes = 96, 64, 3
    seeds = S.pixel_seeds(seed, W * H)
    ctx = P.Context(0)
    r = P.Render(ctx, recipe, hops)
    out = {}
    for aw in (32, 64):
        data = T.serialize(ty, val, aw)
        rr = r if aw == 32 else P.Render(P.Context(0, P.Config(address_width=64)), recipe, hops)
        out[aw] = _run(rr, data, W, H, seeds, passes)
    assert np.array_equal(out[32][0], out[64][0]) and np.array_equal(out[32][1], out[64][1])
    ref = oracle.render(T.serialize(ty, val), recipe, hops, W, H, np.arange(W * H), seeds, passes=passes, threads=8)
    _compare(out[32][0], out[32][1], ref, f"recipe {recipe} seed {seed}",
             min_exact=GRADIENT_MIN_EXACT if recipe == _lib.HTC_RECIPE_EU_GRADIENT else 1.0 - RANDOM_MAX_MISMATCH,
             max_mismatch=RANDOM_MAX_MISMATCH)


def _same(a, b):
    return np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32)) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("which", ["hearth", "euclid"])
def test_nvrtc_generic_equals_handwritten(built, which):
    """The generic templates of the hearth / Euclidean types, compiled at run time, give the
    hand-written kernels' results bit for bit (both follow the reference op for op)."""
    wl = S.config1() if which == "hearth" else S.config0()
    ty = T.hearth_type() if which == "hearth" else T.euclid_type()
    W, H, passes = 200, 150, 2
    seeds = S.pixel_seeds(wl.global_seed, W * H)
    ctx = P.Context(0)
    data = T.serialize(ty, T.hearth_value(wl.scene))
    assert data == wl.scene.to_bytes()
    hand = P.Render(ctx, wl.scene.recipe, wl.scene.hops)
    gen = P.Render.build(ctx, ty, wl.scene.hops)
    assert gen.static_size() == T.static_size(ty)
    a = _run(hand, data, W, H, seeds, passes)
    b = _run(gen, data, W, H, seeds, passes)
    assert _same(a, b)


@pytest.mark.parametrize("recipe", [_lib.HTC_RECIPE_HY_TILED, _lib.HTC_RECIPE_EU_GRADIENT])
def test_nvrtc_build_equals_builtin_recipe(built, recipe):
    ty = T.hy_tiled_type() if recipe == _lib.HTC_RECIPE_HY_TILED else T.eu_gradient_type()
    val = T.hy_example_value() if recipe == _lib.HTC_RECIPE_HY_TILED else T.eu_example_value()
    W, H, passes = 160, 120, 3
    seeds = S.pixel_seeds(9, W * H)
    ctx = P.Context(0)
    data = T.serialize(ty, val)
    a = _run(P.Render(ctx, recipe, 4), data, W, H, seeds, passes)
    b = _run(P.Render.build(ctx, ty, 4), data, W, H, seeds, passes)
    assert _same(a, b)


def test_nvrtc_type_served_by_no_recipe(built):
    """eu.rs's type with each object wrapped in a one-variant object choice: different bytes
    (a usize index, the payload at the choice's alignment), the same results."""
    mat = T.eu_gradient_material()
    shape = T.ShapeChoice("Eu", ("Plane", T.PlaneEu()), ("Sphere", T.Sphere()), ("Cube", T.Cube()))
    covered = T.Covered("Eu", shape, mat)
    wrapped = T.ObjectChoice("Eu", ("Only", covered))
    ty = T.SceneImpl("Eu", T.MappedView("Eu", T.PointView("Eu"), T.Homogenous3()),
                     T.ObjectVec("Eu", T.MappedObject("Eu", wrapped, T.Shift3())), T.GradBg())
    val = T.eu_gradient_random_value(3, 8)
    val2 = dict(val)
    val2["object"] = [{"map": o["map"], "inner": ("Only", o["inner"])} for o in val["object"]]
    d1 = T.serialize(T.eu_gradient_type(), val)
    d2 = T.serialize(ty, val2)
    assert d1 != d2
    W, H, passes = 128, 96, 2
    seeds = S.pixel_seeds(4, W * H)
    ctx = P.Context(0)
    gen = P.Render.build(ctx, ty, 5)
    assert gen.static_size() == T.static_size(ty)
    a = _run(P.Render(ctx, _lib.HTC_RECIPE_EU_GRADIENT, 5), d1, W, H, seeds, passes)
    b = _run(gen, d2, W, H, seeds, passes)
    assert _same(a, b)


def test_generic_errors(built):
    ctx = P.Context(0)
    with pytest.raises(_lib.HtcError) as e:
        P.Render.build(ctx, "SceneImpl<Hy, NoSuchView, ObjectVec<Hy, Sphere>, ConstBg>", 3)
    assert e.value.code == _lib.HTC_ERR_INVALID
    r = P.Render(ctx, _lib.HTC_RECIPE_HY_TILED, 3)
    data = T.serialize(T.hy_tiled_type(), T.hy_example_value())
    with pytest.raises(_lib.HtcError) as e:
        _run(r, data[:100], 8, 8, np.ones(64, dtype=np.uint32), 1)
    assert e.value.code == _lib.HTC_ERR_SCENE
    bad = bytearray(data)
    bad[96:100] = (1000).to_bytes(4, "little")   # more objects than the buffer holds
    with pytest.raises(_lib.HtcError) as e:
        _run(r, bytes(bad), 8, 8, np.ones(64, dtype=np.uint32), 1)
    assert e.value.code == _lib.HTC_ERR_SCENE
    # the program stays usable after the error
    cv, sd = _run(r, data, 8, 8, np.ones(64, dtype=np.uint32), 1)
    assert np.all(cv[:, 3] == 1.0)


def test_nvrtc_compound_type_matches_reference(built):
    """A type no example builds, served only by the run-time compiler: one mapped object
    (Chain<Linear3, Shift3>) whose shape is a vector of mapped shapes (Chain<Shift3, Linear3>),
    gradient background. Against the reference's fixture (g++ draw order) and the C port on a
    fresh scene (OpenCL draw order)."""
    f = np.load(os.path.join(GOLDEN, "eu_compound_640x480.npz"))
    W, H, passes, pix = int(f["width"]), int(f["height"]), int(f["passes"]), f["pixels"]
    ctx = P.Context(0)
    ty = T.eu_compound_type()
    r = P.Render.build(ctx, ty, int(f["hops"]), _lib.HTC_FLAG_JITTER_YX)
    assert r.static_size() == T.static_size(ty)
    seeds = np.zeros(W * H, dtype=np.uint32)
    seeds[pix] = f["seeds_in"]
    cv, sd = _run(r, f["scene"].tobytes(), W, H, seeds, passes)

    class Ref:
        canvas = f["canvas_out"]
        seeds = f["seeds_out"]
    _compare(cv[pix], sd[pix], Ref, "golden eu_compound_640x480", min_exact=GRADIENT_MIN_EXACT)
    val = T.eu_compound_random_value(8, 9)
    data = T.serialize(ty, val)
    W, H = 96, 64
    seeds = S.pixel_seeds(8, W * H)
    cv, sd = _run(P.Render.build(ctx, ty, 6), data, W, H, seeds, 2)
    ref = oracle.render(data, 5, 6, W, H, np.arange(W * H), seeds, passes=2, threads=8)
    _compare(cv, sd, ref, "compound random", min_exact=GRADIENT_MIN_EXACT, max_mismatch=RANDOM_MAX_MISMATCH)
