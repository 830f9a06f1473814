"""Generates the golden fixtures in this folder from oracle/_ref -- the reference's own
kernel sources compiled as host C++ (oracle/ref/Makefile). Run here, where the reference
tree exists; the fixtures are committed so the CPU suite can pin the oracle without it.

    python tests/golden/make_golden.py

Each render fixture holds: the serialized scene bytes, image size, hops, recipe, a pixel
subset, the input seeds, and the reference's canvas + seeds after `passes` passes
(g++ evaluation order of the pixel jitter draws, see oracle.JITTER_YX).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hypertrace_b200 import scene as S  # noqa: E402
from hypertrace_b200 import types as T  # noqa: E402
from oracle import oracle  # noqa: E402

FORCE = "--force" in sys.argv


def bytes_fixture(name, data, recipe, hops, global_seed, W, H, n_pixels, passes, seed):
    path = os.path.join(HERE, f"{name}.npz")
    if os.path.exists(path) and not FORCE:
        return
    rng = np.random.default_rng(seed)
    pix = np.sort(rng.choice(W * H, n_pixels, replace=False)).astype(np.uint32)
    seeds = S.pixel_seeds(global_seed, W * H)[pix]
    out = oracle.render(data, recipe, hops, W, H, pix, seeds, passes=passes, impl="reference", threads=8)
    out64 = oracle.render(data, recipe, hops, W, H, pix, seeds, passes=passes, impl="reference",
                          threads=8, precision=64)
    np.savez_compressed(
        path,
        scene=np.frombuffer(data, dtype=np.uint8), recipe=recipe, hops=hops, width=W, height=H,
        passes=passes, pixels=pix, seeds_in=seeds, canvas_out=out.canvas, seeds_out=out.seeds,
        stats=np.array([out.stats[k] for k in ("samples", "hops", "object_tests", "hits")], dtype=np.uint64),
        canvas_out_f64=out64.canvas, seeds_out_f64=out64.seeds)
    print(name, out.stats)


def render_fixture(name, wl, W, H, n_pixels, passes, seed):
    sc = wl.scene
    bytes_fixture(name, sc.to_bytes(), sc.recipe, sc.hops, wl.global_seed, W, H, n_pixels, passes, seed)


def rng_fixture():
    if os.path.exists(os.path.join(HERE, "rng_stream.npz")) and not FORCE:
        return
    vals, state = oracle.rng_uniforms(0xDEADBEEF, 256, impl="reference")
    np.savez_compressed(os.path.join(HERE, "rng_stream.npz"), seed=np.uint32(0xDEADBEEF), uniforms=vals,
                        state=np.uint32(state))


if __name__ == "__main__":
    if not oracle.ref_available(32):
        raise SystemExit("oracle/_ref is not built (make -C oracle/ref REF=<reference root>)")
    rng_fixture()
    render_fixture("euclidean_320x240", S.config0(), 320, 240, 600, 3, 1)
    render_fixture("hyperbolic_800x600", S.config1(), 800, 600, 600, 2, 2)
    render_fixture("hyperbolic_1920x1080_200obj", S.config2(), 1920, 1080, 300, 2, 3)
    # edge cases: no objects (every path sees the background), one hop, a 1-pixel image
    empty = S.Scene(S.RECIPE_HY, S.mo_identity(), 1.0, (0.2, 0.3, 0.4), [], 3)
    render_fixture("hyperbolic_empty", S.Workload("empty", empty, 16, 8, 1, 11), 16, 8, 128, 2, 4)
    one = S.hyperbolic_scene(3, 2, 2.0, 1, 12)
    render_fixture("hyperbolic_onehop", S.Workload("onehop", one, 40, 30, 1, 12), 40, 30, 400, 3, 5)
    render_fixture("euclidean_1px", S.Workload("1px", S.euclidean_scene(4, 4, 13), 1, 1, 1, 13), 1, 1, 1, 4, 6)
    # the scene types of the reference's hy and eu examples (recipes 3 and 4)
    bytes_fixture("hy_tiled_800x600", T.serialize(T.hy_tiled_type(), T.hy_example_value()), 3, 3, 0x5EED0005,
                  800, 600, 800, 3, 7)
    bytes_fixture("eu_gradient_800x600", T.serialize(T.eu_gradient_type(), T.eu_example_value()), 4, 4, 0x5EED0006,
                  800, 600, 800, 3, 8)
    # a type no example builds (Linear3 chains both ways, shape vector of mapped shapes): the
    # oracle's recipe id 5; the CUDA path compiles it at run time
    bytes_fixture("eu_compound_640x480", T.serialize(T.eu_compound_type(), T.eu_compound_random_value(3, 7)), 5, 6,
                  0x5EED0008, 640, 480, 800, 3, 9)
