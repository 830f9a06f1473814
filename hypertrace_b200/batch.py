"""Batched rendering: many views (either recipe, any resolution / hops / spp) per launch --
one launch per pass index, hop depth and recipe, each over every view's queue of ray states.

`BatchRenderer` wraps the `htc_batch_*` C ABI (include/htcuda.h). `config3()` builds the
mixed workload: 96 views with resolutions from {256x256, 640x480, 1280x720, 1920x1080},
spp uniform in {16, 32, ..., 256}, half Euclidean (8 unit spheres + ground plane, H = 4),
half hyperbolic (20-200 objects, 60 % horospheres, translation distance <= 6, H = 8), each
with a random camera. `autotune()` picks the largest tile size and the residency by timing
one render of one pass per candidate on the actual views.
"""
from __future__ import annotations

import ctypes
import dataclasses
import itertools
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from . import scene as S
from .processing import Canvas, Context, EntityBuffer


@dataclasses.dataclass
class View:
    """One view of a batch: its scene on the device, its canvas, passes per launch."""
    scene: S.Scene
    width: int
    height: int
    spp: int                      # total samples per pixel wanted
    global_seed: int
    buffer: Optional[EntityBuffer] = None
    canvas: Optional[Canvas] = None
    done_passes: int = 0
    flags: int = 0

    def allocate(self, ctx: Context) -> None:
        self.buffer = EntityBuffer(ctx, self.scene)
        self.canvas = Canvas(ctx, (self.width, self.height), self.global_seed)

    def release(self) -> None:
        self.buffer = None
        self.canvas = None

    @property
    def remaining(self) -> int:
        return self.spp - self.done_passes

    def device_bytes(self) -> int:
        # canvas (16 B) and seed (4 B) per pixel, two wavefront queue slots (2 x 68 B) per pixel
        return self.width * self.height * (16 + 4 + 136) + S.scene_size(self.scene.recipe, self.scene.n_objects)

    def descriptor(self, passes: int, address_width: int = 32) -> _lib.HtcView:
        return _lib.HtcView(self.buffer.ptr(), self.buffer.size, self.canvas.image.data_ptr(),
                            self.canvas.seeds.data_ptr(), self.width, self.height, self.scene.recipe,
                            self.scene.hops, self.flags, address_width, passes, 0)


class BatchRenderer:
    """htc_batch: a set of views with their regions of the batch's wavefront queues; render()
    runs every view's passes (bit-identical to rendering each view alone)."""

    def __init__(self, ctx: Context, max_views: int = 1024):
        self.ctx = ctx
        h = ctypes.c_void_p()
        _lib.call("htc_batch_create", max_views, ctypes.byref(h))
        self.handle = h
        self.tile_pixels = 2048
        self.blocks_per_sm = 0

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().htc_batch_destroy(h)
            except Exception:
                pass
            self.handle = None

    def set_views(self, views: Sequence[View], passes: Sequence[int], tile_pixels: Optional[int] = None,
                  blocks_per_sm: Optional[int] = None) -> None:
        if tile_pixels is not None:
            self.tile_pixels = tile_pixels
        if blocks_per_sm is not None:
            self.blocks_per_sm = blocks_per_sm
        arr = (_lib.HtcView * max(len(views), 1))()
        for i, (v, p) in enumerate(zip(views, passes)):
            arr[i] = v.descriptor(p)
        _lib.call("htc_batch_set_views", self.handle, ctypes.cast(arr, ctypes.c_void_p), len(views),
                  self.tile_pixels, self.blocks_per_sm, self.ctx.stream())

    def render(self, stats: Optional[torch.Tensor] = None, graph: bool = False) -> None:
        fn = "htc_batch_graph_launch" if graph else "htc_batch_render"
        _lib.call(fn, self.handle, None if stats is None else stats.data_ptr(), self.ctx.stream())

    def check(self) -> None:
        _lib.call("htc_batch_check", self.handle, self.ctx.stream())

    def reserve(self, pixels: int, max_hops: int) -> None:
        """Size the wavefront queues for view sets of up to `pixels` pixels and `max_hops` hops."""
        _lib.call("htc_batch_reserve", self.handle, pixels, max_hops, self.ctx.stream())



def random_hom3(rng: np.random.Generator) -> S.Hom3:
    """Random camera for the Euclidean views: a random rotation about the origin, looking
    roughly along +z (the scenes' spheres sit at z in [3, 10])."""
    yaw = np.pi + rng.uniform(-0.3, 0.3)
    pitch = rng.uniform(-0.2, 0.2)
    q = S._qmul(S.quat_axis_angle([0, 1, 0], yaw), S.quat_axis_angle([1, 0, 0], pitch))
    return S.Hom3(np.array([rng.uniform(-0.5, 0.5), rng.uniform(-0.5, 0.5), 0.0]), q)


def config3(seed: int = 0x5EED0003, n_views: int = 96, spp_scale: float = 1.0) -> List[View]:
    """The mixed batched workload (see module doc). spp_scale < 1 shortens every view's spp
    (rounded to a multiple of 16, at least 16) for quick runs."""
    rng = np.random.default_rng(seed)
    sizes = [(256, 256), (640, 480), (1280, 720), (1920, 1080)]
    views = []
    for i in range(n_views):
        w, h = sizes[rng.integers(len(sizes))]
        spp = 16 * int(rng.integers(1, 17))
        spp = max(16, int(round(spp * spp_scale / 16)) * 16)
        vseed = int(rng.integers(1 << 31))
        if i % 2 == 0:
            sc = S.euclidean_scene(8, 4, vseed, camera=random_hom3(rng))
        else:
            n = int(rng.integers(20, 201))
            n_h = int(round(0.6 * n))
            cam = S.random_moebius(rng, 1.0)
            sc = S.hyperbolic_scene(n - n_h, n_h, 6.0, 8, vseed, camera=cam)
        views.append(View(sc, w, h, spp, vseed))
    return views


def autotune(renderer: BatchRenderer, views: Sequence[View], passes: int = 1,
             tiles: Sequence[int] = (256, 512, 1024, 2048),
             residency: Sequence[int] = (3, 4, 5)) -> Tuple[int, int, dict]:
    """Times one launch of `passes` passes per candidate (tile size x blocks per SM) on the
    views themselves and returns the fastest (tile_pixels, blocks_per_sm, timings). The
    canvases and seeds are restored afterwards, so tuning leaves no trace in the results.
    Blocks per SM above the kernels' occupancy limit (5 resident blocks of 128 threads at
    their register cap) launch as that limit, so the default candidates stop there."""
    saved = [(v.canvas.image.clone(), v.canvas.seeds.clone()) for v in views]
    timings = {}
    stream = torch.cuda.current_stream(renderer.ctx.device)
    for tile, res in itertools.product(tiles, residency):
        renderer.set_views(views, [passes] * len(views), tile_pixels=tile, blocks_per_sm=res)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        renderer.render()
        e1.record(stream)
        e1.synchronize()
        timings[(tile, res)] = e0.elapsed_time(e1)
    for v, (img, sd) in zip(views, saved):
        v.canvas.image.copy_(img)
        v.canvas.seeds.copy_(sd)
    torch.cuda.synchronize()
    best = min(timings, key=timings.get)
    return best[0], best[1], timings
