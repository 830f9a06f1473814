"""Host mirror of the reference's `processing` crate over the CUDA C ABI.

Same names and meaning as processing/src/*.rs: `Context`, `EntityBuffer`, `Canvas`,
`Render`, `Extractor`, `GammaFilter`, `Packer`, `Pipeline` (processing/src/pipeline.rs:8-67).
Device memory is held in torch tensors (plumbing only); every computation goes through
libhtcuda.so. `Render.render` keeps the reference's blocking semantics (enqueue, then
`finish()`, then `add_pass`, processing/src/render.rs:102-118).
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional, Tuple

import numpy as np
import torch

from . import _lib
from .scene import RECIPE_HY, Scene, serialize


@dataclasses.dataclass
class Config:
    """types::Config (types/src/config.rs:39-49); little-endian only."""
    address_width: int = 32
    double_support: bool = False


class Context:
    """processing::Context: the device plus the serialization config."""

    def __init__(self, device: int = 0, config: Optional[Config] = None):
        if not torch.cuda.is_available():
            raise RuntimeError("the CUDA render path needs a GPU")
        self.device = torch.device("cuda", device)
        self.config = config or Config()
        torch.cuda.set_device(self.device)
        _lib.call("htc_set_device", device)

    def stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream


class EntityBuffer:
    """Serialized scene bytes on the device (processing/src/buffer.rs:13-29).

    `scene` is a scene.Scene (recipes HTC_RECIPE_HY / EU), already serialized bytes, or a
    value of `scene_type` (a hypertrace_b200.types entity type, for any other scene). The
    context's config decides the layout (address width, double_support), as the reference's
    EntityBuffer::new serializes with the context's config."""

    def __init__(self, context: Context, scene, scene_type=None):
        cfg = context.config
        if isinstance(scene, (bytes, bytearray)):
            data = bytes(scene)
        elif scene_type is not None:
            from . import types as T
            data = T.serialize(scene_type, scene, cfg.address_width, cfg.double_support)
        elif cfg.double_support:
            from . import types as T
            ty = T.hearth_type() if scene.recipe == RECIPE_HY else T.euclid_type()
            data = T.serialize(ty, T.hearth_value(scene), cfg.address_width, double_support=True)
        else:
            data = serialize(scene, cfg.address_width)
        host = torch.frombuffer(bytearray(data), dtype=torch.uint8).pin_memory()
        self.tensor = host.to(context.device, non_blocking=True)   # ordered on the current stream
        self.size = len(data)

    def ptr(self) -> int:
        return self.tensor.data_ptr()


class Canvas:
    """float4 accumulation image + per-pixel u32 RNG states (processing/src/canvas.rs:11-16)."""

    def __init__(self, context: Context, shape: Tuple[int, int], global_seed: int = 0xDEADBEEF):
        w, h = shape
        self.shape = (w, h)
        self.context = context
        self.image = torch.zeros(h * w * 4, dtype=torch.float32, device=context.device)
        # pixel_seeds(global_seed, w * h), computed on the device (ordered on the current stream)
        self.seeds = torch.empty(w * h, dtype=torch.int32, device=context.device)
        _lib.call("htc_fill_seeds", self.seeds.data_ptr(), w * h, global_seed & 0xFFFFFFFF, 0, context.stream())
        self.passes = 0

    @property
    def width(self) -> int:
        return self.shape[0]

    @property
    def height(self) -> int:
        return self.shape[1]

    def add_pass(self, n: int = 1) -> None:
        self.passes += n

    def clean(self) -> None:
        """Zero the accumulation; the seeds keep their state (canvas.rs:102-106)."""
        self.image.zero_()
        self.passes = 0


class Render:
    """The render kernel for one scene recipe and hop count (processing/src/render.rs:8-119).

    `Render.new` in the reference generates and JIT-compiles OpenCL C for the scene type;
    here the recipe selects the hand-written sm_100a kernel family.
    """

    def __init__(self, context: Context, recipe: int, hops: int, flags: int = 0):
        self.context = context
        self.recipe = recipe
        self.hops = hops
        handle = ctypes.c_void_p()
        _lib.call("htc_program_create", recipe, hops, context.config.address_width,
                  int(context.config.double_support), flags, ctypes.byref(handle))
        self.handle = handle

    @classmethod
    def build(cls, context: Context, scene_type, hops: int, flags: int = 0) -> "Render":
        """Render::new for any scene type: `scene_type` is a hypertrace_b200.types entity
        type (or its C++ type expression), compiled at run time with NVRTC
        (htc_program_build). Raises HtcError with the compiler log on failure."""
        expr = scene_type if isinstance(scene_type, str) else scene_type.cxx()
        self = cls.__new__(cls)
        self.context = context
        self.recipe = _lib.HTC_RECIPE_CUSTOM
        self.hops = hops
        handle = ctypes.c_void_p()
        log = ctypes.create_string_buffer(1 << 16)
        rc = _lib.lib().htc_program_build(expr.encode(), hops, context.config.address_width, flags, log,
                                          len(log), ctypes.byref(handle))
        self.log = log.value.decode(errors="replace")
        self.handle = handle
        _lib.check(rc)
        return self

    def static_size(self) -> int:
        v = ctypes.c_uint64()
        _lib.call("htc_program_static_size", self.handle, ctypes.byref(v))
        return v.value

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().htc_program_destroy(h)
            except Exception:
                pass
            self.handle = None

    def _check(self, sync: bool) -> None:
        if sync:
            _lib.call("htc_program_check", self.handle, self.context.stream())

    def render(self, scene_buffer: EntityBuffer, canvas: Canvas, stats: Optional[torch.Tensor] = None,
               sync: bool = True) -> None:
        """One pass, blocking like the reference (enqueue, finish, add_pass)."""
        _lib.call("htc_render_ex", self.handle, canvas.width, canvas.height, scene_buffer.ptr(),
                  scene_buffer.size, canvas.image.data_ptr(), canvas.seeds.data_ptr(),
                  None if stats is None else stats.data_ptr(), self.context.stream())
        self._check(sync)
        canvas.add_pass()

    def render_passes(self, scene_buffer: EntityBuffer, canvas: Canvas, passes: int,
                      stats: Optional[torch.Tensor] = None, sync: bool = True) -> None:
        """`passes` passes, each as wavefronts of one launch per hop depth (bit-identical to
        `passes` render calls)."""
        _lib.call("htc_render_passes", self.handle, canvas.width, canvas.height, scene_buffer.ptr(),
                  scene_buffer.size, canvas.image.data_ptr(), canvas.seeds.data_ptr(), passes,
                  None if stats is None else stats.data_ptr(), self.context.stream())
        self._check(sync)
        canvas.add_pass(passes)

    def render_wavefront(self, scene_buffer: EntityBuffer, canvas: Canvas, passes: int,
                         stats: Optional[torch.Tensor] = None, sync: bool = True) -> None:
        """`passes` passes as wavefronts, one launch per hop depth over queues of ray states
        (bit-identical to `passes` render calls)."""
        _lib.call("htc_render_wavefront", self.handle, canvas.width, canvas.height, scene_buffer.ptr(),
                  scene_buffer.size, canvas.image.data_ptr(), canvas.seeds.data_ptr(), passes,
                  None if stats is None else stats.data_ptr(), self.context.stream())
        self._check(sync)
        canvas.add_pass(passes)


class Extractor:
    """image = canvas / passes (processing/src/canvas.rs:239-287)."""

    def __init__(self, context: Context):
        self.context = context

    def process(self, canvas: Canvas, image: torch.Tensor) -> None:
        _lib.call("htc_extract", canvas.width, canvas.height, max(canvas.passes, 1),
                  canvas.image.data_ptr(), image.data_ptr(), self.context.stream())


class GammaFilter:
    """out = pow(max(in, 0), gamma) (processing/src/filter/gamma.rs:1-57)."""

    def __init__(self, context: Context, gamma: float):
        self.context = context
        self.gamma = gamma

    def process(self, width: int, height: int, inp: torch.Tensor, out: torch.Tensor) -> None:
        _lib.call("htc_gamma", width, height, ctypes.c_float(self.gamma), inp.data_ptr(),
                  out.data_ptr(), self.context.stream())


class Packer:
    """u8 = (uchar)(255 * clamp(x, 0, 1)) (processing/src/canvas.rs:289-340)."""

    def __init__(self, context: Context):
        self.context = context

    def process(self, width: int, height: int, image: torch.Tensor, packed: torch.Tensor) -> None:
        _lib.call("htc_pack", width, height, image.data_ptr(), packed.data_ptr(), self.context.stream())


class Pipeline:
    """processing::Pipeline (processing/src/pipeline.rs:8-67)."""

    def __init__(self, context: Context, canvas_size: Tuple[int, int], scene: Scene,
                 filter: Optional[GammaFilter] = None, flags: int = 0, global_seed: int = 0xDEADBEEF,
                 fused_post: bool = True):
        self.context = context
        self.scene_buffer = EntityBuffer(context, scene)
        self.render_ = Render(context, scene.recipe, scene.hops, flags)
        self.extractor = Extractor(context)
        self.packer = Packer(context)
        self.filter = filter or GammaFilter(context, 1.0 / 2.2)
        self.canvas = Canvas(context, canvas_size, global_seed)
        w, h = canvas_size
        self.image_src = torch.empty(w * h * 4, dtype=torch.float32, device=context.device)
        self.image_dst = torch.empty_like(self.image_src)
        self.packed = torch.empty(w * h * 4, dtype=torch.uint8, device=context.device)
        self.image = torch.empty(w * h * 4, dtype=torch.uint8, pin_memory=True)
        self.fused_post = fused_post

    def set_scene(self, scene: Scene) -> None:
        self.scene_buffer = EntityBuffer(self.context, scene)

    def render(self, passes: int = 1) -> None:
        if passes == 1:
            self.render_.render(self.scene_buffer, self.canvas)
        else:
            self.render_.render_passes(self.scene_buffer, self.canvas, passes)

    def get_image(self) -> np.ndarray:
        """Extract, gamma, pack, then a blocking device-to-host read (pipeline.rs:53-62)."""
        w, h = self.canvas.shape
        if self.fused_post:
            _lib.call("htc_extract_gamma_pack", w, h, max(self.canvas.passes, 1),
                      ctypes.c_float(self.filter.gamma), self.canvas.image.data_ptr(),
                      self.packed.data_ptr(), self.context.stream())
        else:
            self.extractor.process(self.canvas, self.image_src)
            self.filter.process(w, h, self.image_src, self.image_dst)
            self.packer.process(w, h, self.image_dst, self.packed)
        self.image.copy_(self.packed, non_blocking=True)
        torch.cuda.current_stream(self.context.device).synchronize()
        return self.image.numpy().reshape(h, w, 4)

    def clean(self) -> None:
        self.canvas.clean()
