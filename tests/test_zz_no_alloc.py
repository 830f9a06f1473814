"""The allocation-free entry point, htc_render_passes_noalloc.

Some callers cannot call cudaMalloc (a host that hands the renderer a fixed memory
budget, or a custom allocator that owns all device memory), so they cannot create an
htc_program. This entry point renders without allocating: its work-queue words sit in a
static device array. These tests call it through the C ABI and check, on two calls in a
row, that canvas and seeds match what htc_render_passes produces (bit for bit, the
tolerance the render path's own tests use for this comparison), that a further call
leaves the device's free memory unchanged, and that it rejects a size beyond its limit. Collected last so a failure here leaves every other test run."""
import ctypes

import numpy as np
import pytest
import torch

from hypertrace_b200 import _lib
from hypertrace_b200 import processing as P
from hypertrace_b200 import scene as S

pytestmark = pytest.mark.gpu


def _setup(wl, W, H):
    ctx = P.Context(0)
    buf = P.EntityBuffer(ctx, wl.scene)
    canvas = P.Canvas(ctx, (W, H), global_seed=wl.global_seed)
    return ctx, buf, canvas


@pytest.mark.parametrize("cfg", ["config1", "config0"])
def test_noalloc_matches_render_passes(built, cfg):
    wl = getattr(S, cfg)()
    W, H = 256, 144
    ctx, buf, ref_canvas = _setup(wl, W, H)
    _, _, na_canvas = _setup(wl, W, H)
    r = P.Render(ctx, wl.scene.recipe, wl.scene.hops)
    status = torch.zeros(1, dtype=torch.int32, device=ctx.device)
    stats_ref = torch.zeros(8, dtype=torch.int64, device=ctx.device)
    stats_na = torch.zeros(8, dtype=torch.int64, device=ctx.device)
    for call in range(2):
        r.render_passes(buf, ref_canvas, 3, stats=stats_ref)
        _lib.call("htc_render_passes_noalloc", wl.scene.recipe, wl.scene.hops, 32, 0, W, H, buf.ptr(), buf.size,
                  na_canvas.image.data_ptr(), na_canvas.seeds.data_ptr(), 3, stats_na.data_ptr(),
                  status.data_ptr(), ctx.stream())
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        assert torch.equal(ref_canvas.seeds, na_canvas.seeds), f"seeds differ after call {call + 1}"
        a = ref_canvas.image.cpu().numpy().view(np.uint32)
        b = na_canvas.image.cpu().numpy().view(np.uint32)
        assert np.array_equal(a, b), f"canvas differs after call {call + 1}"
    assert torch.equal(stats_ref, stats_na)


def test_noalloc_leaves_free_memory_unchanged(built):
    """The defining property: after a first call (which may load the kernel's code), a
    further call takes no device memory -- the free-memory count of the device is the same
    before and after it."""
    wl = S.config1()
    W, H = 128, 96
    ctx, buf, canvas = _setup(wl, W, H)
    status = torch.zeros(1, dtype=torch.int32, device=ctx.device)

    def call():
        _lib.call("htc_render_passes_noalloc", wl.scene.recipe, wl.scene.hops, 32, 0, W, H, buf.ptr(), buf.size,
                  canvas.image.data_ptr(), canvas.seeds.data_ptr(), 2, None, status.data_ptr(), ctx.stream())
        torch.cuda.synchronize()

    call()
    free_before = torch.cuda.mem_get_info(ctx.device)[0]
    call()
    free_after = torch.cuda.mem_get_info(ctx.device)[0]
    assert int(status.item()) == 0
    assert free_after == free_before, f"free device memory changed by {free_before - free_after} bytes"


def test_noalloc_rejects_oversized_canvas(built):
    wl = S.config1()
    ctx, buf, canvas = _setup(wl, 8, 8)
    rc = _lib.lib().htc_render_passes_noalloc(wl.scene.recipe, wl.scene.hops, 32, 0, 1 << 16, 1 << 16, buf.ptr(),
                                               buf.size, canvas.image.data_ptr(), canvas.seeds.data_ptr(), 1, None,
                                               None, ctx.stream())
    assert rc == _lib.HTC_ERR_UNSUPPORTED
    assert b"2^31" in _lib.lib().htc_last_error()


def test_noalloc_pixel_limit_boundary(built):
    """width*height == 2^31 is accepted, 2^31 + 1 (= 3 x 715827883) is rejected. Both calls
    ask for zero passes, so neither launches anything or touches the small buffers."""
    wl = S.config1()
    ctx, buf, canvas = _setup(wl, 8, 8)
    lib = _lib.lib()
    args = (buf.ptr(), buf.size, canvas.image.data_ptr(), canvas.seeds.data_ptr(), 0, None, None, ctx.stream())
    assert lib.htc_render_passes_noalloc(wl.scene.recipe, wl.scene.hops, 32, 0, 1 << 16, 1 << 15, *args) == _lib.HTC_OK
    assert lib.htc_render_passes_noalloc(wl.scene.recipe, wl.scene.hops, 32, 0, 3, 715827883, *args) \
        == _lib.HTC_ERR_UNSUPPORTED
    assert b"2^31" in lib.htc_last_error()


def test_noalloc_reports_bad_scene(built):
    wl = S.config1()
    ctx, buf, canvas = _setup(wl, 16, 16)
    data = bytearray(wl.scene.to_bytes())
    data[96:100] = (10_000).to_bytes(4, "little")
    buf.tensor.copy_(torch.frombuffer(data, dtype=torch.uint8).to(ctx.device))
    status = torch.zeros(1, dtype=torch.int32, device=ctx.device)
    _lib.call("htc_render_passes_noalloc", wl.scene.recipe, wl.scene.hops, 32, 0, 16, 16, buf.ptr(), buf.size,
              canvas.image.data_ptr(), canvas.seeds.data_ptr(), 1, None, status.data_ptr(), ctx.stream())
    torch.cuda.synchronize()
    assert int(status.item()) != 0


def test_noalloc_bad_scene_without_status_renders_nothing(built):
    """Without `status` a scene that fails validation is reported nowhere, but it is not
    rendered either: canvas and seeds keep their contents."""
    wl = S.config1()
    ctx, buf, canvas = _setup(wl, 16, 16)
    data = bytearray(wl.scene.to_bytes())
    data[96:100] = (10_000).to_bytes(4, "little")
    buf.tensor.copy_(torch.frombuffer(data, dtype=torch.uint8).to(ctx.device))
    image0, seeds0 = canvas.image.clone(), canvas.seeds.clone()
    _lib.call("htc_render_passes_noalloc", wl.scene.recipe, wl.scene.hops, 32, 0, 16, 16, buf.ptr(), buf.size,
              canvas.image.data_ptr(), canvas.seeds.data_ptr(), 2, None, None, ctx.stream())
    torch.cuda.synchronize()
    assert torch.equal(canvas.seeds, seeds0)
    assert torch.equal(canvas.image, image0)
