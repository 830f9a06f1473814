"""Serving: requests rendered while others are on the GPU (continuous batching) give the
same result as each request rendered alone, bit for bit; admission respects the budget."""
import numpy as np
import pytest
import torch

from hypertrace_b200 import batch as B
from hypertrace_b200 import processing as P
from hypertrace_b200 import scene as S
from hypertrace_b200 import serve as V

pytestmark = pytest.mark.gpu


def _requests(n=12, rate=400.0, seed=9):
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        if i % 3 == 2:
            sc = S.euclidean_scene(int(rng.integers(2, 9)), 4, 50 + i, camera=B.random_hom3(rng))
            out.append(V.Request(i, V.BATCH, t, B.View(sc, 80, 60, 32, 500 + i), quantum=8))
        else:
            sc = S.hyperbolic_scene(int(rng.integers(3, 20)), int(rng.integers(3, 30)), 5.0, 8, 70 + i,
                                    camera=S.random_moebius(rng, 1.0))
            out.append(V.Request(i, V.INTERACTIVE, t, B.View(sc, 96, 54, 8, 600 + i)))
    return out


@pytest.mark.parametrize("budget", [120 << 30, 2_000_000])
def test_served_equals_alone(built, budget):
    ctx = P.Context(0)
    reqs = _requests()
    srv = V.Server(ctx, hbm_budget_bytes=budget, tile_pixels=512)
    res = srv.run(reqs, keep_images=True)
    assert res["requests"] == len(reqs) and srv.steps >= 2
    for r in _requests():
        v = r.view
        v.allocate(ctx)
        P.Render(ctx, v.scene.recipe, v.scene.hops).render_passes(v.buffer, v.canvas, v.spp)
        torch.cuda.synchronize()
        served = next(q for q in reqs if q.rid == r.rid)
        assert np.array_equal(served.seeds, v.canvas.seeds.cpu().numpy().view(np.uint32).reshape(v.height, v.width))
        assert np.array_equal(served.canvas.view(np.uint32),
                              v.canvas.image.cpu().numpy().reshape(v.height, v.width, 4).view(np.uint32))
        assert served.finished >= served.arrival


def test_oversized_request_is_refused_and_memory_returns(built):
    """A request needing more device memory than the whole budget is refused at submission
    (HTC_ERR_BUDGET); the others are served and the budget's bytes all come back."""
    from hypertrace_b200 import _lib
    import ctypes
    ctx = P.Context(0)
    reqs = _requests(n=5)
    sc = S.hyperbolic_scene(3, 3, 5.0, 8, 1)
    reqs.append(V.Request(99, V.INTERACTIVE, 0.0, B.View(sc, 1280, 720, 8, 7)))   # 1280x720 x 160 B > 2 MB
    srv = V.Server(ctx, hbm_budget_bytes=2_000_000, tile_pixels=512)
    res = srv.run(reqs)
    assert res["refused"] == 1 and res["requests"] == 5
    assert next(r for r in reqs if r.rid == 99).refused
    info = _lib.HtcServerInfo()
    _lib.call("htc_server_stats", srv.handle, ctypes.byref(info))
    assert info.used_bytes == 0 and info.active == 0 and info.waiting == 0 and info.in_flight == 0


def test_plain_fifo_runs(built):
    ctx = P.Context(0)
    reqs = _requests(n=4)
    res = V.plain_fifo(ctx, reqs)
    assert res["requests"] == 4 and res["all"]["p99_ms"] > 0
