"""Host logic of the continuous-batching server, on the CPU: the step planner
(htc_serve_plan through the C ABI: interactive frames first and whole, batch jobs by quantum
within the step's sample budget), argument checks of the server entry points, and the
request stream generator. No GPU: the planner only reads sizes and pass counts."""
import ctypes

from hypertrace_b200 import _lib
from hypertrace_b200 import serve as V

I, B = _lib.HTC_PRIORITY_INTERACTIVE, _lib.HTC_PRIORITY_BATCH


def test_interactive_first_and_whole():
    # (pixels, remaining passes, quantum, priority) in arrival order: a batch job, then two frames
    items = [(100, 32, 8, B), (100, 8, 8, I), (100, 8, 8, I)]
    # both frames whole (800 samples each), the batch job gets what is left: 400 samples = 4 passes
    assert V.Server.plan(items, 2000) == [4, 8, 8]
    # a frame that no longer fits waits for the next step; the batch job takes the rest
    assert V.Server.plan(items, 1000) == [2, 8, 0]


def test_batch_jobs_fill_the_budget_by_quantum():
    items = [(100, 64, 8, B), (100, 64, 8, B), (100, 64, 8, B)]
    plan = V.Server.plan(items, 2000)
    assert plan == [8, 8, 4]
    assert sum(px * p for (px, _, _, _), p in zip(items, plan)) <= 2000


def test_quantum_capped_by_remaining_passes():
    assert V.Server.plan([(100, 3, 8, B)], 10_000) == [3]


def test_oversized_work_still_makes_progress():
    # a frame larger than the whole step budget runs alone; a batch job gets one pass
    assert V.Server.plan([(400, 8, 8, I), (400, 8, 8, B)], 100) == [8, 0]
    assert V.Server.plan([(400, 8, 8, B)], 100) == [1]


def test_finished_items_get_nothing():
    assert V.Server.plan([(100, 0, 8, I), (100, 0, 8, B), (100, 2, 8, B)], 10_000) == [0, 0, 2]


def test_step_pixels_bounded_for_the_queue_reservation():
    """A step's views cover at most step_samples pixels plus one oversized view: the bound
    the server reserves its wavefront queues for."""
    import numpy as np
    rng = np.random.default_rng(5)
    items = [(int(rng.integers(8, 90)) * int(rng.integers(8, 90)), 8, 8, I if rng.random() < 0.7 else B)
             for _ in range(40)]
    plan = V.Server.plan(items, 16_000)
    pixels = [px for (px, _, _, _), p in zip(items, plan) if p]
    assert sum(pixels) <= 16_000 + max(pixels)


def test_server_entry_points_reject_bad_arguments_without_device():
    lib = _lib.lib()
    h = ctypes.c_void_p()
    assert lib.htc_server_create(0, 1000, 8, ctypes.byref(h)) == _lib.HTC_ERR_INVALID
    n = ctypes.c_uint32()
    assert lib.htc_server_step(None, None, None) == _lib.HTC_ERR_INVALID
    assert lib.htc_server_poll(None, None, 0, ctypes.byref(n), 0) == _lib.HTC_ERR_INVALID
    rid = ctypes.c_uint64()
    assert lib.htc_server_submit(None, None, ctypes.byref(rid)) == _lib.HTC_ERR_INVALID
    out = (ctypes.c_uint32 * 1)()
    assert lib.htc_serve_plan(None, 1, 100, ctypes.cast(out, ctypes.c_void_p)) == _lib.HTC_ERR_INVALID


def test_request_stream():
    reqs = V.make_requests(50, 100.0, seed=3)
    arrivals = [r.arrival for r in reqs]
    assert arrivals == sorted(arrivals) and len(reqs) == 50
    kinds = {r.kind for r in reqs}
    assert kinds == {V.INTERACTIVE, V.BATCH}
    for r in reqs:
        if r.kind == V.INTERACTIVE:
            assert (r.view.width, r.view.height, r.view.spp) == (1280, 720, 8)
