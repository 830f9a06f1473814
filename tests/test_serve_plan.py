"""Host logic of the continuous-batching server, on the CPU: step planning (interactive frames
first and whole, batch jobs by quantum within the step's sample budget) and the request
stream generator. No GPU: the planner only reads view sizes and pass counts."""
import numpy as np

from hypertrace_b200 import batch as B
from hypertrace_b200 import scene as S
from hypertrace_b200 import serve as V


def _server(step_samples):
    srv = object.__new__(V.Server)   # the planner needs no device state
    srv.step_samples = step_samples
    return srv


def _req(rid, kind, arrival, w, h, spp, done=0, quantum=8):
    v = B.View(S.euclidean_scene(2, 4, rid), w, h, spp, rid)
    v.done_passes = done
    return V.Request(rid, kind, arrival, v, quantum=quantum)


def test_interactive_first_and_whole():
    srv = _server(2000)
    reqs = [_req(0, V.BATCH, 0.0, 10, 10, 32), _req(1, V.INTERACTIVE, 0.5, 10, 10, 8),
            _req(2, V.INTERACTIVE, 0.1, 10, 10, 8)]
    plan = srv._plan(reqs)
    # interactive frames in arrival order, all their passes; then the batch job with what is left
    assert [(r.rid, p) for r, p in plan] == [(2, 8), (1, 8), (0, 4)]
    # a frame that no longer fits waits for the next step; the batch job takes the rest
    srv = _server(1000)
    assert [(r.rid, p) for r, p in srv._plan(reqs)] == [(2, 8), (0, 2)]


def test_batch_jobs_fill_the_budget_by_quantum():
    srv = _server(2000)
    reqs = [_req(0, V.BATCH, 0.0, 10, 10, 64, quantum=8), _req(1, V.BATCH, 0.1, 10, 10, 64, quantum=8),
            _req(2, V.BATCH, 0.2, 10, 10, 64, quantum=8)]
    plan = srv._plan(reqs)
    assert [(r.rid, p) for r, p in plan] == [(0, 8), (1, 8), (2, 4)]
    assert sum(r.view.width * r.view.height * p for r, p in plan) <= 2000


def test_quantum_capped_by_remaining_passes():
    srv = _server(10_000)
    plan = srv._plan([_req(0, V.BATCH, 0.0, 10, 10, 64, done=61, quantum=8)])
    assert [(r.rid, p) for r, p in plan] == [(0, 3)]


def test_oversized_work_still_makes_progress():
    srv = _server(100)
    # a frame larger than the whole step budget runs alone; a batch job gets one pass
    plan = srv._plan([_req(0, V.INTERACTIVE, 0.0, 20, 20, 8), _req(1, V.BATCH, 0.0, 20, 20, 8)])
    assert [(r.rid, p) for r, p in plan] == [(0, 8)]
    plan = srv._plan([_req(1, V.BATCH, 0.0, 20, 20, 8)])
    assert [(r.rid, p) for r, p in plan] == [(1, 1)]


def test_step_pixels_bounded_for_the_queue_reservation():
    """A step's views cover at most step_samples pixels plus one oversized view: the bound
    the server reserves its wavefront queues for."""
    srv = _server(16_000)
    rng = np.random.default_rng(5)
    reqs = [_req(i, V.INTERACTIVE if rng.random() < 0.7 else V.BATCH, float(i), int(rng.integers(8, 90)),
                 int(rng.integers(8, 90)), 8) for i in range(40)]
    plan = srv._plan(reqs)
    pixels = [r.view.width * r.view.height for r, _ in plan]
    assert sum(pixels) <= srv.step_samples + max(pixels)


def test_request_stream():
    reqs = V.make_requests(50, 100.0, seed=3)
    arrivals = [r.arrival for r in reqs]
    assert arrivals == sorted(arrivals) and len(reqs) == 50
    kinds = {r.kind for r in reqs}
    assert kinds == {V.INTERACTIVE, V.BATCH}
    for r in reqs:
        if r.kind == V.INTERACTIVE:
            assert (r.view.width, r.view.height, r.view.spp) == (1280, 720, 8)
