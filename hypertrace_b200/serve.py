"""Continuous-batching render server.

Requests arrive over time (Poisson). Admitted requests keep their canvas, RNG seeds and
scene on the device until they finish; every step is ONE batched render (htc_batch_*: a
launch per pass, hop depth and recipe, each over every view of the step) over the admitted
requests, so requests that arrive while others render join the next step and their work
overlaps on the GPU. Two classes: interactive frames (all their passes in the next step,
admitted first) and batch jobs (a quantum of passes per step). Admission is bounded by an
HBM budget (what does not fit waits on the host) and allocates at most a few requests per
loop turn, so that a burst of arrivals does not hold the next step back.

Results are bit-identical to rendering each request alone (each pixel keeps its RNG stream
and sample order), which tests/test_gpu_serve.py checks in a mixed run.

`plain_fifo()` is the comparison: one request at a time, each pass a launch of the plain
one-pass kernel (the shape of the reference's Pipeline loop).
"""
from __future__ import annotations

import collections
import dataclasses
import time
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from . import scene as S
from .batch import BatchRenderer, View, config3
from .processing import Context, Render

INTERACTIVE = 0
BATCH = 1


@dataclasses.dataclass
class Request:
    rid: int
    kind: int
    arrival: float                 # seconds after the start of the run
    view: View
    quantum: int = 16              # passes per step for batch jobs
    admitted: float = -1.0
    finished: float = -1.0
    refused: bool = False           # larger than the whole HBM budget
    image: Optional[np.ndarray] = None

    @property
    def samples(self) -> int:
        return self.view.width * self.view.height * self.view.spp


def geodesic_step(rng: np.random.Generator, length: float) -> np.ndarray:
    """A random camera step of hyperbolic length `length`: the controller's
    `map.chain(step)` (viewer/src/controllers/isotropic.rs:21-24) with a random direction."""
    phi, theta = rng.uniform(0, 2 * np.pi), rng.uniform(0, np.pi)
    look = S.mo_chain(S.mo_zrotate(phi), S.mo_yrotate(theta))
    inv = np.linalg.inv(look)
    return S.mo_normalize(S.mo_chain(look, S.mo_chain(S.mo_zshift(length), inv)))


def make_requests(n: int, rate: float, seed: int = 0x5EED0004, interactive_share: float = 0.7,
                  batch_spp_scale: float = 0.125, n_sessions: int = 8) -> List[Request]:
    """Poisson arrivals at `rate` req/s. Interactive: 1280x720, 8 spp, hyperbolic scene of a
    session (20-200 objects) whose camera advances by a random geodesic step each frame.
    Batch: a view drawn as in the mixed batched workload (spp scaled by batch_spp_scale)."""
    rng = np.random.default_rng(seed)
    sessions = []
    for k in range(n_sessions):
        nobj = int(rng.integers(20, 201))
        nh = int(round(0.6 * nobj))
        sessions.append([S.hyperbolic_scene(nobj - nh, nh, 6.0, 8, seed + 31 * k), S.mo_identity()])
    pool = config3(seed + 1, n_views=64, spp_scale=batch_spp_scale)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        if rng.random() < interactive_share:
            sess = sessions[int(rng.integers(n_sessions))]
            sess[1] = S.mo_chain(sess[1], geodesic_step(rng, 0.05))
            sc = dataclasses.replace(sess[0], camera=sess[1].copy())
            view = View(sc, 1280, 720, 8, int(rng.integers(1 << 31)))
            out.append(Request(i, INTERACTIVE, t, view))
        else:
            v = pool[int(rng.integers(len(pool)))]
            view = View(v.scene, v.width, v.height, v.spp, int(rng.integers(1 << 31)))
            out.append(Request(i, BATCH, t, view))
    return out


class Server:
    """Continuous batching over the htc_batch launch."""

    def __init__(self, ctx: Context, hbm_budget_bytes: int = 120 << 30, tile_pixels: int = 512,
                 blocks_per_sm: int = 0, gamma: float = 1.0 / 2.2, step_samples: int = 16_000_000):
        self.ctx = ctx
        self.budget = hbm_budget_bytes
        self.step_samples = step_samples    # work of one step: bounds the wait of a new arrival
        self.renderer = BatchRenderer(ctx, max_views=4096)
        # queues for the largest step (its views cover at most step_samples pixels, plus one
        # oversized job), so that set_views never has to grow them mid-run
        self.renderer.reserve(min(step_samples + 1920 * 1080, hbm_budget_bytes // 136), 8)
        self.admit_per_step = 4             # allocations per loop turn: spreads the host work
        self.tile_pixels = tile_pixels
        self.blocks_per_sm = blocks_per_sm
        self.gamma = gamma
        self.steps = 0
        self.device_s = 0.0
        self._step_events = []

    def _enqueue_finish(self, r: Request, keep_image: bool) -> dict:
        """Post chain + read-back of a finished request, enqueued on the stream (no wait)."""
        v = r.view
        w, h = v.width, v.height
        packed = torch.empty(w * h * 4, dtype=torch.uint8, device=self.ctx.device)
        _lib.call("htc_extract_gamma_pack", w, h, v.spp, _lib.ctypes.c_float(self.gamma),
                  v.canvas.image.data_ptr(), packed.data_ptr(), self.ctx.stream())
        out = {"image": torch.empty(w * h * 4, dtype=torch.uint8, pin_memory=True)}
        out["image"].copy_(packed, non_blocking=True)
        if keep_image:
            out["canvas"] = torch.empty(w * h * 4, dtype=torch.float32, pin_memory=True)
            out["canvas"].copy_(v.canvas.image, non_blocking=True)
            out["seeds"] = torch.empty(w * h, dtype=torch.int32, pin_memory=True)
            out["seeds"].copy_(v.canvas.seeds, non_blocking=True)
        v.release()   # stream-ordered reuse: the caching allocator hands the blocks out later
        return out

    def _retire(self, step, t0: float, keep_images: bool) -> int:
        event, finishing = step
        event.synchronize()
        t = time.perf_counter() - t0
        for r, out in finishing:
            r.finished = t
            w, h = r.view.width, r.view.height
            if keep_images:
                r.image = out["image"].numpy().reshape(h, w, 4)
                r.canvas = out["canvas"].numpy().reshape(h, w, 4)   # type: ignore[attr-defined]
                r.seeds = out["seeds"].numpy().view(np.uint32).reshape(h, w)   # type: ignore[attr-defined]
        return len(finishing)

    def _plan(self, active: Sequence[Request]):
        """Work of the next step, at most `step_samples` samples (always at least one job):
        interactive frames first, whole, in arrival order; then batch jobs in arrival order,
        each up to its quantum of passes, with whatever budget is left."""
        plan, budget = [], self.step_samples
        for r in sorted((r for r in active if r.kind == INTERACTIVE), key=lambda r: r.arrival):
            cost = r.view.width * r.view.height * r.view.remaining
            if cost <= budget or not plan:
                plan.append((r, r.view.remaining))
                budget -= cost
        for r in sorted((r for r in active if r.kind == BATCH), key=lambda r: r.arrival):
            px = r.view.width * r.view.height
            p = min(r.quantum, r.view.remaining, budget // px if px else 0)
            if p <= 0 and not plan:
                p = 1
            if p > 0:
                plan.append((r, p))
                budget -= p * px
        return plan

    def run(self, requests: Sequence[Request], keep_images: bool = False, depth: int = 2) -> Dict[str, object]:
        """Serve `requests` in real time (arrival times relative to the call).

        Steps are planned on the host from the state the already-enqueued steps will leave
        (which requests a step finishes is known when it is enqueued), so up to `depth` steps
        are in flight and the host's planning, admission and read-back overlap the GPU."""
        arrivals = sorted(requests, key=lambda r: r.arrival)
        ai = 0
        waiting = collections.deque()          # arrived, not yet admitted (FIFO per class)
        waiting_i = collections.deque()
        active: List[Request] = []
        inflight = collections.deque()
        used = 0
        t0 = time.perf_counter()
        stream = torch.cuda.current_stream(self.ctx.device)
        done = 0
        while done < len(arrivals):
            now = time.perf_counter() - t0
            while ai < len(arrivals) and arrivals[ai].arrival <= now:
                (waiting_i if arrivals[ai].kind == INTERACTIVE else waiting).append(arrivals[ai])
                ai += 1
            # admission: interactive first, then batch jobs, while the HBM budget allows;
            # a request larger than the whole budget can never run and is refused
            admits = 0
            for q in (waiting_i, waiting):
                while q and q[0].view.device_bytes() > self.budget:
                    r = q.popleft()
                    r.refused = True
                    done += 1
                while q and admits < self.admit_per_step and used + q[0].view.device_bytes() <= self.budget:
                    r = q.popleft()
                    r.view.allocate(self.ctx)
                    admits += 1
                    r.admitted = time.perf_counter() - t0
                    used += r.view.device_bytes()
                    active.append(r)
            while inflight and inflight[0][0].query():
                done += self._retire(inflight.popleft(), t0, keep_images)
            if not active:
                if inflight:
                    done += self._retire(inflight.popleft(), t0, keep_images)
                elif ai < len(arrivals):
                    time.sleep(max(0.0, min(arrivals[ai].arrival - now, 0.005)))
                continue
            if len(inflight) >= depth:
                done += self._retire(inflight.popleft(), t0, keep_images)
                continue
            plan = self._plan(active)
            self.renderer.set_views([r.view for r, _ in plan], [p for _, p in plan],
                                    tile_pixels=self.tile_pixels, blocks_per_sm=self.blocks_per_sm)
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            self.renderer.render()
            e1 = torch.cuda.Event(enable_timing=True)
            e1.record(stream)
            self._step_events.append((e0, e1))
            self.steps += 1
            for r, p in plan:
                r.view.done_passes += p
            finishing, still = [], []
            for r in active:
                if r.view.remaining == 0:
                    used -= r.view.device_bytes()
                    finishing.append((r, self._enqueue_finish(r, keep_images)))
                else:
                    still.append(r)
            active = still
            ev = torch.cuda.Event()
            ev.record(stream)
            inflight.append((ev, finishing))
        while inflight:
            done += self._retire(inflight.popleft(), t0, keep_images)
        torch.cuda.synchronize()
        self.device_s = sum(a.elapsed_time(b) for a, b in self._step_events) * 1e-3
        self.renderer.check()
        return summarize(arrivals, time.perf_counter() - t0, self.device_s, self.steps)


def plain_fifo(ctx: Context, requests: Sequence[Request], gamma: float = 1.0 / 2.2) -> Dict[str, object]:
    """One request at a time in arrival order; each pass one launch of the plain kernel."""
    arrivals = sorted(requests, key=lambda r: r.arrival)
    renders: Dict[tuple, Render] = {}
    t0 = time.perf_counter()
    dev_s = 0.0
    stream = torch.cuda.current_stream(ctx.device)
    for r in arrivals:
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        v = r.view
        v.allocate(ctx)
        r.admitted = time.perf_counter() - t0
        key = (v.scene.recipe, v.scene.hops)
        if key not in renders:
            renders[key] = Render(ctx, *key)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(v.spp):
            renders[key].render(v.buffer, v.canvas, sync=False)
        e1.record(stream)
        packed = torch.empty(v.width * v.height * 4, dtype=torch.uint8, device=ctx.device)
        _lib.call("htc_extract_gamma_pack", v.width, v.height, v.spp, _lib.ctypes.c_float(gamma),
                  v.canvas.image.data_ptr(), packed.data_ptr(), ctx.stream())
        packed.cpu()
        dev_s += e0.elapsed_time(e1) * 1e-3
        r.finished = time.perf_counter() - t0
        v.release()
    return summarize(arrivals, time.perf_counter() - t0, dev_s, len(arrivals))


def summarize(reqs: Sequence[Request], wall_s: float, device_s: float, steps: int) -> Dict[str, object]:
    refused = sum(r.refused for r in reqs)
    reqs = [r for r in reqs if not r.refused]
    out: Dict[str, object] = {"requests": len(reqs), "refused": refused, "wall_s": wall_s, "device_s": device_s,
                              "steps": steps}
    total = sum(r.samples for r in reqs)
    out["throughput_msamples_per_s"] = total / wall_s / 1e6
    out["throughput_req_per_s"] = len(reqs) / wall_s
    for kind, name in ((INTERACTIVE, "interactive"), (BATCH, "batch")):
        lat = np.array([r.finished - r.arrival for r in reqs if r.kind == kind])
        if len(lat):
            out[name] = {"count": int(len(lat)), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                         "p99_ms": float(np.percentile(lat, 99) * 1e3)}
    lat = np.array([r.finished - r.arrival for r in reqs])
    out["all"] = {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3)}
    return out
