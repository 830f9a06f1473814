"""Continuous-batching render server.

Requests arrive over time (Poisson). Admitted requests keep their canvas, RNG seeds and
scene on the device until they finish; every step is ONE batched render (htc_batch_*: a
launch per pass, hop depth and recipe, each over every view of the step) over the admitted
requests, so requests that arrive while others render join the next step and their work
overlaps on the GPU. Two classes: interactive frames (all their passes in the next step,
admitted first) and batch jobs (a quantum of passes per step). Admission is bounded by an
HBM budget (what does not fit waits on the host; device memory comes from a stream-ordered
pool, so admitting never synchronises the device). The server itself -- admission,
planning, the step's view table, read-back and release -- is native (htc_server_*,
hypertrace_b200/csrc/htserve.cu); `Server` drives it from a Python loop of one submit per
arrival, one step and one poll per turn.

Results are bit-identical to rendering each request alone (each pixel keeps its RNG stream
and sample order), which tests/test_gpu_serve.py checks in a mixed run.

`plain_fifo()` is the comparison: one request at a time, each pass a launch of the plain
one-pass kernel (the shape of the reference's Pipeline loop).
"""
from __future__ import annotations

import collections
import ctypes
import dataclasses
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from . import scene as S
from .batch import View, config3
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
    """Continuous batching through the native server (htc_server_*, include/htcuda.h).

    The Python loop only hands arrivals to htc_server_submit, calls htc_server_step (which
    admits by the HBM budget, plans, renders one batched step and enqueues the read-back of
    what it completes, with up to `depth` steps in flight) and collects finished requests
    with htc_server_poll."""

    def __init__(self, ctx: Context, hbm_budget_bytes: int = 120 << 30, tile_pixels: int = 512,
                 blocks_per_sm: int = 0, gamma: float = 1.0 / 2.2, step_samples: int = 16_000_000,
                 depth: int = 2, admit_per_step: int = 8, max_views: int = 4096):
        self.ctx = ctx
        self.budget = hbm_budget_bytes
        self.step_samples = step_samples
        self.tile_pixels = tile_pixels
        self.gamma = gamma
        self.steps = 0
        self.device_s = 0.0
        self.feed = 32              # requests handed to the native server ahead of admission
        self._pinned = {}           # pinned host buffers by (size, dtype), reused across requests
        h = ctypes.c_void_p()
        _lib.call("htc_server_create", hbm_budget_bytes, step_samples, max_views, ctypes.byref(h))
        self.handle = h
        # queues for the largest step (its views cover at most step_samples pixels, plus one
        # oversized job), so that no step has to grow them
        _lib.call("htc_server_configure", h, depth, tile_pixels, admit_per_step,
                  min(step_samples + 1920 * 1080, hbm_budget_bytes // 136), ctx.stream())

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().htc_server_destroy(h)
            except Exception:
                pass
            self.handle = None

    def _buffer(self, n: int, dtype) -> torch.Tensor:
        free = self._pinned.get((n, dtype))
        return free.pop() if free else torch.empty(n, dtype=dtype, pin_memory=True)

    def _release(self, out: Dict[str, torch.Tensor]) -> None:
        for t in out.values():
            self._pinned.setdefault((t.numel(), t.dtype), []).append(t)

    def _submit(self, r: Request, keep_images: bool) -> int:
        v = r.view
        data = v.scene.to_bytes()
        w, h = v.width, v.height
        r._scene = np.frombuffer(data, dtype=np.uint8).copy()   # type: ignore[attr-defined]
        r._out = {"image": self._buffer(w * h * 4, torch.uint8)}   # type: ignore[attr-defined]
        if keep_images:
            r._out["canvas"] = self._buffer(w * h * 4, torch.float32)
            r._out["seeds"] = self._buffer(w * h, torch.int32)
        req = _lib.HtcRequest(r._scene.ctypes.data, len(data), w, h, v.scene.recipe, v.scene.hops, v.flags, 32,
                              v.spp, v.global_seed & 0xFFFFFFFF,
                              _lib.HTC_PRIORITY_INTERACTIVE if r.kind == INTERACTIVE else _lib.HTC_PRIORITY_BATCH,
                              r.quantum, self.gamma, 0, r._out["image"].data_ptr(),
                              r._out["canvas"].data_ptr() if keep_images else None,
                              r._out["seeds"].data_ptr() if keep_images else None)
        rid = ctypes.c_uint64()
        rc = _lib.lib().htc_server_submit(self.handle, ctypes.byref(req), ctypes.byref(rid))
        if rc == _lib.HTC_ERR_BUDGET:
            r.refused = True
            return 0
        _lib.check(rc)
        return rid.value

    def run(self, requests: Sequence[Request], keep_images: bool = False) -> Dict[str, object]:
        """Serve `requests` in real time (arrival times relative to the call). Arrivals wait
        in two host queues (interactive first) and are handed to the native server while it
        holds fewer than `feed` requests not yet admitted, so that a burst of arrivals costs
        one loop turn a few submissions at a time."""
        arrivals = sorted(requests, key=lambda r: r.arrival)
        ai, done = 0, 0
        pending = {INTERACTIVE: collections.deque(), BATCH: collections.deque()}
        by_id: Dict[int, Request] = {}
        ids = (ctypes.c_uint64 * 256)()
        n = ctypes.c_uint32()
        rendered = ctypes.c_uint32()
        info = _lib.HtcServerInfo()
        stream = torch.cuda.current_stream(self.ctx.device)
        step_events = []
        t0 = time.perf_counter()
        while done < len(arrivals):
            now = time.perf_counter() - t0
            while ai < len(arrivals) and arrivals[ai].arrival <= now:
                pending[arrivals[ai].kind].append(arrivals[ai])
                ai += 1
            _lib.call("htc_server_stats", self.handle, ctypes.byref(info))
            room = self.feed - info.waiting
            for q in (pending[INTERACTIVE], pending[BATCH]):
                while q and room > 0:
                    r = q.popleft()
                    rid = self._submit(r, keep_images)
                    if rid:
                        by_id[rid] = r
                        room -= 1
                    else:
                        done += 1
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _lib.call("htc_server_step", self.handle, self.ctx.stream(), ctypes.byref(rendered))
            if rendered.value:
                e1 = torch.cuda.Event(enable_timing=True)
                e1.record(stream)
                step_events.append((e0, e1))
                self.steps += 1
            _lib.call("htc_server_poll", self.handle, ids, len(ids), ctypes.byref(n), 0)
            t = time.perf_counter() - t0
            for i in range(n.value):
                r = by_id.pop(ids[i])
                r.finished = t
                done += 1
                if keep_images:
                    w, h = r.view.width, r.view.height
                    r.image = r._out["image"].numpy().reshape(h, w, 4).copy()
                    r.canvas = r._out["canvas"].numpy().reshape(h, w, 4).copy()   # type: ignore[attr-defined]
                    r.seeds = r._out["seeds"].numpy().view(np.uint32).reshape(h, w).copy()   # type: ignore[attr-defined]
                self._release(r._out)   # type: ignore[attr-defined]
                r._out = None   # type: ignore[attr-defined]
            if not rendered.value:
                _lib.call("htc_server_stats", self.handle, ctypes.byref(info))
                idle = not pending[INTERACTIVE] and not pending[BATCH]
                if idle and info.in_flight == 0 and info.active == 0 and info.waiting == 0 and ai < len(arrivals):
                    time.sleep(max(0.0, min(arrivals[ai].arrival - (time.perf_counter() - t0), 0.005)))
                elif info.in_flight:
                    time.sleep(0.0002)
        torch.cuda.synchronize()
        self.device_s = sum(a.elapsed_time(b) for a, b in step_events) * 1e-3
        return summarize(arrivals, time.perf_counter() - t0, self.device_s, self.steps)

    @staticmethod
    def plan(items: Sequence[Tuple[int, int, int, int]], step_samples: int) -> List[int]:
        """htc_serve_plan on (pixels, remaining passes, quantum, priority) items in arrival
        order: the passes the next step gives each."""
        arr = (_lib.HtcPlanItem * max(len(items), 1))()
        for i, (px, rem, q, pri) in enumerate(items):
            arr[i] = _lib.HtcPlanItem(px, rem, q, pri, 0)
        out = (ctypes.c_uint32 * max(len(items), 1))()
        _lib.call("htc_serve_plan", ctypes.cast(arr, ctypes.c_void_p), len(items), step_samples,
                  ctypes.cast(out, ctypes.c_void_p))
        return list(out)[:len(items)]


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
