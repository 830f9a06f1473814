#!/usr/bin/env python
"""Benchmark: Msamples/s and ray-bounces/s of the path-tracing hot path at 1080p hyperbolic.

Workload (one GPU): the 1920x1080 hyperbolic scene of 200 objects (60 % horospheres,
40 % geodesic planes) placed by random det-1 Moebius maps with translation distance up to 6,
H = 8 light hops, synthetic and seeded (hypertrace_b200.scene.config2). A step renders
`--passes` passes over the whole frame (each pass is one sample per pixel) through
htc_render_passes, which runs each pass as wavefronts: one launch of render_wave per hop
depth over queues of ray states. The frame's 256 spp are 256 / passes such steps. The
one-pass kernel (one launch per pass) and the persistent kernel are timed beside it.

    python bench.py [--gpus N --steps K --warmup W --passes P]
    python bench.py --impl reference      # the reference's own kernel code on the host CPU

On one GPU the line also carries, measured after the timed region:
  parity    the full frame rendered for 16 passes against the reference's kernel code
            (oracle/_ref) on random pixels: mismatched / bit-exact fractions, and the
            per-pixel error against the FP64 build of the same code;
  batched   the mixed workload of 96 views (resolutions 256x256 to 1920x1080, spp 16-256,
            half Euclidean, half hyperbolic with 20-200 objects) through one launch per pass,
            hop depth and recipe over all views, against the same views rendered one at a
            time with the one-pass kernel (one launch per pass) and with wavefronts;
  serving   Poisson arrivals at 50 and 2000 requests/s (70 % interactive 1280x720 8-spp
            frames with a moving camera, 30 % batch jobs) through the continuous-batching
            server, against a FIFO server that renders one request at a time with the
            one-pass kernel: throughput and p50 / p99 latency per class.

Under torchrun (N > 1) each rank renders its own frame (replicas: the path has no exchange
step); the reported value is all ranks' samples over the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "Msamples/s at 1080p hyperbolic (1920x1080, 200 objects, H=8)"
UNIT = "Msamples/s"

# Measured per path advanced by render_wave on this frame: one ncu capture of the 8 launches
# of one pass (hop depths 0-7) of `python bench.py --steps 1 --warmup 1 --no-extras --no-e2e
# --no-cpu-baseline`, each counter summed over the 8 launches and divided by the pass's path-hops
# (1920 x 1080 x hops per sample of that run). FP32 operations count 2 per FFMA, 1 per FADD /
# FMUL, twice that for their packed forms (FFMA2 / FADD2 / FMUL2); instructions are warp
# instructions issued; DRAM bytes are read + written. Frozen from that capture (the summary with
# the command is profiles/render_wave_hy1080p_200obj.md): re-capture after a kernel change.
FP32_OPS_PER_HOP = 4243.3       # 41.63e9 per pass over 9.81e6 path-hops
WARP_INSTR_PER_HOP = 284.84     # 2.794e9 per pass
DRAM_BYTES_PER_HOP = 147.77     # 1.450e9 per pass
# The reference's own FP32 count per hop for comparison: every object's detect maps the ray in
# and out (two ray maps of 256 operations, object/mapped.inl:32,34, plus the shape test), i.e.
# 527 per object and hop. Distance culling skips 98 % of those tests, so this count can exceed
# the chip's peak: it measures how much of the reference's algorithm each second covers, not
# how busy the FP32 pipes are.
REF_OPS_PER_OBJECT_TEST = 527


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--passes", type=int, default=4, help="passes (samples per pixel) per step")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["hy1080", "batched", "serving", "accuracy", "examples"], default="hy1080",
                    help="hy1080: the headline 1080p hyperbolic frame; batched: 96 mixed views, one launch "
                         "per pass, hop depth and recipe over all of them; serving: Poisson requests through "
                         "the continuous-batching server")
    ap.add_argument("--spp-scale", type=float, default=1.0, help="batched: scale of every view's spp")
    ap.add_argument("--requests", type=int, default=1000, help="serving: requests per arrival rate")
    ap.add_argument("--rates", type=str, default="50,2000", help="serving: arrival rates (req/s)")
    ap.add_argument("--parity-pixels", type=int, default=4096, help="parity: pixels compared with the oracle")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the parity, batched and serving measurements of the default line")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--case", type=str, default="", help="examples: run only the cases whose name contains this")
    return ap.parse_args()


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"ht_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- CPU side
def cpu_baseline(wl, seconds: float, threads: int = 0):
    """The reference's own kernel code (oracle/_ref, host C++) on this box's cores, on a
    bounded sample of the workload: chunks of pixels of the frame, one pass each, until
    `seconds` of wall time are spent. Falls back to the C restatement when _ref is absent."""
    from oracle import oracle
    kind = "reference" if oracle.ref_available(32) else "port"
    cores = threads or os.cpu_count() or 1
    sc = wl.scene
    data = sc.to_bytes()
    W, H = wl.width, wl.height
    rng = np.random.default_rng(0)
    chunk = 2048
    samples = 0
    from hypertrace_b200.scene import pixel_seeds
    seeds_all = pixel_seeds(wl.global_seed, W * H)
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        pix = rng.choice(W * H, chunk, replace=False).astype(np.uint32)
        seeds = seeds_all[pix]
        flags = oracle.JITTER_YX if kind == "port" else 0
        r = oracle.render(data, sc.recipe, sc.hops, W, H, pix, seeds, passes=1, impl=kind, threads=cores,
                          flags=flags)
        samples += r.stats["samples"]
    dt = time.perf_counter() - t0
    return {"value": samples / dt / 1e6, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{samples} samples (random pixels of the 1920x1080 frame, 1 pass each) in {dt:.1f} s"}


def measure_parity(ctx, wl, n_pixels: int, passes: int = 16):
    """Parity of the timed path at the workload's own size, outside the timed region: the
    whole frame rendered for `passes` passes (wavefronts) from its seeds, `n_pixels` random
    pixels compared with the reference's own kernel code built for the host (oracle/_ref,
    f32) over the same passes; a pixel is mismatched when its RNG state differs or its
    radiance is off by more than 1e-4 relative (floor 1e-3). The FP64 build of the same
    code gives each pixel's error of the FP32 result (relative, floor 1e-3), over all
    sampled pixels and over those whose path the FP64 run takes too (same RNG state)."""
    import torch
    from hypertrace_b200 import processing as P
    from hypertrace_b200 import _lib
    from oracle import oracle
    sc = wl.scene
    W, H = wl.width, wl.height
    impl = "reference" if oracle.ref_available(32) and oracle.ref_available(64) else "port"
    buf = P.EntityBuffer(ctx, sc)
    canvas = P.Canvas(ctx, (W, H), global_seed=wl.global_seed)
    seeds0 = canvas.seeds.cpu().numpy().view(np.uint32).copy()
    P.Render(ctx, sc.recipe, sc.hops, _lib.HTC_FLAG_JITTER_YX).render_passes(buf, canvas, passes)
    torch.cuda.synchronize()
    rng = np.random.default_rng(99)
    pix = np.sort(rng.choice(W * H, n_pixels, replace=False)).astype(np.uint32)
    gpu = canvas.image.cpu().numpy().reshape(-1, 4)[pix]
    gseeds = canvas.seeds.cpu().numpy().view(np.uint32)[pix]
    cores = os.cpu_count() or 1
    data = sc.to_bytes()
    t0 = time.perf_counter()
    f32 = oracle.render(data, sc.recipe, sc.hops, W, H, pix, seeds0[pix], passes=passes, impl=impl,
                        threads=cores, flags=oracle.JITTER_YX)
    f64 = oracle.render(data, sc.recipe, sc.hops, W, H, pix, seeds0[pix], passes=passes, impl=impl,
                        threads=cores, flags=oracle.JITTER_YX, precision=64)
    cpu_s = time.perf_counter() - t0
    same = gseeds == f32.seeds
    rel = (np.abs(gpu - f32.canvas) / np.maximum(np.abs(f32.canvas), 1e-3)).max(axis=1)
    mismatch = (~same) | (rel > 1e-4)
    exact = same & np.all(gpu.view(np.uint32) == f32.canvas.view(np.uint32), axis=1)
    g = gpu[:, :3] / passes
    c64 = f64.canvas[:, :3] / passes
    rel64 = (np.abs(g - c64) / np.maximum(np.abs(c64), 1e-3)).max(axis=1)
    same64 = f64.seeds == gseeds
    return {"pixels": int(n_pixels), "passes": passes, "checker": f"oracle/_ref ({impl})", "cpu_s": round(cpu_s, 2),
            "mismatch_frac": float(mismatch.mean()), "rng_mismatch_frac": float((~same).mean()),
            "hops_per_pixel": f32.stats["hops"] / n_pixels,
            "mismatch_per_hop": float(mismatch.mean()) / max(f32.stats["hops"] / n_pixels, 1e-9),
            "bit_exact_frac": float(exact.mean()),
            "f64_rel_err": {"median": float(np.median(rel64)), "mean": float(rel64.mean()), "max": float(rel64.max()),
                            "same_path_frac": float(same64.mean()),
                            "same_path_max": float(rel64[same64].max()) if same64.any() else None,
                            "same_path_mean": float(rel64[same64].mean()) if same64.any() else None}}


def run_reference(args, rank: int):
    """--impl reference: time the reference's CPU implementation with all host threads."""
    if rank != 0:
        return
    from hypertrace_b200 import scene as S
    from oracle import oracle
    wl = S.config2()
    kind = "reference" if oracle.ref_available(32) else "port"
    sc = wl.scene
    data = sc.to_bytes()
    W, H = wl.width, wl.height
    cores = os.cpu_count() or 1
    pix_per_step = 4096
    rng = np.random.default_rng(1)
    seeds_all = S.pixel_seeds(wl.global_seed, W * H)

    def step():
        pix = rng.choice(W * H, pix_per_step, replace=False).astype(np.uint32)
        r = oracle.render(data, sc.recipe, sc.hops, W, H, pix, seeds_all[pix], passes=1, impl=kind,
                          threads=cores, flags=0 if kind == "reference" else oracle.JITTER_YX)
        return r.stats

    for _ in range(args.warmup):
        step()
    samples = hops = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st = step()
        samples += st["samples"]
        hops += st["hops"]
    dt = time.perf_counter() - t0
    value = samples / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl.name, "width": W, "height": H, "objects": sc.n_objects, "hops": sc.hops,
                   "pixels_per_step": pix_per_step, "passes_per_step": 1},
        "ray_bounces_per_s": hops / dt,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{args.steps} steps x {pix_per_step} random pixels x 1 pass of the 1080p frame"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU side
def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist
    import ctypes
    from hypertrace_b200 import scene as S
    from hypertrace_b200 import processing as P
    from hypertrace_b200 import _lib
    from hypertrace_b200 import build as hb

    hb.build()
    torch.cuda.set_device(local_rank)
    if args.workload == "batched":
        return bench_batched(args)
    if args.workload == "serving":
        return bench_serving(args)
    if args.workload == "examples":
        return bench_examples(args)
    if args.workload == "accuracy":
        return bench_accuracy(args)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    wl = S.config2()
    sc = wl.scene
    W, H = wl.width, wl.height
    ctx = P.Context(local_rank)
    dev = ctx.device
    stream = torch.cuda.current_stream(dev)
    buf = P.EntityBuffer(ctx, sc)
    from hypertrace_b200 import replicas
    canvas = P.Canvas(ctx, (W, H), global_seed=replicas.replica_seed(wl.global_seed, rank))
    render = P.Render(ctx, sc.recipe, sc.hops)
    stats = torch.zeros(8, dtype=torch.int64, device=dev)
    l2_flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    # FP32 peak of this GPU (roofline denominator): FMA probe, best of several launches.
    probe_blocks = 148 * 8
    scratch = torch.empty(probe_blocks * 256, dtype=torch.float32, device=dev)
    flops = ctypes.c_double()
    best = 0.0
    for i in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.call("htc_fp32_probe", scratch.data_ptr(), probe_blocks, 4096, ctypes.byref(flops), stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        if i > 0:
            best = max(best, flops.value / (e0.elapsed_time(e1) * 1e-3))
    fp32_peak_tflops = best / 1e12

    def step(with_stats):
        render.render_passes(buf, canvas, args.passes, stats=stats if with_stats else None, sync=False)

    for _ in range(args.warmup):
        step(False)
    _lib.call("htc_program_check", render.handle, stream.cuda_stream)

    # ---------------- timed region: K steps, device time per launch, L2 flushed in between
    stats.zero_()
    clocks = ClockSampler(local_rank)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_wall = time.perf_counter()
    times = []
    for _ in range(args.steps):
        l2_flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step(True)
        e1.record(stream)
        times.append((e0, e1))
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    _lib.call("htc_program_check", render.handle, stream.cuda_stream)
    launch_ms = [a.elapsed_time(b) for a, b in times]
    dev_s = sum(launch_ms) * 1e-3
    st = stats.cpu().numpy().astype(np.float64)
    samples, hops, tests, hits, exact = st[:5]
    all_samples, max_s, all_hops = replicas.aggregate(samples, dev_s, hops, device=dev)
    value = all_samples / max_s / 1e6

    # roofline of render_wave (one launch per hop depth, `passes * hops` launches per step):
    # measured operations per path-hop x this run's path-hops, over the device time of the
    # step, which also holds the coherence sort between hop depths (4 launches per depth of a
    # hyperbolic pass after the first)
    launches = args.steps * args.passes * sc.hops
    sort_launches = args.steps * args.passes * (sc.hops - 1) * 4 if sc.recipe == _lib.HTC_RECIPE_HY else 0
    per_launch_s = dev_s / launches
    achieved = FP32_OPS_PER_HOP * hops / dev_s / 1e12 if FP32_OPS_PER_HOP else None
    ref_tflops = tests * REF_OPS_PER_OBJECT_TEST / dev_s / 1e12

    # ---------------- the persistent kernel (all passes in one launch) on the same frame,
    # through the entry point that still uses it, for comparison
    persistent = None
    if rank == 0:
        status = ctypes.c_uint32(0)
        p_ms = []
        for i in range(3):   # the first call sets the entry point up on this device: untimed
            stats.zero_()
            l2_flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _lib.call("htc_render_passes_noalloc", sc.recipe, sc.hops, 32, 0, W, H, buf.ptr(), buf.size,
                      canvas.image.data_ptr(), canvas.seeds.data_ptr(), args.passes, stats.data_ptr(),
                      ctypes.byref(status), stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            if i > 0:
                p_ms.append(e0.elapsed_time(e1))
        ms = float(np.mean(p_ms))
        ps = stats.cpu().numpy()
        persistent = {"value": float(ps[0]) / ms / 1e3, "unit": UNIT, "ms_per_launch": ms,
                      "ray_bounces_per_s": float(ps[1]) / ms * 1e3, "kernel": "render_persistent"}

    # ---------------- the one-pass kernel (one launch per pass, the reference's kernel shape)
    plain = None
    if rank == 0:
        stats.zero_()
        w_ms = []
        for _ in range(args.steps):
            l2_flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.passes):
                render.render(buf, canvas, stats=stats, sync=False)
            e1.record(stream)
            w_ms.append((e0, e1))
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in w_ms)
        ws = stats.cpu().numpy()
        plain = {"value": float(ws[0]) / ms / 1e3, "unit": UNIT, "ms_per_step": ms / args.steps,
                 "ray_bounces_per_s": float(ws[1]) / ms * 1e3, "kernel": "render_plain, one launch per pass"}

    # ---------------- e2e through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        pipe = P.Pipeline(ctx, (W, H), sc, global_seed=replicas.replica_seed(wl.global_seed, rank))
        host_scene = torch.frombuffer(bytearray(sc.to_bytes()), dtype=torch.uint8).pin_memory()
        host_image = torch.empty(W * H * 4, dtype=torch.uint8).pin_memory()
        for _ in range(2):
            pipe.render(args.passes)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            pipe.scene_buffer.tensor.copy_(host_scene, non_blocking=True)      # set_scene upload
            pipe.render_.render_passes(pipe.scene_buffer, pipe.canvas, args.passes, sync=False)
            _lib.call("htc_extract_gamma_pack", W, H, max(pipe.canvas.passes, 1), ctypes.c_float(1 / 2.2),
                      pipe.canvas.image.data_ptr(), pipe.packed.data_ptr(), stream.cuda_stream)
            host_image.copy_(pipe.packed, non_blocking=True)                  # get_image read-back
            stream.synchronize()
        ev1.record(stream)
        torch.cuda.synchronize()
        e2e_s = ev0.elapsed_time(ev1) * 1e-3
        tt = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_samples = float(W * H * args.passes * args.steps * world)
        e2e = {"value": e2e_samples / float(tt.item()) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": int(host_scene.numel()), "d2h_bytes_per_step": int(host_image.numel()),
               "wall_s": time.perf_counter() - t0}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(wl, args.cpu_seconds)

    # ---------------- untimed extras of the one-GPU line: parity at size, batched, serving
    parity = batched = serving = None
    if world == 1 and not args.no_extras:
        parity = measure_parity(ctx, wl, args.parity_pixels)
        batched = measure_batched(args)
        serving = measure_serving(args)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_s / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": wl.name, "width": W, "height": H, "objects": sc.n_objects, "hops": sc.hops,
                       "passes_per_step": args.passes, "kernel": "render_wave, one launch per hop depth",
                       "parallelism": f"replicas{world}",
                       "l2": "flushed between steps (256 MB device write outside the timed events)"},
            "ray_bounces_per_s": all_hops / max_s,
            "hops_per_sample": hops / max(samples, 1),
            "exact_tests_per_hop": exact / max(hops, 1),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak_tflops, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak_tflops if achieved and fp32_peak_tflops else None,
                         "traffic": DRAM_BYTES_PER_HOP * hops / launches if DRAM_BYTES_PER_HOP else None,
                         "source": "FP32 operations and DRAM bytes per path-hop: constants from one ncu "
                                   "capture of a pass's 8 render_wave launches (ffma x2 + fadd + fmul, packed "
                                   "forms x2), times this run's path-hops, over the step's device time (the "
                                   "sort launches between hop depths included); traffic per render_wave launch",
                         "peak_source": "measured FFMA probe (htc_fp32_probe) on this GPU in this run",
                         "issue": {"achieved_ginstr_per_s": WARP_INSTR_PER_HOP * hops / dev_s / 1e9
                                   if WARP_INSTR_PER_HOP else None,
                                   "peak_ginstr_per_s": 148 * 4 * (clk.get("sm_mhz") or 1965.0) / 1e3,
                                   "frac": WARP_INSTR_PER_HOP * hops / dev_s / 1e9
                                   / (148 * 4 * (clk.get("sm_mhz") or 1965.0) / 1e3) if WARP_INSTR_PER_HOP else None,
                                   "note": "warp instructions issued (the kernel is issue-bound) against one per "
                                           "cycle per SM sub-partition at the sampled SM clock"},
                         "reference_count_tflops": ref_tflops,
                         "reference_count_note": "the reference's FP32 count (527 per object test, hops x "
                                                 "objects tests) over the same time: above the peak because "
                                                 "culling skips 98 % of those tests"},
            "parity": parity,
            "batched": batched,
            "serving": serving,
            "persistent": persistent,
            "plain_one_pass": plain,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": launches + sort_launches,
            "wall_s_timed": t_wall,
            "launch_ms": [round(x, 3) for x in launch_ms],
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _time_ms(fn, stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def measure_batched(args):
    """The mixed workload (96 views: resolutions from {256^2, 640x480, 1280x720, 1920x1080},
    spp in {16..256} x --spp-scale, half Euclidean / half hyperbolic with 20-200 objects):
    batched wavefronts (one launch per pass and hop depth covering every view, autotuned tile
    size / residency, CUDA graphs, 16 passes of every unfinished view per step) against the
    same views rendered one at a time with the plain one-pass kernel and with the single-view
    wavefront form (htc_render_passes). Results of the three are bit-identical
    (tests/test_gpu_batch.py), so RMSE against any reference is equal."""
    import torch
    from hypertrace_b200 import batch as B
    from hypertrace_b200 import processing as P
    ctx = P.Context(0)
    stream = torch.cuda.current_stream(ctx.device)
    views = B.config3(spp_scale=args.spp_scale)
    for v in views:
        v.allocate(ctx)
    total_samples = sum(v.width * v.height * v.spp for v in views)
    br = B.BatchRenderer(ctx, max_views=128)
    tile, res, timings = B.autotune(br, views)
    stats = torch.zeros(8, dtype=torch.int64, device=ctx.device)
    dev_ms, steps, launches = 0.0, 0, 0
    active_key = None
    while any(v.remaining for v in views):
        active = [v for v in views if v.remaining]
        passes = [min(16, v.remaining) for v in active]
        key = (tuple(id(v) for v in active), tuple(passes))
        if key != active_key:
            br.set_views(active, passes, tile_pixels=tile, blocks_per_sm=res)
            active_key = key
        dev_ms += _time_ms(lambda: br.render(stats=stats, graph=True), stream)
        for v, p in zip(active, passes):
            v.done_passes += p
        steps += 1
    br.check()
    st = stats.cpu().numpy().astype(np.float64)
    batched = {"value": st[0] / dev_ms / 1e3, "unit": UNIT, "device_ms": dev_ms, "steps": steps,
               "ray_bounces_per_s": st[1] / dev_ms * 1e3, "tile_pixels": tile, "blocks_per_sm": res,
               "autotune_ms": {f"{k[0]}x{k[1]}": round(t, 3) for k, t in timings.items()}}
    for v in views:
        v.release()

    def per_view(wavefront):
        vs = B.config3(spp_scale=args.spp_scale)
        ms = 0.0
        renders = {}
        # each program's wavefront queues, sized once by its largest view, outside the timing
        for v in sorted(vs, key=lambda v: -v.width * v.height):
            key = (v.scene.recipe, v.scene.hops)
            if key not in renders and wavefront:
                v.allocate(ctx)
                renders[key] = P.Render(ctx, *key)
                renders[key].render_wavefront(v.buffer, v.canvas, 1)
                v.release()
        for v in vs:
            v.allocate(ctx)
            key = (v.scene.recipe, v.scene.hops)
            r = renders.setdefault(key, P.Render(ctx, *key))
            if wavefront:
                ms += _time_ms(lambda: r.render_wavefront(v.buffer, v.canvas, v.spp, sync=False), stream)
            else:
                ms += _time_ms(lambda: [r.render(v.buffer, v.canvas, sync=False) for _ in range(v.spp)], stream)
            v.release()
        return {"value": total_samples / ms / 1e3, "unit": UNIT, "device_ms": ms}

    plain = per_view(False)
    single = per_view(True)
    return {"workload": "mixed-96-views", "spp_scale": args.spp_scale, "total_samples": total_samples,
            "passes_per_step": 16, "batched": batched, "plain_per_view": plain, "wavefront_per_view": single,
            "speedup_vs_plain": batched["value"] / plain["value"],
            "speedup_vs_wavefront_per_view": batched["value"] / single["value"]}


def bench_batched(args):
    out = measure_batched(args)
    line = {"metric": "Msamples/s, mixed batched workload (96 views, one launch per pass and hop depth)",
            "value": out["batched"]["value"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic", "config": {k: out[k] for k in ("workload", "spp_scale", "total_samples",
                                                                "passes_per_step")}}
    line.update({k: v for k, v in out.items() if k not in line["config"]})
    print(json.dumps(line), flush=True)


def measure_serving(args):
    """Poisson arrivals (70 % interactive 1280x720 8-spp frames with a moving camera, 30 %
    batch jobs drawn from the mixed workload), served by continuous batching under a 120 GB
    budget, against one-request-at-a-time plain kernels; p50/p99 latency per class."""
    import torch
    from hypertrace_b200 import processing as P
    from hypertrace_b200 import serve as V
    ctx = P.Context(0)
    # warm-up: compile-free, but the first launches load modules and size caches
    V.Server(ctx).run(V.make_requests(6, 1000.0, seed=1))
    out = {}
    for rate in [float(x) for x in args.rates.split(",")]:
        served = V.Server(ctx).run(V.make_requests(args.requests, rate))
        plain = V.plain_fifo(ctx, V.make_requests(args.requests, rate))
        out[str(int(rate))] = {"served": served, "plain_fifo": plain,
                               "throughput_ratio": served["throughput_msamples_per_s"]
                               / plain["throughput_msamples_per_s"]}
        torch.cuda.synchronize()
    return {"workload": "serving", "requests_per_rate": args.requests, "hbm_budget_gb": 120,
            "interactive": "1280x720 x 8 spp hyperbolic, moving camera", "batch_spp_scale": 0.125,
            "requests_stated": "10^4 requests per rate swept over 50-2000 req/s; this line runs "
                               f"{args.requests} per rate at {args.rates} req/s", "rates": out}


def bench_serving(args):
    out = measure_serving(args)
    first = out["rates"][next(iter(out["rates"]))]
    line = {"metric": "serving: throughput and p50/p99 frame latency, continuous batching vs plain per-request",
            "value": first["served"]["throughput_msamples_per_s"], "unit": UNIT, "n_gpus": 1,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {k: v for k, v in out.items() if k != "rates"}, "rates": out["rates"]}
    print(json.dumps(line), flush=True)


def bench_examples(args):
    """The generic scene programs on the scene types of the reference's hy and eu examples
    (main/examples/hy.rs: tiled planes and horospheres, transparent material, H = 3;
    main/examples/eu.rs: plane / sphere / cube, refractive material, gradient background,
    H = 4) and on a heavier random scene of the hy type: built-in recipe and the same type
    compiled at run time with NVRTC, each against the reference's own kernel code on the host
    cores (oracle/_ref, all threads, a bounded pixel sample)."""
    import torch
    from hypertrace_b200 import _lib
    from hypertrace_b200 import processing as P
    from hypertrace_b200 import scene as S
    from hypertrace_b200 import types as T
    from oracle import oracle
    ctx = P.Context(0)
    stream = torch.cuda.current_stream(ctx.device)
    cores = os.cpu_count() or 1
    cases = [("hy-tiled-example-800x600-h3", T.hy_tiled_type(), T.hy_example_value(), _lib.HTC_RECIPE_HY_TILED, 3, 800, 600),
             ("eu-gradient-example-800x600-h4", T.eu_gradient_type(), T.eu_example_value(), _lib.HTC_RECIPE_EU_GRADIENT,
              4, 800, 600),
             ("hy-tiled-random-1920x1080-64obj-h8", T.hy_tiled_type(), T.hy_tiled_random_value(17, 64, 3.0),
              _lib.HTC_RECIPE_HY_TILED, 8, 1920, 1080)]
    results = {}
    passes = 16
    cases = [c for c in cases if args.case in c[0]]
    for name, ty, val, recipe, hops, W, H in cases:
        data = T.serialize(ty, val)
        buf = P.EntityBuffer(ctx, data)
        res = {}
        for kind, render in (("builtin", P.Render(ctx, recipe, hops)), ("nvrtc", P.Render.build(ctx, ty, hops))):
            canvas = P.Canvas(ctx, (W, H), global_seed=0x5EED0007)
            stats = torch.zeros(8, dtype=torch.int64, device=ctx.device)
            for _ in range(max(args.warmup, 1)):
                render.render_passes(buf, canvas, passes, sync=False)
            torch.cuda.synchronize()
            stats.zero_()
            ms = 0.0
            for _ in range(args.steps):
                ms += _time_ms(lambda: render.render_passes(buf, canvas, passes, stats=stats, sync=False), stream)
            render._check(True)
            st = stats.cpu().numpy().astype(np.float64)
            res[kind] = {"Msamples_per_s": st[0] / ms / 1e3, "ray_bounces_per_s": st[1] / ms * 1e3,
                         "ms_per_step": ms / args.steps, "object_tests_per_hop": st[2] / max(st[1], 1)}
        cpu = None
        if oracle.ref_available():
            rng = np.random.default_rng(3)
            n = 4096 if W * H > 4096 else W * H
            pix = np.sort(rng.choice(W * H, n, replace=False)).astype(np.uint32)
            seeds = S.pixel_seeds(1, W * H)[pix]
            t0 = time.perf_counter()
            oracle.render(data, recipe, hops, W, H, pix, seeds, passes=2, impl="reference", threads=cores)
            dt = time.perf_counter() - t0
            cpu = {"Msamples_per_s": n * 2 / dt / 1e6, "cores": cores, "kind": "reference",
                   "sample": f"{n} random pixels x 2 passes"}
        res["cpu_reference"] = cpu
        if cpu:
            res["speedup_builtin_vs_cpu"] = res["builtin"]["Msamples_per_s"] / cpu["Msamples_per_s"]
        results[name] = res
    print(json.dumps({"metric": "Msamples/s, generic scene programs (reference example scene types)",
                      "unit": UNIT, "passes_per_step": passes, "steps": args.steps, "data": "synthetic",
                      "results": results}), flush=True)


def bench_accuracy(args):
    """Error of the FP32 GPU result against the FP64 CPU oracle (same scene bytes, seeds and
    passes) per pixel, and RMSE of the FP32 GPU image and of the FP64 image against a converged
    FP64 image (many more passes), on random pixel subsets of the hyperbolic workloads."""
    import torch
    from hypertrace_b200 import processing as P
    from hypertrace_b200 import scene as S
    from oracle import oracle
    ctx = P.Context(0)
    out = {}
    cores = os.cpu_count() or 1
    for name, wl, n_pix, passes, conv_passes in (("hyperbolic-800x600-18obj-h6", S.config1(), 400, 64, 1024),
                                                 ("hyperbolic-1920x1080-200obj-h8", S.config2(), 200, 64, 512)):
        sc = wl.scene
        W, H = wl.width, wl.height
        buf = P.EntityBuffer(ctx, sc)
        canvas = P.Canvas(ctx, (W, H), global_seed=wl.global_seed)
        seeds0 = canvas.seeds.cpu().numpy().view(np.uint32).copy()
        P.Render(ctx, sc.recipe, sc.hops).render_passes(buf, canvas, passes)
        torch.cuda.synchronize()
        gpu = canvas.image.cpu().numpy().reshape(-1, 4)
        rng = np.random.default_rng(11)
        pix = np.sort(rng.choice(W * H, n_pix, replace=False)).astype(np.uint32)
        data = sc.to_bytes()
        f32 = oracle.render(data, sc.recipe, sc.hops, W, H, pix, seeds0[pix], passes=passes, threads=cores)
        f64 = oracle.render(data, sc.recipe, sc.hops, W, H, pix, seeds0[pix], passes=passes, threads=cores,
                            precision=64)
        conv_seeds = S.pixel_seeds(wl.global_seed ^ 0xC0FFEE, W * H)[pix]
        conv = oracle.render(data, sc.recipe, sc.hops, W, H, pix, conv_seeds, passes=conv_passes, threads=cores,
                             precision=64)
        g = gpu[pix, :3] / passes
        c32 = f32.canvas[:, :3] / passes
        c64 = f64.canvas[:, :3] / passes
        cc = conv.canvas[:, :3] / conv_passes
        rel = np.abs(g - c64) / np.maximum(np.abs(c64), 1e-3)
        same_path = f64.seeds == f32.seeds
        out[name] = {
            "pixels": int(n_pix), "passes": passes, "converged_passes": conv_passes,
            "gpu_vs_cpu_f32_bit_identical_fraction": float(np.mean(np.all(g == c32, axis=1))),
            "gpu_vs_f64_rel_err": {"mean": float(rel.mean()), "median": float(np.median(rel)),
                                   "max": float(rel.max())},
            "gpu_vs_f64_rel_err_on_same_paths": {
                "fraction_of_pixels": float(same_path.mean()),
                "max": float(rel[same_path].max()) if same_path.any() else None},
            "rmse_vs_converged_f64": {"gpu_f32": float(np.sqrt(np.mean((g - cc) ** 2))),
                                      "cpu_f64": float(np.sqrt(np.mean((c64 - cc) ** 2)))},
        }
    print(json.dumps({"metric": "error of the FP32 GPU path vs the FP64 oracle", "data": "synthetic",
                      "results": out}), flush=True)


if __name__ == "__main__":
    main()
