"""GPU parity: the CUDA render path against the CPU oracle on the same scene bytes and seeds.

The bar (per pixel, per pass):
  * RNG state bit-exact -- a mismatch can only come from a branch that flipped on a
    last-ulp difference of a transcendental (cos/sin/log/pow differ between CUDA and the
    host libm); the fraction of such pixels is bounded below;
  * radiance within 1e-4 relative (abs floor 1e-3) on every pixel whose RNG state agrees.
"""
import numpy as np
import pytest
import torch

from hypertrace_b200 import scene as S
from hypertrace_b200 import processing as P
from hypertrace_b200 import _lib
from oracle import oracle

pytestmark = pytest.mark.gpu

RTOL = 1e-4
ATOL_FLOOR = 1e-3
# A pixel is "mismatched" when its RNG state differs or its radiance is off by more than
# RTOL: both can only come from a branch that flipped on a last-ulp difference of a
# transcendental (CUDA's logf / FP64 sincos / pow vs the host libm). Bound on their share:
MAX_MISMATCH = 0.002
# The same bound per executed hop, for runs long enough that flips compound along a pixel's
# RNG stream: the GPU takes cos / sin in FP64 rounded once and CUDA's logf, the reference's
# host build calls glibc's cosf / sinf / logf, which round differently on a small share of
# arguments. In the C restatement, swapping in the FP64-rounded cos / sin alone gives 0.3 %
# mismatched pixels over 16 passes of the 1080p frame (about 76 hops per pixel): 4e-5 per hop;
# the GPU shows 0.365 % (4.8e-5 per hop). Bound: 1e-4.
MAX_FLIP_PER_HOP = 1e-4


def _compare(gpu_canvas, gpu_seeds, ref, label, min_exact=1.0 - MAX_MISMATCH, max_mismatch=MAX_MISMATCH):
    same = gpu_seeds == ref.seeds
    rel = (np.abs(gpu_canvas - ref.canvas) / np.maximum(np.abs(ref.canvas), ATOL_FLOOR)).max(axis=1)
    mismatch = (~same) | (rel > RTOL)
    frac = float(mismatch.mean())
    assert frac <= max_mismatch, f"{label}: {frac:.4f} of pixels mismatch (rng {(~same).mean():.4f})"
    # the typical pixel is bit-identical, not merely close
    exact = np.all(gpu_canvas.view(np.uint32) == ref.canvas.view(np.uint32), axis=1) & same
    assert exact.mean() >= min_exact, f"{label}: only {exact.mean():.4f} bit-exact"
    print(f"{label}: mismatched fraction {frac:.5f}, bit-exact {exact.mean():.5f}")
    return frac


def _render_gpu(wl, W, H, passes, form, flags=0):
    """form "render": `passes` htc_render calls (the one-pass kernel); "render_passes": one
    htc_render_passes call (wavefronts, or the one-pass kernel for small cheap canvases)."""
    ctx = P.Context(0)
    buf = P.EntityBuffer(ctx, wl.scene)
    canvas = P.Canvas(ctx, (W, H), global_seed=wl.global_seed)
    seeds0 = canvas.seeds.cpu().numpy().view(np.uint32).copy()
    r = P.Render(ctx, wl.scene.recipe, wl.scene.hops, flags)
    if form == "render_passes":
        r.render_passes(buf, canvas, passes)
    else:
        for _ in range(passes):
            r.render(buf, canvas)
    torch.cuda.synchronize()
    return (seeds0, canvas.image.cpu().numpy().reshape(-1, 4).copy(),
            canvas.seeds.cpu().numpy().view(np.uint32).copy())


@pytest.mark.parametrize("cfg", ["config0", "config1", "config2"])
@pytest.mark.parametrize("form", ["render", "render_passes"])
def test_render_matches_oracle(built, cfg, form):
    wl = getattr(S, cfg)()
    W, H = (wl.width, wl.height) if cfg != "config2" else (480, 270)
    passes = 2
    seeds0, cv, sd = _render_gpu(wl, W, H, passes, form)
    rng = np.random.default_rng(7)
    pix = np.sort(rng.choice(W * H, min(W * H, 1500), replace=False)).astype(np.uint32)
    ref = oracle.render(wl.scene.to_bytes(), wl.scene.recipe, wl.scene.hops, W, H, pix, seeds0[pix],
                        passes=passes, threads=8)
    _compare(cv[pix], sd[pix], ref, f"{cfg} {form}")


def test_full_frame_config2_matches_reference(built):
    """The 1080p stress workload at its own size: the whole 1920x1080 frame of 200 objects
    (H = 8) rendered on the GPU for 16 passes (wavefronts), 20 000 random pixels compared
    with the reference's own kernel code built for the host (oracle/_ref; the C
    restatement, which reproduces it bit for bit, where _ref is not built) over the same 16
    passes from the same seeds. Branch flips on last-ulp transcendental differences compound
    along a pixel's RNG stream, so this is where the mismatch bound matters."""
    wl = S.config2()
    W, H, passes = wl.width, wl.height, 16
    impl = "reference" if oracle.ref_available() else "port"
    seeds0, cv, sd = _render_gpu(wl, W, H, passes, "render_passes", flags=_lib.HTC_FLAG_JITTER_YX)
    rng = np.random.default_rng(2024)
    pix = np.sort(rng.choice(W * H, 20000, replace=False)).astype(np.uint32)
    import os
    ref = oracle.render(wl.scene.to_bytes(), wl.scene.recipe, wl.scene.hops, W, H, pix, seeds0[pix],
                        passes=passes, threads=os.cpu_count() or 8, impl=impl, flags=oracle.JITTER_YX)
    assert ref.stats["samples"] == len(pix) * passes
    hops_per_pixel = ref.stats["hops"] / len(pix)
    bound = 1.0 - (1.0 - MAX_FLIP_PER_HOP) ** hops_per_pixel
    frac = _compare(cv[pix], sd[pix], ref, f"config2 full frame, {passes} passes, vs {impl}",
                    min_exact=1.0 - bound, max_mismatch=bound)
    print(f"hops per pixel {hops_per_pixel:.1f}, mismatch bound {bound:.4f}, flips per hop {frac / hops_per_pixel:.2e}")


@pytest.mark.parametrize("cfg", ["config0", "config1"])
def test_render_passes_equals_repeated_render(built, cfg):
    """One htc_render_passes call of P passes == P htc_render calls, bit for bit."""
    wl = getattr(S, cfg)()
    W, H = 160, 120
    _, cv_a, sd_a = _render_gpu(wl, W, H, 5, "render")
    _, cv_b, sd_b = _render_gpu(wl, W, H, 5, "render_passes")
    assert np.array_equal(sd_a, sd_b)
    assert np.array_equal(cv_a.view(np.uint32), cv_b.view(np.uint32))


@pytest.mark.parametrize("W,H,seed", [(1, 1, 0), (33, 7, 5), (1920, 1080, 0xDEADBEEF), (640, 480, 0xFFFFFFFF)])
def test_device_seeds_equal_host_seeds(built, W, H, seed):
    """Canvas seeds come from htc_fill_seeds on the device; they equal scene.pixel_seeds."""
    canvas = P.Canvas(P.Context(0), (W, H), global_seed=seed)
    assert np.array_equal(canvas.seeds.cpu().numpy().view(np.uint32), S.pixel_seeds(seed, W * H))


@pytest.mark.parametrize("sort", [True, False])
@pytest.mark.parametrize("cfg,W,H,passes", [("config0", 160, 120, 5), ("config1", 200, 150, 3),
                                           ("config2", 480, 270, 2), ("config1", 33, 7, 4),
                                           ("config1", 1, 1, 3), ("config0", 1, 37, 2)])
def test_wavefront_equals_repeated_plain(built, cfg, W, H, passes, sort):
    """Hop-depth wavefronts over ray-state queues == P plain launches, bit for bit, with the
    same statistics (samples, hops, hits, exact tests); hyperbolic queues with and without the
    coherence sort between hop depths."""
    wl = getattr(S, cfg)()
    ctx = P.Context(0)
    buf = P.EntityBuffer(ctx, wl.scene)
    r = P.Render(ctx, wl.scene.recipe, wl.scene.hops, 0 if sort else _lib.HTC_FLAG_NO_SORT)
    out = []
    for wave in (False, True):
        canvas = P.Canvas(ctx, (W, H), global_seed=wl.global_seed)
        stats = torch.zeros(8, dtype=torch.int64, device=ctx.device)
        if wave:
            r.render_wavefront(buf, canvas, passes, stats=stats)
        else:
            for _ in range(passes):
                r.render(buf, canvas, stats=stats)
        torch.cuda.synchronize()
        out.append((canvas.image.cpu().numpy().view(np.uint32).copy(), canvas.seeds.cpu().numpy().copy(),
                    stats.cpu().numpy().copy()))
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][2], out[1][2])
    assert out[1][2][_lib.STAT_SAMPLES] == W * H * passes


@pytest.mark.parametrize("seed", [None, 3, 4])
def test_sorted_wavefront_full_frame(built, seed):
    """The coherence sort at full size: one pass of the 1920x1080 hyperbolic frame (and of
    random hyperbolic scenes) with and without it gives the same canvas, seeds and statistics,
    so every queued path ran exactly once, whatever order the sort gave it."""
    if seed is None:
        wl = S.config2()
        scene, W, H, gs = wl.scene, wl.width, wl.height, wl.global_seed
    else:
        rng = np.random.default_rng(seed)
        scene = S.hyperbolic_scene(30 + 50 * seed, 60, 6.0, 8, 700 + seed, camera=S.random_moebius(rng, 1.0))
        W, H, gs = 1280, 720, seed
    ctx = P.Context(0)
    buf = P.EntityBuffer(ctx, scene)
    out = []
    for flags in (0, _lib.HTC_FLAG_NO_SORT):
        r = P.Render(ctx, scene.recipe, scene.hops, flags)
        canvas = P.Canvas(ctx, (W, H), global_seed=gs)
        stats = torch.zeros(8, dtype=torch.int64, device=ctx.device)
        r.render_wavefront(buf, canvas, 1, stats=stats)
        torch.cuda.synchronize()
        out.append((canvas.image.view(torch.int32).cpu(), canvas.seeds.cpu(), stats.cpu()))
    assert torch.equal(out[0][0], out[1][0])
    assert torch.equal(out[0][1], out[1][1])
    assert torch.equal(out[0][2], out[1][2])
    assert int(out[0][2][_lib.STAT_SAMPLES]) == W * H


def test_wavefront_single_hop_and_reuse(built):
    """H = 1 (hop 0 only, nothing queued) and a program reused across canvas sizes (queues grow)."""
    wl = S.config1()
    ctx = P.Context(0)
    buf = P.EntityBuffer(ctx, wl.scene)
    for hops in (1, wl.scene.hops):
        r = P.Render(ctx, wl.scene.recipe, hops)
        for W, H in ((64, 48), (300, 200), (64, 48)):
            a = P.Canvas(ctx, (W, H), global_seed=5)
            b = P.Canvas(ctx, (W, H), global_seed=5)
            for _ in range(2):
                r.render(buf, a)
            r.render_wavefront(buf, b, 2)
            torch.cuda.synchronize()
            assert torch.equal(a.seeds, b.seeds)
            assert torch.equal(a.image.view(torch.int32), b.image.view(torch.int32))


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("cfg", ["config0", "config1"])
def test_render_matches_reference_kernel(built, cfg):
    """Directly against the reference's own kernel compiled for the host (g++ jitter order)."""
    wl = getattr(S, cfg)()
    W, H = 200, 150
    seeds0, cv, sd = _render_gpu(wl, W, H, 2, "render_passes", flags=_lib.HTC_FLAG_JITTER_YX)
    pix = np.arange(0, W * H, 13, dtype=np.uint32)
    ref = oracle.render(wl.scene.to_bytes(), wl.scene.recipe, wl.scene.hops, W, H, pix, seeds0[pix],
                        passes=2, threads=8, impl="reference")
    _compare(cv[pix], sd[pix], ref, f"{cfg} vs reference")


def test_post_chain_matches_oracle(built):
    ctx = P.Context(0)
    W, H = 97, 61
    rng = np.random.default_rng(3)
    acc = (rng.random((W * H, 4), dtype=np.float32) * 6 - 1).astype(np.float32)
    acc[::17] = 0.0
    passes = 5
    img_ref, packed_ref = oracle.extract_gamma_pack(acc, passes, 1 / 2.2)
    canvas = torch.from_numpy(acc.reshape(-1)).to(ctx.device)
    image = torch.empty_like(canvas)
    image2 = torch.empty_like(canvas)
    packed = torch.empty(W * H * 4, dtype=torch.uint8, device=ctx.device)
    fused = torch.empty_like(packed)
    st = ctx.stream()
    _lib.call("htc_extract", W, H, passes, canvas.data_ptr(), image.data_ptr(), st)
    _lib.call("htc_gamma", W, H, P.ctypes.c_float(1 / 2.2), image.data_ptr(), image2.data_ptr(), st)
    _lib.call("htc_pack", W, H, image2.data_ptr(), packed.data_ptr(), st)
    _lib.call("htc_extract_gamma_pack", W, H, passes, P.ctypes.c_float(1 / 2.2), canvas.data_ptr(),
              fused.data_ptr(), st)
    torch.cuda.synchronize()
    g = image2.cpu().numpy().reshape(-1, 4)
    rel = np.abs(g - img_ref) / np.maximum(np.abs(img_ref), 1e-6)
    assert rel.max() < 2e-7
    pk = packed.cpu().numpy().reshape(-1, 4)
    fz = fused.cpu().numpy().reshape(-1, 4)
    assert np.array_equal(pk, fz)
    assert (pk != packed_ref).mean() < 1e-3
    assert np.abs(pk.astype(int) - packed_ref.astype(int)).max() <= 1


def test_pack_bytes_equal_oracle(built):
    """Pack alone on the same float image, byte for byte (canvas.rs:176-186: 0xFF * clamp,
    rounded toward zero). The image holds every k/255 with its float neighbours (where the
    truncation decides between k - 1 and k), 0, -0, 1 and its neighbours, NaN, infinities,
    denormals, huge values and uniform randoms in [-0.5, 1.5]."""
    ctx = P.Context(0)
    k = np.arange(256, dtype=np.float32) / np.float32(255)
    edge = np.concatenate([k, np.nextafter(k, np.float32(-1)), np.nextafter(k, np.float32(2))])
    special = np.array([0.0, -0.0, 1.0, np.nextafter(np.float32(1), np.float32(2)),
                        np.nextafter(np.float32(1), np.float32(0)), np.nan, np.inf, -np.inf, 1e-45, -1e-45,
                        1e-38, 3e38, -3e38, 0.5, 254.5 / 255, 254.99998 / 255], dtype=np.float32)
    rnd = np.random.default_rng(5).uniform(-0.5, 1.5, 40000).astype(np.float32)
    img = np.concatenate([edge, special, rnd]).astype(np.float32)
    img = np.concatenate([img, np.zeros((-len(img)) % 4, dtype=np.float32)]).reshape(-1, 4)
    n = img.shape[0]
    want = oracle.pack(img)
    image = torch.from_numpy(img.reshape(-1).copy()).to(ctx.device)
    packed = torch.empty(n * 4, dtype=torch.uint8, device=ctx.device)
    _lib.call("htc_pack", n, 1, image.data_ptr(), packed.data_ptr(), ctx.stream())
    torch.cuda.synchronize()
    got = packed.cpu().numpy().reshape(-1, 4)
    bad = np.nonzero(np.any(got != want, axis=1))[0]
    assert bad.size == 0, f"{bad.size} pixels differ, first {img[bad[:4]]} -> {got[bad[:4]]} vs {want[bad[:4]]}"


@pytest.mark.parametrize("aw", [32, 64])
@pytest.mark.parametrize("cfg", ["config1", "config0"])
def test_double_support_scene_renders_as_its_f32_serialization(built, cfg, aw):
    """A scene serialized with double_support (8-byte f64 fields, f64 vectors and maps aligned
    to their size) is narrowed on the device to the f32 layout, each f64 rounded to the
    nearest f32 -- what the reference serializes without double_support -- and renders bit
    for bit as the f32 serialization does (one-pass kernel and htc_render_passes)."""
    wl = getattr(S, cfg)()
    W, H = 96, 64
    out = []
    for double in (False, True):
        ctx = P.Context(0, P.Config(address_width=aw, double_support=double))
        buf = P.EntityBuffer(ctx, wl.scene)
        r = P.Render(ctx, wl.scene.recipe, wl.scene.hops)
        a = P.Canvas(ctx, (W, H), global_seed=wl.global_seed)
        r.render(buf, a)
        r.render_passes(buf, a, 3)
        torch.cuda.synchronize()
        out.append((buf.size, r.static_size(), a.image.cpu().numpy().view(np.uint32).copy(), a.seeds.cpu().numpy().copy()))
    (fsize, fstatic, fimg, fseeds), (dsize, dstatic, dimg, dseeds) = out
    assert dsize > fsize and dstatic > fstatic   # the double layout is larger
    assert np.array_equal(fseeds, dseeds)
    assert np.array_equal(fimg, dimg)


def test_double_support_bad_object_count_is_reported(built):
    wl = S.config1()
    ctx = P.Context(0, P.Config(double_support=True))
    buf = P.EntityBuffer(ctx, wl.scene)
    data = bytearray(buf.tensor.cpu().numpy().tobytes())
    data[192:196] = (10_000).to_bytes(4, "little")   # object count of the double layout
    buf.tensor.copy_(torch.frombuffer(data, dtype=torch.uint8).to(ctx.device))
    r = P.Render(ctx, wl.scene.recipe, wl.scene.hops)
    with pytest.raises(_lib.HtcError) as e:
        r.render(buf, P.Canvas(ctx, (16, 16)))
    assert e.value.code == _lib.HTC_ERR_SCENE


def test_invalid_scene_is_reported(built):
    ctx = P.Context(0)
    wl = S.config1()
    data = bytearray(wl.scene.to_bytes())
    data[96:100] = (10_000).to_bytes(4, "little")   # object count beyond the buffer
    buf = P.EntityBuffer(ctx, wl.scene)
    buf.tensor.copy_(torch.frombuffer(data, dtype=torch.uint8).to(ctx.device))
    canvas = P.Canvas(ctx, (32, 32))
    r = P.Render(ctx, wl.scene.recipe, wl.scene.hops)
    with pytest.raises(_lib.HtcError) as e:
        r.render(buf, canvas)
    assert e.value.code == _lib.HTC_ERR_SCENE
    # the program stays usable afterwards
    good = P.EntityBuffer(ctx, wl.scene)
    r.render(good, canvas)


GOLDEN = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", ["euclidean_320x240", "hyperbolic_800x600", "hyperbolic_1920x1080_200obj",
                                  "hyperbolic_empty", "hyperbolic_onehop", "euclidean_1px"])
@pytest.mark.parametrize("form", ["render", "render_passes"])
def test_render_matches_golden(built, name, form):
    """Against fixtures produced by the reference's own kernel code (g++ draw order)."""
    import os
    f = np.load(os.path.join(GOLDEN, name + ".npz"))
    W, H, passes = int(f["width"]), int(f["height"]), int(f["passes"])
    pix = f["pixels"]
    ctx = P.Context(0)
    scene = torch.from_numpy(f["scene"].copy()).to(ctx.device)
    canvas = torch.zeros(W * H * 4, dtype=torch.float32, device=ctx.device)
    seeds = np.zeros(W * H, dtype=np.uint32)
    seeds[pix] = f["seeds_in"]
    seeds_t = torch.from_numpy(seeds.view(np.int32)).to(ctx.device)
    stats = torch.zeros(8, dtype=torch.int64, device=ctx.device)
    r = P.Render(ctx, int(f["recipe"]), int(f["hops"]), _lib.HTC_FLAG_JITTER_YX)
    if form == "render_passes":
        _lib.call("htc_render_passes", r.handle, W, H, scene.data_ptr(), scene.numel(), canvas.data_ptr(),
                  seeds_t.data_ptr(), passes, None, ctx.stream())
    else:
        for _ in range(passes):
            _lib.call("htc_render", r.handle, W, H, scene.data_ptr(), scene.numel(), canvas.data_ptr(),
                      seeds_t.data_ptr(), ctx.stream())
    _lib.call("htc_program_check", r.handle, ctx.stream())
    cv = canvas.cpu().numpy().reshape(-1, 4)[pix]
    sd = seeds_t.cpu().numpy().view(np.uint32)[pix]

    class Ref:
        canvas = f["canvas_out"]
        seeds = f["seeds_out"]
    _compare(cv, sd, Ref, f"golden {name} {form}")
