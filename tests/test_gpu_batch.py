"""Batched launches: every view's result equals rendering it alone (bit for bit), for a
mix of recipes, sizes and pass counts, directly and through the captured CUDA graph."""
import numpy as np
import pytest
import torch

from hypertrace_b200 import batch as B
from hypertrace_b200 import processing as P
from hypertrace_b200 import scene as S

pytestmark = pytest.mark.gpu


def _views(seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for i, (w, h) in enumerate([(64, 48), (37, 29), (128, 72), (16, 16), (96, 40), (50, 50)]):
        if i % 2 == 0:
            sc = S.euclidean_scene(int(rng.integers(2, 9)), 4, 100 + i, camera=B.random_hom3(rng))
        else:
            sc = S.hyperbolic_scene(int(rng.integers(2, 30)), int(rng.integers(2, 40)), 5.0, 8, 200 + i,
                                    camera=S.random_moebius(rng, 1.0))
        out.append(B.View(sc, w, h, 4, 1000 + i))
    return out


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("tile", [64, 1000])
def test_batch_equals_alone(built, graph, tile):
    ctx = P.Context(0)
    views = _views()
    alone = _views()
    for v in views + alone:
        v.allocate(ctx)
    passes = [1, 3, 2, 4, 1, 2]
    br = B.BatchRenderer(ctx, max_views=16)
    br.set_views(views, passes, tile_pixels=tile, blocks_per_sm=0)
    for _ in range(2):
        br.render(graph=graph)
    br.check()
    for v, p in zip(alone, passes):
        r = P.Render(ctx, v.scene.recipe, v.scene.hops)
        r.render_passes(v.buffer, v.canvas, 2 * p)
    torch.cuda.synchronize()
    for a, b in zip(views, alone):
        assert torch.equal(a.canvas.seeds, b.canvas.seeds)
        assert np.array_equal(a.canvas.image.cpu().numpy().view(np.uint32), b.canvas.image.cpu().numpy().view(np.uint32))


def test_batch_zero_pass_view_untouched(built):
    ctx = P.Context(0)
    views = _views()[:3]
    for v in views:
        v.allocate(ctx)
    before = views[1].canvas.image.clone()
    br = B.BatchRenderer(ctx, max_views=4)
    br.set_views(views, [1, 0, 1], tile_pixels=256)
    br.render()
    br.check()
    torch.cuda.synchronize()
    assert torch.equal(before, views[1].canvas.image)


def test_batch_autotune_restores_state(built):
    ctx = P.Context(0)
    views = _views()
    for v in views:
        v.allocate(ctx)
    snap = [v.canvas.seeds.clone() for v in views]
    br = B.BatchRenderer(ctx, max_views=16)
    tile, res, t = B.autotune(br, views, tiles=(128, 1024), residency=(4, 6))
    assert (tile, res) in t and len(t) == 4
    for v, s in zip(views, snap):
        assert torch.equal(v.canvas.seeds, s)


def test_batch_large_views_adaptive_tiles(built):
    """Views large enough that launches pick tiles above 128 slots (two 1920x1080 views and a
    small one), queues sized by htc_batch_reserve: equal to each view rendered alone."""
    def make():
        return [B.View(S.hyperbolic_scene(30, 45, 6.0, 8, 77, camera=S.random_moebius(np.random.default_rng(3), 1.0)),
                       1920, 1080, 2, 901),
                B.View(S.euclidean_scene(8, 4, 78, camera=B.random_hom3(np.random.default_rng(4))), 1920, 1080, 2, 902),
                B.View(S.hyperbolic_scene(5, 7, 5.0, 8, 79), 96, 40, 2, 903)]
    ctx = P.Context(0)
    views, alone = make(), make()
    for v in views + alone:
        v.allocate(ctx)
    br = B.BatchRenderer(ctx, max_views=8)
    br.reserve(2 * 1920 * 1080 + 96 * 40, 8)
    br.set_views(views, [2, 2, 2], tile_pixels=2048, blocks_per_sm=0)
    br.render()
    br.check()
    for v in alone:
        P.Render(ctx, v.scene.recipe, v.scene.hops).render_passes(v.buffer, v.canvas, 2)
    torch.cuda.synchronize()
    for a, b in zip(views, alone):
        assert torch.equal(a.canvas.seeds, b.canvas.seeds)
        assert torch.equal(a.canvas.image.view(torch.int32), b.canvas.image.view(torch.int32))


def test_batch_mixed_hop_counts(built):
    """Views of 1, 2, 3 and 5 light hops in one batch (hop-depth launches past a view's H find
    no paths of it): each equal to the view rendered alone."""
    def make():
        return [B.View(S.hyperbolic_scene(6, 9, 5.0, 1, 61), 70, 30, 3, 701),
                B.View(S.euclidean_scene(5, 2, 62), 40, 40, 2, 702),
                B.View(S.hyperbolic_scene(12, 15, 5.0, 5, 63), 50, 66, 4, 703),
                B.View(S.euclidean_scene(3, 3, 64), 33, 17, 1, 704)]
    ctx = P.Context(0)
    views, alone = make(), make()
    for v in views + alone:
        v.allocate(ctx)
    br = B.BatchRenderer(ctx, max_views=8)
    br.set_views(views, [v.spp for v in views], tile_pixels=512)
    br.render(graph=True)
    br.check()
    for v in alone:
        P.Render(ctx, v.scene.recipe, v.scene.hops).render_passes(v.buffer, v.canvas, v.spp)
    torch.cuda.synchronize()
    for a, b in zip(views, alone):
        assert torch.equal(a.canvas.seeds, b.canvas.seeds)
        assert torch.equal(a.canvas.image.view(torch.int32), b.canvas.image.view(torch.int32))


def test_batch_graph_recaptures_for_new_stats_and_grown_queues(built):
    """The captured graph's kernels hold the stats pointer and the queue buffers: a launch
    with another stats buffer, and one after htc_batch_reserve grew the queues, capture anew —
    the new buffer gets the statistics, the old one stays as it was, and the results still
    equal the views rendered alone."""
    ctx = P.Context(0)
    views, alone = _views(5), _views(5)
    for v in views + alone:
        v.allocate(ctx)
    br = B.BatchRenderer(ctx, max_views=16)
    br.set_views(views, [2] * len(views), tile_pixels=256, blocks_per_sm=0)
    s1 = torch.zeros(8, dtype=torch.int64, device=ctx.device)
    s2 = torch.zeros(8, dtype=torch.int64, device=ctx.device)
    br.render(stats=s1, graph=True)
    torch.cuda.synchronize()
    first = s1.clone()
    br.render(stats=s2, graph=True)
    torch.cuda.synchronize()
    assert torch.equal(s1, first)   # the second launch wrote to s2 only
    n = 2 * sum(v.width * v.height for v in views)   # samples of two passes of every view
    assert int(first[0]) == n and int(s2[0]) == n and int(s2[1]) > 0
    br.reserve(4 * 1920 * 1080, 8)   # grows the queues (and the sort buffers) after a capture
    br.render(stats=s2, graph=True)
    br.check()
    for v in alone:
        P.Render(ctx, v.scene.recipe, v.scene.hops).render_passes(v.buffer, v.canvas, 6)
    torch.cuda.synchronize()
    assert int(s2[0]) == 2 * n and torch.equal(s1, first)
    for a, b in zip(views, alone):
        assert torch.equal(a.canvas.seeds, b.canvas.seeds)
        assert torch.equal(a.canvas.image.view(torch.int32), b.canvas.image.view(torch.int32))
