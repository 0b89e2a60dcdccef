"""CUDA graphs of batch calls (gcf_set_graphs): a repeated call is captured
once and replayed as one graph launch, with the eager call's results bit
for bit -- also after the image contents change in place, and for host
images in page-locked memory."""
import numpy as np
import pytest

from gctffind_b200 import synth

pytestmark = pytest.mark.gpu


def _specs(n, seed):
    rng = np.random.default_rng(seed)
    sizes = ((1536, 1536), (2048, 1536), (1280, 1792))
    out = []
    for k in range(n):
        w, h = sizes[k % len(sizes)]
        px = float(rng.uniform(0.9, 1.5))
        df = float(rng.uniform(9000.0, 30000.0))
        ast = float(rng.uniform(0.0, 800.0))
        out.append(synth.MicrographSpec(width=w, height=h, pixel_size=px, df_min=df - ast / 2, df_max=df + ast / 2,
                                        azimuth_deg=float(rng.uniform(-90, 90)), dose=1.5, seed=seed * 50 + k))
    return out


def _same(a, b):
    return [r.as_dict() for r in a] == [r.as_dict() for r in b]


@pytest.mark.parametrize("mode_name", ["GCF_SEARCH_PLAIN", "GCF_SEARCH_BF16"])
def test_graph_replay_matches_eager(gpu_lib, mode_name):
    import torch
    G = gpu_lib
    mode = getattr(G, mode_name)
    specs = _specs(6, 31)
    imgs = [synth.make_micrograph(s, device="cuda") for s in specs]
    pxs = [s.pixel_size for s in specs]
    op = G.make_optics()
    eager_ctx = G.Context(0, 512, 0)
    eager_ctx.run_batch(imgs, pxs, op, mode=mode)   # first call also makes tables / model rows
    eager = eager_ctx.run_batch(imgs, pxs, op, mode=mode)
    eager_launches = eager_ctx.launch_count()
    ctx = G.Context(0, 512, 0)
    ctx.set_graphs(True)
    seen = []
    for _ in range(4):
        res = ctx.run_batch(imgs, pxs, op, mode=mode)
        assert _same(res, eager)
        seen.append(ctx.graph_info()["graph_launches"])
    # first call eager, then captured and replayed
    assert seen == [0, 1, 1, 1], ctx.graph_info()
    info = ctx.graph_info()
    assert info["nodes"] > 0 and info["kernels"] == eager_launches
    assert ctx.stage_times()["total"] > 0
    # new contents in the same buffers: the replay computes them
    imgs[0].copy_(synth.make_micrograph(_specs(1, 77)[0], device="cuda")[:imgs[0].shape[0], :imgs[0].shape[1]])
    imgs[3].mul_(1.5)
    torch.cuda.synchronize()
    res = ctx.run_batch(imgs, pxs, op, mode=mode)
    assert ctx.graph_info()["graph_launches"] == 1
    assert _same(res, eager_ctx.run_batch(imgs, pxs, op, mode=mode))
    # another batch: eager again, its own graph from its second call on
    res2 = ctx.run_batch(imgs[:3], pxs[:3], op, mode=mode)
    assert ctx.graph_info()["graph_launches"] == 0
    ref2 = eager_ctx.run_batch(imgs[:3], pxs[:3], op, mode=mode)
    assert _same(res2, ref2)
    # calls that alternate between batches and methods never replay another
    # call's graph
    ref1 = eager_ctx.run_batch(imgs, pxs, op, mode=mode)
    other = G.GCF_SEARCH_BF16 if mode == G.GCF_SEARCH_PLAIN else G.GCF_SEARCH_PLAIN
    ref3 = eager_ctx.run_batch(imgs[:3], pxs[:3], op, mode=other)
    for args, ref in [((imgs[:3], pxs[:3], mode), ref2), ((imgs[:3], pxs[:3], mode), ref2),
                      ((imgs, pxs, mode), ref1), ((imgs[:3], pxs[:3], other), ref3),
                      ((imgs[:3], pxs[:3], other), ref3), ((imgs[:3], pxs[:3], mode), ref2),
                      ((imgs, pxs, mode), ref1)]:
        assert _same(ctx.run_batch(args[0], args[1], op, mode=args[2]), ref), ctx.graph_info()
    ctx.close()
    eager_ctx.close()


def test_graph_pinned_host_inputs(gpu_lib):
    G = gpu_lib
    specs = _specs(3, 41)
    host = [synth.make_micrograph(s, device="cpu").pin_memory() for s in specs]
    pxs = [s.pixel_size for s in specs]
    op = G.make_optics()
    ref_ctx = G.Context(0, 512, 0)
    ref = ref_ctx.run_batch(host, pxs, op, mode=G.GCF_SEARCH_BF16)
    ctx = G.Context(0, 512, 0)
    ctx.set_graphs(True)
    for k in range(3):
        assert _same(ctx.run_batch(host, pxs, op, mode=G.GCF_SEARCH_BF16), ref)
        assert ctx.graph_info()["graph_launches"] == (0 if k == 0 else 1), ctx.graph_info()
    # pageable host memory never takes a graph
    pageable = [h.clone().numpy() for h in host]
    for _ in range(2):
        assert _same(ctx.run_batch(pageable, pxs, op, mode=G.GCF_SEARCH_BF16), ref)
        assert ctx.graph_info()["graph_launches"] == 0
    ctx.close()
    ref_ctx.close()


def test_autotune_picks_the_fastest_trial_and_keeps_results(gpu_lib):
    """gcf_autotune: its picks are the fastest of its timed trials; the
    tile-kernel shape does not change any spectrum (the work items and the
    order of every sum are shape-independent), and the product tile changes
    no result beyond the BF16 table's own rounding."""
    G = gpu_lib
    ctx = G.Context(0, 512, 0)
    t = ctx.autotune()
    fm = {k: v for k, v in t["fused_ms"].items() if v > 0}
    gm = {k: v for k, v in t["gemm_ms"].items() if v > 0}
    assert fm and gm
    assert str(t["fused_shape"]) == min(fm, key=fm.get)
    picked = ("p" if t["gemm_persistent"] else "") + f'{t["gemm_tile_n"]}x{t["gemm_stages"]}'
    assert picked == min(gm, key=gm.get)
    # cached: a second call (another context) returns the same picks without trials
    other = G.Context(0, 512, 0)
    assert other.autotune() == t
    other.close()
    specs = _specs(4, 53)
    imgs = [synth.make_micrograph(s, device="cuda") for s in specs]
    pxs = [s.pixel_size for s in specs]
    op = G.make_optics()
    ref_ctx = G.Context(0, 512, 0)
    for shape in (8, 816):
        ref_ctx.set_fused_shape(shape)
        a = ref_ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_PLAIN)
        b = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_PLAIN)
        assert _same(a, b)
    a = ref_ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_BF16)
    b = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_BF16)
    for x, y in zip(a, b):
        step = max(20.0, 0.105 * 0.5 * (x.df_min + x.df_max) / 31.0)
        assert abs(x.df_min - y.df_min) <= step and abs(x.df_max - y.df_max) <= step
        assert abs(x.score - y.score) <= 2e-3
    ctx.close()
    ref_ctx.close()
