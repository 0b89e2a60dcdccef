"""The BF16 contraction search (gcf_run_batch_mode, GCF_SEARCH_BF16) against
the plain FP32 search (GCF_SEARCH_PLAIN) of the same batch.

The contraction scores every candidate of every micrograph on a BF16
tensor-core table, so its optimum may sit a little off the plain search's;
the FP32 re-score and local passes then refine on each micrograph's own
band.  Accuracy bar: defocus within one search step of the
plain path's last mean-defocus line search (max(20 A, 0.105 * mean / 31))
for at least 99 % of micrographs -- here every one of the batch -- with a
median |d defocus| <= 20 A; azimuth within 2 degrees (mod 180) where the
astigmatism exceeds 200 A; the re-scored CC no lower than the plain one
minus 2e-3 (both are FP32 CCs with FP64 sums on the same band).
"""
import numpy as np
import pytest

from gctffind_b200 import synth

pytestmark = pytest.mark.gpu


def _ang(a, b):
    d = (a - b) % 180.0
    return min(d, 180.0 - d)


def _batch(n, seed, sizes=((2048, 2048), (2880, 2046), (1919, 1855))):
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n):
        w, h = sizes[int(rng.integers(0, len(sizes)))]
        px = float(rng.uniform(0.8, 1.5))
        px_n = max(px, 1.2)
        df = float(rng.uniform(max(5000.0, 3300.0 * px_n * px_n), 40000.0))
        ast = float(rng.uniform(0.0, 1000.0))
        ang = float(rng.uniform(-90.0, 90.0))
        specs.append(synth.MicrographSpec(width=w, height=h, pixel_size=px, df_min=df - ast / 2,
                                          df_max=df + ast / 2, azimuth_deg=ang,
                                          dose=float(rng.uniform(0.5, 2.0)), seed=seed * 100 + k))
    return specs


def _compare(plain, fast, specs):
    ddf = []
    for p, f, s in zip(plain, fast, specs):
        mp, mf = 0.5 * (p.df_min + p.df_max), 0.5 * (f.df_min + f.df_max)
        step = max(20.0, 0.105 * mp / 31.0)
        assert abs(f.df_min - p.df_min) <= step and abs(f.df_max - p.df_max) <= step, (p, f, step)
        if p.df_max - p.df_min > 200.0:
            assert _ang(f.azimuth, p.azimuth) <= 2.0, (p, f)
        assert f.score >= p.score - 2e-3, (p, f)
        ddf.append(abs(mf - mp))
    return float(np.median(ddf))


def test_bf16_search_matches_plain(gpu_lib):
    import torch
    G = gpu_lib
    specs = _batch(16, 5)
    imgs = [synth.make_micrograph(s, device="cuda") for s in specs]
    pxs = [s.pixel_size for s in specs]
    ctx = G.Context(0, 512, 0)
    op = G.make_optics()
    plain = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_PLAIN)
    plain_counts = ctx.search_counts()
    fast = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_BF16)
    fc = ctx.fast_counts()
    fast_counts = ctx.search_counts()
    ctx.close()
    med = _compare(plain, fast, specs)
    assert med <= 20.0, med
    # the contraction's work: every micrograph scored on the table, a few
    # candidates re-scored in FP32
    assert fc["table_cand"] > 16 * 1000 and fc["tensor_macs"] > 0
    assert fc["rescored"] == 16 * (4 + 27 * 4)
    assert fast_counts["cand2d"] < plain_counts["cand2d"] / 20
    torch.cuda.empty_cache()


def test_bf16_search_host_inputs_and_repeat(gpu_lib):
    """Host inputs give the device inputs' results, and a second call (the
    model rows kept from the first) repeats them bit for bit."""
    G = gpu_lib
    specs = _batch(6, 9)
    imgs = [synth.make_micrograph(s, device="cpu").numpy() for s in specs]
    pxs = [s.pixel_size for s in specs]
    ctx = G.Context(0, 512, 0)
    op = G.make_optics()
    a = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_BF16)
    import torch
    b = ctx.run_batch([torch.from_numpy(x).cuda() for x in imgs], pxs, op, mode=G.GCF_SEARCH_BF16)
    c = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_BF16)
    ctx.close()
    for x, y, z in zip(a, b, c):
        assert x.as_dict() == y.as_dict() == z.as_dict()


def test_bf16_mode_rejects_bad_mode(gpu_lib):
    G = gpu_lib
    ctx = G.Context(0, 512, 0)
    img = np.zeros((1024, 1024), np.float32)
    with pytest.raises(G.GcfError):
        ctx.run_batch([img], [1.35], G.make_optics(), mode=7)
    ctx.close()
