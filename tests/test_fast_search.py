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


@pytest.mark.parametrize("tile", [256, 1024])
def test_bf16_search_other_tile_sizes(gpu_lib, tile):
    """The contraction bins whatever half spectrum the tile size gives (the
    batched-cuFFT spectrum at tiles 256 and 1024): the BF16 search still lands within one search
    step of the plain search of the same batch for at least 7 of 8
    micrographs, with a median |d defocus| <= 30 A."""
    G = gpu_lib
    specs = _batch(8, 21)
    imgs = [synth.make_micrograph(s, device="cuda") for s in specs]
    pxs = [s.pixel_size for s in specs]
    ctx = G.Context(0, tile, 0)
    op = G.make_optics()
    plain = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_PLAIN)
    fast = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_BF16)
    ctx.close()
    within, ddf = 0, []
    for p, f in zip(plain, fast):
        mp = 0.5 * (p.df_min + p.df_max)
        step = max(20.0, 0.105 * mp / 31.0)
        within += abs(f.df_min - p.df_min) <= step and abs(f.df_max - p.df_max) <= step
        ddf.append(abs(0.5 * (f.df_min + f.df_max) - mp))
    assert within >= 7, (tile, within, plain, fast)
    assert float(np.median(ddf)) <= 30.0, ddf


def test_phase_plate_data_take_the_plain_search(gpu_lib):
    """The table has no extra-phase dimension: with ext_phase_range > 0 the
    BF16 and learned methods return the plain search's results bit for bit."""
    G = gpu_lib
    specs = _batch(3, 33)
    imgs = [synth.make_micrograph(s, device="cuda") for s in specs]
    pxs = [s.pixel_size for s in specs]
    ctx = G.Context(0, 512, 0)
    G.load_learned(ctx)
    op = G.make_optics(ext_phase_deg=40.0, ext_phase_range=60.0)
    plain = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_PLAIN)
    for mode in (G.GCF_SEARCH_BF16, G.GCF_SEARCH_LEARNED):
        fast = ctx.run_batch(imgs, pxs, op, mode=mode)
        assert [r.as_dict() for r in fast] == [r.as_dict() for r in plain]
    ctx.close()


def test_learned_batch_over_one_network_chunk(gpu_lib):
    """520 micrographs in one learned call: the network runs in chunks of
    512 spectra, and every micrograph -- those of the second chunk included
    -- lands within one search step of the plain search for >= 97 % of the
    batch, median |d defocus| <= 20 A."""
    import torch
    G = gpu_lib
    n = 520
    specs = _batch(n, 44, sizes=((1536, 1536),))
    for s in specs:
        s.dose = max(s.dose, 1.5)
    imgs = [synth.make_micrograph(s, device="cuda") for s in specs]
    pxs = [s.pixel_size for s in specs]
    ctx = G.Context(0, 512, 0)
    G.load_learned(ctx)
    op = G.make_optics()
    plain = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_PLAIN)
    fast = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_LEARNED)
    ctx.close()
    within, ddf = [], []
    for p, f in zip(plain, fast):
        mp = 0.5 * (p.df_min + p.df_max)
        step = max(20.0, 0.105 * mp / 31.0)
        within.append(abs(f.df_min - p.df_min) <= step and abs(f.df_max - p.df_max) <= step)
        ddf.append(abs(0.5 * (f.df_min + f.df_max) - mp))
    assert np.mean(within) >= 0.97 and np.mean(within[512:]) >= 0.75, (np.mean(within), within[512:])
    assert float(np.median(ddf)) <= 20.0
    del imgs
    torch.cuda.empty_cache()


@pytest.mark.parametrize("mode_name", ["GCF_SEARCH_BF16", "GCF_SEARCH_LEARNED"])
def test_fast_methods_on_a_single_micrograph(gpu_lib, mode_name):
    """A batch of one: the table has one micrograph's angle bins, the tile
    plan one column block; the result within one search step of the plain
    search."""
    G = gpu_lib
    spec = synth.MicrographSpec(width=2048, height=2048, pixel_size=1.3, df_min=21800.0, df_max=22400.0,
                                azimuth_deg=-35.0, dose=2.0, seed=808)
    img = synth.make_micrograph(spec, device="cuda")
    ctx = G.Context(0, 512, 0)
    if mode_name == "GCF_SEARCH_LEARNED":
        G.load_learned(ctx)
    op = G.make_optics()
    p = ctx.run_batch([img], [1.3], op, mode=G.GCF_SEARCH_PLAIN)[0]
    f = ctx.run_batch([img], [1.3], op, mode=getattr(G, mode_name))[0]
    ctx.close()
    step = max(20.0, 0.105 * 0.5 * (p.df_min + p.df_max) / 31.0)
    assert abs(f.df_min - p.df_min) <= step and abs(f.df_max - p.df_max) <= step, (p, f)
    assert f.score >= p.score - 2e-3
