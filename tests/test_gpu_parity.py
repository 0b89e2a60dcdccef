"""GPU parity: the CUDA path (through the C ABI) against the FP64 oracle.

Tolerances (the path's accuracy bar: averaged spectra within 1e-4 relative,
defocus within one reference search step, astigmatism angle within 1 degree,
CC within 1e-3):
  raw averaged spectrum : |gpu - orc| <= 1e-4 * |orc| + 1e-5 * mean(orc) per pixel
  ctf spectrum          : |gpu - orc| <= 1e-4 * rms(orc) per pixel
  radial average        : |gpu - orc| <= 1e-4 * rms(orc) per bin
  search results        : |d df| <= one search step (the last DfMean step,
                          max(20 A, range/31) <= 60 A here), |d azimuth| <= 1 deg
                          (modulo 180), |d CC| <= 1e-3
"""
import numpy as np
import pytest

from gctffind_b200 import synth

pytestmark = pytest.mark.gpu

TILE = 256
PX = 1.35


def _img(seed=3, w=1024, h=1024, px=PX, df=(14800.0, 15200.0), az=20.0, dose=3.0, tilt=0.0):
    spec = synth.MicrographSpec(width=w, height=h, pixel_size=px, df_min=df[0], df_max=df[1],
                                azimuth_deg=az, dose=dose, seed=seed, tilt_deg=tilt)
    return synth.make_micrograph(spec).numpy()


def _ang_diff(a, b):
    d = (a - b) % 180.0
    return min(d, 180.0 - d)


def _assert_result_close(g, o, df_tol=60.0, ang_tol=1.0, cc_tol=1e-3):
    assert abs(g.df_min - o.df_min) <= df_tol, (g, o.as_dict())
    assert abs(g.df_max - o.df_max) <= df_tol, (g, o.as_dict())
    if abs(o.df_max - o.df_min) > 50.0:   # azimuth is meaningless without astigmatism
        assert _ang_diff(g.azimuth, o.azimuth) <= ang_tol, (g, o.as_dict())
    assert abs(g.score - o.score) <= cc_tol, (g, o.as_dict())


@pytest.fixture(scope="module")
def case(gpu_lib, oracle):
    G = gpu_lib
    img = _img()
    ctx = G.Context(0, TILE, 0)
    op = G.make_optics(pixel_size=PX)
    ctx.setup(op, img.shape[1], img.shape[0])
    ctx.gen_half_spectrum(img)
    p = oracle.params(pixel_size=PX, tile_size=TILE)
    ores, oraw, octf, ofull = oracle.find_ctf_image(img, PX, p, want_spectra=True)
    return dict(G=G, ctx=ctx, img=img, op=op, p=p, ores=ores, oraw=oraw, octf=octf, ofull=ofull)


def test_raw_spectrum_matches_oracle(case):
    g = case["ctx"].half_spectrum(raw=True).astype(np.float64)
    o = case["oraw"]
    tol = 1e-4 * np.abs(o) + 1e-5 * o.mean()
    err = np.abs(g - o)
    assert np.all(err <= tol), float((err / (np.abs(o) + 1e-30)).max())


def test_ctf_spectrum_matches_oracle_given_gpu_raw(case, oracle):
    # isolate background + lowpass: oracle fed with the GPU raw spectrum
    graw = case["ctx"].half_spectrum(raw=True).astype(np.float64)
    octf, lp = oracle.ctf_spectrum(graw, 0)
    g = case["ctx"].half_spectrum(raw=False).astype(np.float64)
    rms = np.sqrt(np.mean(octf ** 2))
    assert lp == 1
    assert np.max(np.abs(g - octf)) <= 1e-4 * rms


def test_lowpass512_matches_oracle_and_cufft_variant(gpu_lib, oracle):
    """Tile 512: the separable warp-FFT lowpass (rows, then columns, each
    pair of real lines as one complex FFT) against the oracle's background
    removal + FP64 lowpass of the same raw spectrum, and against the
    batched-cuFFT comparison variant (2D R2C / C2R), both within 1e-4 of the
    rms per pixel; the variance gate (faint image) keeps the unfiltered
    spectrum in both variants."""
    G = gpu_lib
    img = _img(seed=17, w=1536, h=1536)
    out = {}
    for impl in (G.GCF_SPECT_FUSED, G.GCF_SPECT_CUFFT):
        ctx = G.Context(0, 512, 0)
        ctx.set_spectrum_impl(impl)
        ctx.setup(G.make_optics(pixel_size=PX), 1536, 1536)
        ctx.gen_half_spectrum(img)
        graw = ctx.half_spectrum(raw=True).astype(np.float64)
        g = ctx.half_spectrum(raw=False).astype(np.float64)
        octf, lp = oracle.ctf_spectrum(graw, 0)
        assert lp == 1
        rms = np.sqrt(np.mean(octf ** 2))
        assert np.max(np.abs(g - octf)) <= 1e-4 * rms, impl
        out[impl] = g
        # the variance gate: a faint image keeps the background-removed spectrum
        faint = img * np.float32(1e-4)
        ctx.gen_half_spectrum(faint)
        fraw = ctx.half_spectrum(raw=True).astype(np.float64)
        fctf, flp = oracle.ctf_spectrum(fraw, 0)
        assert flp == 0
        f = ctx.half_spectrum(raw=False).astype(np.float64)
        assert np.max(np.abs(f - fctf)) <= 1e-4 * np.sqrt(np.mean(fctf ** 2)), impl
        ctx.close()
    a, b = out[G.GCF_SPECT_FUSED], out[G.GCF_SPECT_CUFFT]
    assert np.max(np.abs(a - b)) <= 1e-4 * np.sqrt(np.mean(b ** 2))


def test_radial_average_matches_oracle(case, oracle):
    g_ctf = case["ctx"].half_spectrum(raw=False).astype(np.float64)
    orad = oracle.radial_average(g_ctf)
    grad = case["ctx"].radial_average().astype(np.float64)
    rms = np.sqrt(np.mean(orad ** 2))
    assert np.max(np.abs(grad - orad)) <= 1e-4 * rms


def test_do2d_matches_oracle(case):
    r = case["ctx"].do2d()
    o = case["ores"]
    assert abs(r.df_1d - o.df_1d) <= 20.0, (r, o.as_dict())
    _assert_result_close(r, o)
    # and the synthetic truth (14800 / 15200 at 20 degrees) within 150 A / 3 degrees
    assert abs(r.df_min - 14800.0) < 150.0 and abs(r.df_max - 15200.0) < 150.0
    assert _ang_diff(r.azimuth, 20.0) < 3.0


def test_do1d_refine1d_match_oracle(case, oracle):
    """CFindCtf1D::Do1D / Refine1D on the GPU spectrum vs the oracle's 1D
    searches on the same spectrum: same grid point, CC within 1e-4."""
    ctx = case["ctx"]
    g_ctf = ctx.half_spectrum(raw=False).astype(np.float64)
    ctx.set_phase(0.0, 0.0)
    r1 = ctx.do1d()
    df, ph, sc = oracle.search1d(g_ctf, PX, case["p"])
    assert r1.df_min == r1.df_max == pytest.approx(df, abs=0.01)
    assert r1.score == pytest.approx(sc, abs=1e-4)
    ctx.set_phase(0.0, 0.0)
    r2 = ctx.refine1d(14000.0, 4000.0)
    df2, ph2, sc2 = oracle.refine1d(g_ctf, PX, case["p"], 14000.0, 4000.0)
    assert r2.df_min == pytest.approx(df2, abs=0.01)
    assert r2.score == pytest.approx(sc2, abs=1e-4)


def test_do2d_search_on_oracle_spectrum(case, oracle):
    # search alone: both sides on (nearly) the same spectrum
    r = case["ctx"].do2d()
    s = oracle.search(case["ctx"].half_spectrum(raw=False).astype(np.float64), PX, case["p"])
    _assert_result_close(r, s, df_tol=25.0, ang_tol=1.0, cc_tol=2e-4)


def test_search_counts_match_oracle(case, oracle):
    """gcf_get_search_counts: the 1D grid points and 2D candidates a Do2D
    evaluates on the device equal the oracle's count of GCC1D / GCC2D
    evaluations on the same spectrum (exactly when both searches end on the
    same grid point; the line-search windows follow the running best)."""
    ctx = case["ctx"]
    ctx.set_phase(0.0, 0.0)
    c0 = ctx.search_counts()
    r = ctx.do2d()
    c1 = ctx.search_counts()
    d = {k: c1[k] - c0[k] for k in c0}
    oracle.counts(reset=True)
    s = oracle.search(ctx.half_spectrum(raw=False).astype(np.float64), PX, case["p"])
    o2d, o1d = oracle.counts(reset=True)
    assert d["cand1d"] == o1d > 0
    assert d["pairs1d"] > d["cand1d"]
    assert d["cand2d"] > 2601                          # the 51 x 51 astigmatism grid and more
    assert d["pairs2d"] % d["cand2d"] == 0             # every candidate covers the whole band
    same = (r.df_min, r.df_max, r.azimuth, r.ext_phase) == (s.df_min, s.df_max, s.azimuth, s.ext_phase)
    if same:
        assert d["cand2d"] == o2d
    else:
        assert abs(d["cand2d"] - o2d) <= 0.02 * o2d


def test_refine_matches_oracle(case, oracle):
    ctx = case["ctx"]
    rin = [15100.0, 7550.0, 0.01, 0.04, 10.0, 30.0, 0.0, 0.0]
    r = ctx.refine(rin[0:2], rin[2:4], rin[4:6], rin[6:8])
    o = oracle.search(ctx.half_spectrum(raw=False).astype(np.float64), PX, case["p"], mode=1,
                      refine_in=rin)
    _assert_result_close(r, o, df_tol=25.0, cc_tol=2e-4)


def test_full_spectrum_matches_oracle(case, oracle):
    ctx = case["ctx"]
    r = ctx.do2d()
    g = ctx.full_spectrum(r).astype(np.float64)
    octf = ctx.half_spectrum(raw=False).astype(np.float64)
    ores = oracle.OrcResult(r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score, 0, 0, 0, 0, 1)
    o = oracle.full_spectrum(octf, PX, case["p"], ores).astype(np.float64)
    rms = np.sqrt(np.mean(o ** 2))
    assert np.max(np.abs(g - o)) <= 1e-4 * rms


def test_series_matches_oracle(gpu_lib, oracle):
    G = gpu_lib
    tilts = [-6.0, -3.0, 0.0, 3.0, 6.0]
    imgs = [_img(seed=10 + i, w=768, h=768, df=(19850.0, 20150.0), az=-35.0, tilt=t)
            for i, t in enumerate(tilts)]
    so = G.series_order(tilts)
    ctx = G.Context(0, TILE, 0)
    op = G.make_optics(pixel_size=PX)
    gres = ctx.run_series(imgs, op, so.order, is_tomo=True)
    p = oracle.params(pixel_size=PX, tile_size=TILE)
    ores = oracle.series(imgs, p, so.order, True)
    for g, o in zip(gres, ores):
        _assert_result_close(g, o)


def test_batch_mixed_sizes(gpu_lib, oracle):
    G = gpu_lib
    specs = [(768, 640, 1.35, (9900.0, 10100.0)), (1024, 768, 1.5, (24800.0, 25200.0))]
    imgs = [_img(seed=40 + i, w=w, h=h, px=px, df=df) for i, (w, h, px, df) in enumerate(specs)]
    ctx = G.Context(0, TILE, 0)
    op = G.make_optics()
    gres = ctx.run_batch(imgs, [s[2] for s in specs], op)
    for img, s, g in zip(imgs, specs, gres):
        p = oracle.params(pixel_size=s[2], tile_size=TILE)
        o = oracle.find_ctf_image(img, s[2], p)
        _assert_result_close(g, o)


@pytest.mark.parametrize("impl", ["GCF_RESCALE_CUFFT", "GCF_RESCALE_LINES"])
def test_rescale_matches_oracle(gpu_lib, oracle, impl):
    """The rescale (R2C, crop, C2R with each row's DC and Nyquist terms taken
    as real) against the oracle's FP64 restatement: max |d| <= 1e-5 x rms."""
    G = gpu_lib
    img = _img(seed=7, w=1024, h=1024, px=0.8, df=(9900.0, 10100.0))
    ctx = G.Context(0, TILE, 0)
    ctx.set_rescale_impl(getattr(G, impl))
    g = ctx.rescale(img, 0.8).astype(np.float64)
    ctx.close()
    o = oracle.rescale(img, 0.8).astype(np.float64)
    assert g.shape == o.shape == (682, 682)
    rel = np.abs(g - o).max() / np.sqrt((o * o).mean())
    assert rel <= 1e-5, rel


def test_errors_are_status_codes(gpu_lib):
    G = gpu_lib
    ctx = G.Context(0, TILE, 0)
    with pytest.raises(G.GcfError):
        ctx.do2d()   # no spectrum yet
    op = G.make_optics(pixel_size=PX)
    small = np.zeros((100, 100), np.float32)
    ctx.setup(op, 100, 100)
    with pytest.raises(G.GcfError):
        ctx.gen_half_spectrum(small)


# ---------------------------------------------------------------------------
# 512 x 512 tiles: the fused tile-FFT kernel (default) and the cuFFT variant
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("w", [1536, 1538])   # tile starts 16-byte aligned / not aligned
def test_fused_spectrum_matches_oracle_and_cufft(gpu_lib, oracle, w):
    G = gpu_lib
    img = _img(seed=21, w=w, h=1536, df=(17800.0, 18200.0), az=-10.0)
    op = G.make_optics(pixel_size=PX)
    fused = G.Context(0, 512, 0)   # fused is the default for 512
    fused.setup(op, w, 1536)
    fused.gen_half_spectrum(img)
    gf = fused.half_spectrum(raw=True).astype(np.float64)
    cuf = G.Context(0, 512, 0, spectrum_impl=G.GCF_SPECT_CUFFT)
    cuf.setup(op, w, 1536)
    cuf.gen_half_spectrum(img)
    gc = cuf.half_spectrum(raw=True).astype(np.float64)
    o = oracle.avg_spectrum(img, 512)
    tol = 1e-4 * np.abs(o) + 1e-5 * o.mean()
    assert np.all(np.abs(gf - o) <= tol), float((np.abs(gf - o) / np.abs(o)).max())
    assert np.all(np.abs(gc - o) <= tol), float((np.abs(gc - o) / np.abs(o)).max())
    r1, r2 = fused.do2d(), cuf.do2d()
    p = oracle.params(pixel_size=PX, tile_size=512)
    ores = oracle.find_ctf_image(img, PX, p)
    _assert_result_close(r1, ores)
    _assert_result_close(r2, ores)


def test_largest_frame_matches_oracle(gpu_lib, oracle):
    """A K3 super-resolution sized frame, 11520 x 8184 at 1.2 A/px (no
    rescale): 44 x 30 = 1320 tiles in 55 work items of one launch.  The
    averaged spectrum within the per-pixel tolerance and the Do2D result
    within one search step of the oracle's."""
    G = gpu_lib
    w, h, px = 11520, 8184, 1.2
    img = _img(seed=61, w=w, h=h, px=px, df=(21800.0, 22300.0), az=35.0, dose=1.5)
    ctx = G.Context(0, 512, 0)
    op = G.make_optics(pixel_size=px)
    ctx.setup(op, w, h)
    ctx.gen_half_spectrum(img)
    g = ctx.half_spectrum(raw=True).astype(np.float64)
    o = oracle.avg_spectrum(img, 512)
    tol = 1e-4 * np.abs(o) + 1e-5 * o.mean()
    assert np.all(np.abs(g - o) <= tol), float((np.abs(g - o) / np.abs(o)).max())
    ctx.set_phase(0.0, 0.0)
    r = ctx.do2d()
    ores = oracle.find_ctf_image(img, px, oracle.params(pixel_size=px, tile_size=512))
    _assert_result_close(r, ores)
    ctx.close()


def test_fused_batch_deterministic(gpu_lib):
    G = gpu_lib
    imgs = [_img(seed=30 + i, w=1024 + 512 * (i % 2), h=1024, df=(15000.0, 15100.0)) for i in range(3)]
    ctx = G.Context(0, 512, 0)
    op = G.make_optics()
    a = ctx.run_batch(imgs, [PX] * 3, op)
    b = ctx.run_batch(imgs, [PX] * 3, op)
    for x, y in zip(a, b):
        assert x.as_dict() == y.as_dict()


def test_every_cluster_shape_gives_the_same_spectrum(gpu_lib):
    """The tile kernel's cluster shapes (8, 816, 16, 162, 168) split a tile's
    rows and columns differently over CTAs and warps, but every FFT and every
    sum runs in the same order: the averaged spectrum is bit-identical."""
    G = gpu_lib
    img = _img(seed=44, w=2560, h=2048, df=(16800.0, 17300.0), az=25.0)
    op = G.make_optics(pixel_size=PX)
    out = {}
    for shape in (8, 816, 16, 162, 168):
        ctx = G.Context(0, 512, 0)
        ctx.set_fused_shape(shape)
        ctx.setup(op, 2560, 2048)
        ctx.gen_half_spectrum(img)
        out[shape] = ctx.half_spectrum(raw=True)
        ctx.close()
    for shape, g in out.items():
        assert np.array_equal(g, out[8]), shape


def test_cluster_less_ctas_do_not_change_spectra(gpu_lib):
    """Twelve 4096 x 4096 micrographs (10 work items each) through one
    gcf_run_batch call: with 120 items in one launch the cluster-less tile
    CTAs take items from the back of the queue while the clusters take the
    rest.  Each micrograph alone (10 items, clusters only) must give the same
    result fields bit for bit, since an item's partial spectrum does not
    depend on which kernel computed it."""
    import torch
    G = gpu_lib
    n = 12
    imgs = [torch.from_numpy(_img(seed=90 + i, w=4096, h=4096, df=(14600.0 + 150 * i, 15200.0 + 150 * i),
                                  az=10.0 * i)).cuda() for i in range(n)]
    ctx = G.Context(0, 512, 0)
    op = G.make_optics(pixel_size=PX)
    batch = ctx.run_batch(imgs, [PX] * n, op)
    for img, rb in zip(imgs, batch):
        ctx.setup(op, 4096, 4096)
        ctx.gen_half_spectrum(img)
        ctx.set_phase(0.0, 0.0)
        rs = ctx.do2d()
        assert [rs.df_min, rs.df_max, rs.azimuth, rs.score, rs.df_1d] == \
            [rb.df_min, rb.df_max, rb.azimuth, rb.score, rb.df_1d]
    ctx.close()


def _bg_curves(case):
    x = np.arange(257, dtype=np.float64)
    yield (1000 * np.exp(-x / 40) + 50 * np.cos(x / 3) ** 2 + 20).astype(np.float32)
    yield case["ctx"].radial_average().astype(np.float32)
    rng = np.random.default_rng(9)
    yield (500 / (1 + x / 10) + rng.uniform(0, 30, 257)).astype(np.float32)
    yield (2000 * np.exp(-np.arange(1025) / 150) + 5).astype(np.float32)


def test_background1d_matches_oracle(case, oracle):
    """GBackground1D: start and background bit-identical to the oracle
    (same double fit order, same float window sums), Remove1D identical,
    Remove2D to one float rounding (FMA in the interpolation)."""
    ctx = case["ctx"]
    for sp in _bg_curves(case):
        bg, st = ctx.background1d(sp)
        obg, ost = oracle.background1d(sp)
        assert st == ost
        assert np.array_equal(bg, obg)
        r1 = ctx.remove_background1d(sp, bg, st)
        assert np.array_equal(r1, oracle.remove_bg1d(sp, obg, ost))
    half = case["ctx"].half_spectrum(raw=True)
    sp = case["ctx"].radial_average().astype(np.float32)
    bg, st = ctx.background1d(sp)
    g2 = ctx.remove_background2d(half, bg, st)
    o2 = oracle.remove_bg2d(half, bg, st)
    assert np.allclose(g2, o2, rtol=1e-6, atol=1e-6 * np.abs(half).max())


def test_series_host_and_device_inputs_agree(gpu_lib):
    """gcf_run_series streams host inputs chunk by chunk (uploads overlapped
    with spectra and searches) and takes device inputs in one batch; both
    give bit-identical results and full spectra."""
    import torch
    G = gpu_lib
    tilts = [3.0 * (k - 5) for k in range(11)]
    imgs = [_img(seed=40 + k, w=1024, h=1024, df=(15000.0 + 30 * k, 15400.0 + 30 * k), tilt=t)
            for k, t in enumerate(tilts)]
    so = G.series_order(tilts)
    op = G.make_optics(pixel_size=PX)
    ctx = G.Context(0, 512, 0)
    rh, fh = ctx.run_series(imgs, op, so.order, is_tomo=True, want_full=True)
    dev = [torch.from_numpy(a).cuda() for a in imgs]
    rd, fd = ctx.run_series(dev, op, so.order, is_tomo=True, want_full=True)
    ctx.close()
    for a, b in zip(rh, rd):
        assert [a.df_min, a.df_max, a.azimuth, a.ext_phase, a.score] == \
            [b.df_min, b.df_max, b.azimuth, b.ext_phase, b.score]
    assert np.array_equal(fh, fd)


@pytest.mark.parametrize("n", [1, 2, 3])
def test_short_series_host_and_device_inputs_agree(gpu_lib, n):
    """Series of 1 to 3 packages: the device path splits a series into the
    first package and the rest (two tile launches with their cluster-less
    CTAs) and the host path into upload chunks; both must give the same rows."""
    import torch
    G = gpu_lib
    tilts = [3.0 * (k - n // 2) for k in range(n)]
    imgs = [_img(seed=70 + k, w=1024, h=1024, df=(15000.0 + 40 * k, 15400.0 + 40 * k), tilt=t)
            for k, t in enumerate(tilts)]
    so = G.series_order(tilts)
    op = G.make_optics(pixel_size=PX)
    ctx = G.Context(0, 512, 0)
    rh = ctx.run_series(imgs, op, so.order, is_tomo=True)
    rd = ctx.run_series([torch.from_numpy(a).cuda() for a in imgs], op, so.order, is_tomo=True)
    ctx.close()
    for a, b in zip(rh, rd):
        assert [a.df_min, a.df_max, a.azimuth, a.ext_phase, a.score] == \
            [b.df_min, b.df_max, b.azimuth, b.ext_phase, b.score]
        assert abs(a.df_min - 15000.0) < 600.0
