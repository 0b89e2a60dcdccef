"""GPU parity against the reference itself: the reference's own CTF path,
compiled from the GCtfFind sources into oracle/_ref/libgcfref.so (recipe
oracle/ref/Makefile), run on the same inputs as the B200 library (through
its C ABI) and the FP64 oracle.

The reference computes in float32 with float tree reductions, the B200
library with float32 spectra and FP64 sums, so the two agree to rounding:
  rescaled image       : max |d| <= 1e-5 x rms
  averaged spectrum    : |d| <= 1e-4 x |ref| + 1e-5 x rms per pixel
  ctf spectrum         : max |d| <= 5e-4 x rms at least 9 pixels away from
                         the y = 0 row and the x = tile/2 column, where the
                         reference's lowpass reads undefined values (one row
                         past its buffer, FindCTF/GCalcSpectrum.cu:53; the
                         padding of an in-place C2R, FindCTF/CFindCtfBase.cpp:
                         212-218) that its blur spreads a few pixels inward
  full spectrum        : max |d| <= 5e-3 x rms away from the same border
  search results       : the path's accuracy bar -- defocus within one search
                         step of the final iteration (max(20 A, range / 31))
                         -> 60 A here, azimuth 1 degree (mod 180) when the
                         astigmatism exceeds 50 A, extra phase 2 degrees,
                         CC 1e-3; observed: equal to float rounding
"""
import os

import numpy as np
import pytest

from gctffind_b200 import synth

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def ref():
    from oracle import refimpl
    if not refimpl.available():
        pytest.skip("reference build oracle/_ref/libgcfref.so not present")
    return refimpl


def _img(w, h, px, df, az, seed, tilt=0.0, phase=0.0):
    spec = synth.MicrographSpec(width=w, height=h, pixel_size=px, df_min=df[0], df_max=df[1],
                                azimuth_deg=az, dose=3.0, seed=seed, tilt_deg=tilt,
                                ext_phase_deg=phase)
    return synth.make_micrograph(spec, device="cpu").numpy().astype(np.float32)


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / np.sqrt((b * b).mean()))


def _ang(a, b):
    d = (a - b) % 180.0
    return min(d, 180.0 - d)


def _close(g, r, df_tol=60.0, ang_tol=1.0, cc_tol=1e-3, ph_tol=2.0):
    """g, r: (df_min, df_max, azimuth, ext_phase, score)."""
    assert abs(g[0] - r[0]) <= df_tol and abs(g[1] - r[1]) <= df_tol, (g, r)
    if abs(r[1] - r[0]) > 50.0:
        assert _ang(g[2], r[2]) <= ang_tol, (g, r)
    assert abs(g[3] - r[3]) <= ph_tol, (g, r)
    assert abs(g[4] - r[4]) <= cc_tol, (g, r)


def _mine_single(G, img, px, tile, log_spect=0, phase=0.0, phase_range=0.0, refine=None):
    ctx = G.Context(0, tile, log_spect)
    resc = ctx.rescale(img, px)
    nw, nh, npx = G.rescale_dims(img.shape[1], img.shape[0], px)
    ctx.setup(G.make_optics(pixel_size=npx, ext_phase_deg=phase, ext_phase_range=phase_range), nw, nh)
    ctx.gen_half_spectrum(resc)
    raw, ctf = ctx.half_spectrum(True), ctx.half_spectrum(False)
    if refine is None:
        ctx.set_phase(phase, max(phase_range, 0.0))
        r = ctx.do2d()
    else:
        r = ctx.refine(refine[0:2], refine[2:4], refine[4:6], refine[6:8])
    full = ctx.full_spectrum(r)
    ctx.close()
    return resc, raw, ctf, full, [r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score]


CASES = [
    # w, h, px, df, az, seed, phase (truth), tile, log, phase0, range, refine
    (2048, 2048, 1.0, (21000.0, 21700.0), 50.0, 106, 0.0, 512, 0, 0.0, 0.0, None),
    (1024, 1024, 1.35, (25000.0, 25800.0), -15.0, 105, 0.0, 512, 0, 0.0, 0.0, None),
    (2048, 2048, 1.35, (9000.0, 9400.0), -70.0, 107, 60.0, 512, 0, 45.0, 90.0, None),
    (1024, 896, 1.5, (20000.0, 20500.0), 75.0, 103, 0.0, 256, 1, 0.0, 0.0, None),
    (1024, 1024, 1.35, (18000.0, 18400.0), 10.0, 104, 0.0, 512, 0, 0.0, 0.0,
     [18300.0, 9000.0, 0.011, 0.04, 12.0, 30.0, 0.0, 0.0]),
    # tile 1024 (batched-cuFFT spectrum), rescaled from 1.0 A/px
    (3072, 3072, 1.0, (30000.0, 30600.0), -35.0, 108, 0.0, 1024, 0, 0.0, 0.0, None),
    # odd raw sizes, rescale by 1.5 (0.8 A/px), tile 256, log spectrum
    (1501, 1101, 0.8, (12000.0, 12300.0), 5.0, 109, 0.0, 256, 1, 0.0, 0.0, None),
    # odd raw width without rescale: the last column is dropped (new size even)
    (1023, 777, 1.5, (26000.0, 26600.0), 60.0, 110, 0.0, 256, 0, 0.0, 0.0, None),
    # a tile size that is not a power of two (batched cuFFT with mixed radices)
    (1536, 1536, 1.35, (19000.0, 19500.0), -50.0, 112, 0.0, 384, 0, 0.0, 0.0, None),
]


@pytest.mark.parametrize("case", CASES, ids=["px1.0_t512", "px1.35_t512", "phase_t512", "log_t256",
                                             "refine_t512", "px1.0_t1024", "odd_rescale_log_t256",
                                             "odd_width_t256", "px1.35_t384"])
def test_single_micrograph_matches_reference(gpu_lib, ref, case):
    w, h, px, df, az, seed, phase_truth, tile, log, ph0, phr, refine = case
    img = _img(w, h, px, df, az, seed, phase=phase_truth)
    R = ref.single(img, px, tile=tile, log_spect=log, ext_phase_deg=ph0, ext_phase_range=phr,
                   refine=refine)
    resc, raw, ctf, full, res = _mine_single(gpu_lib, img, px, tile, log, ph0, phr, refine)
    assert resc.shape == R["rescaled"].shape
    assert _rel(resc, R["rescaled"]) <= 1e-5
    Rr = R["raw_half"].astype(np.float64)
    rms = np.sqrt((Rr * Rr).mean())
    assert np.all(np.abs(raw - Rr) <= 1e-4 * np.abs(Rr) + 1e-5 * rms)
    m = np.ones(ctf.shape, bool)
    m[:9, :] = m[tile - 8:, :] = False
    m[:, tile // 2 - 8:] = False
    C = R["ctf_half"].astype(np.float64)
    assert np.abs(ctf - C)[m].max() <= 5e-4 * np.sqrt((C * C).mean())
    fm = np.ones(full.shape, bool)
    fm[:9, :] = fm[-8:, :] = False
    fm[:, :9] = fm[:, -8:] = False
    fm[:, tile // 2 - 8: tile // 2 + 9] = False
    ref_res = [float(x) for x in R["result"]]
    if max(abs(a - b) for a, b in zip(res, ref_res)) > 0.01:
        # a neighbouring candidate won a CC tie (float vs FP64 sums): the
        # fitted CTF drawn into the left half differs, so compare the
        # spectrum half only
        fm[:, : tile // 2 + 9] = False
    F = R["full"].astype(np.float64)
    assert np.abs(full - F)[fm].max() <= 5e-3 * np.sqrt((F * F).mean())
    _close(res, ref_res)


@pytest.mark.parametrize("phase", [(0.0, 0.0), (30.0, 60.0)], ids=["no_phase", "phase_search"])
def test_do1d_and_refine1d_match_reference(gpu_lib, ref, phase):
    """CFindCtf1D::Do1D and Refine1D: same grid point as the reference (the
    1D grids are float expressions evaluated identically), CC to 1e-4."""
    G = gpu_lib
    img = _img(2048, 2048, 1.35, (17000.0, 17400.0), 30.0, 701, phase=phase[0] + 5.0)
    ctx = G.Context(0, 512, 0)
    ctx.setup(G.make_optics(pixel_size=1.35, ext_phase_deg=phase[0], ext_phase_range=phase[1]),
              2048, 2048)
    ctx.gen_half_spectrum(img)
    ctx.set_phase(*phase)
    r1 = ctx.do1d()
    ctx.set_phase(*phase)
    r2 = ctx.refine1d(16000.0, 5000.0)
    ctx.close()
    d1, p1, c1 = ref.single1d(img, 1.35, ext_phase_deg=phase[0], ext_phase_range=phase[1])
    d2, p2, c2 = ref.single1d(img, 1.35, ext_phase_deg=phase[0], ext_phase_range=phase[1],
                              refine=(16000.0, 5000.0))
    for r, (d, p, c) in ((r1, (d1, p1, c1)), (r2, (d2, p2, c2))):
        assert r.df_min == r.df_max
        assert abs(r.df_min - d) <= 10.0, (r, d, p, c)      # 10 A: the finest 1D step
        assert abs(r.ext_phase - p) <= 1e-3 + (phase[1] / 36.0), (r, d, p, c)
        assert abs(r.score - c) <= 1e-4, (r, d, p, c)


def test_phase_plate_set_matches_reference(gpu_lib, ref):
    """Micrographs (not a tilt series) with extra-phase search: Do2D, then
    refines whose windows include the phase, each starting from a newly set
    up search object."""
    G = gpu_lib
    imgs = [_img(1024, 1024, 1.35, (12000.0 + 300 * k, 12500.0 + 300 * k), -20.0 + 15 * k, 600 + k,
                 phase=35.0 + 5 * k) for k in range(4)]
    R, _, _ = ref.run_series(imgs, 1.35, list(range(4)), is_tomo=False, ext_phase_deg=30.0,
                             ext_phase_range=60.0, tile=512)
    ctx = G.Context(0, 512, 0)
    op = G.make_optics(pixel_size=1.35, ext_phase_deg=30.0, ext_phase_range=60.0)
    mine = ctx.run_series(imgs, op, list(range(4)), is_tomo=False)
    ctx.close()
    for k in range(4):
        r = mine[k]
        _close([r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score], [float(x) for x in R[k]])


def test_series_matches_reference(gpu_lib, ref):
    G = gpu_lib
    tilts = [3.0 * (k - 3) for k in range(7)]
    imgs = [_img(1024, 1024, 1.35, (15800.0 + 40 * k, 16200.0 + 40 * k), 25.0, 300 + k, tilt=t)
            for k, t in enumerate(tilts)]
    order = G.series_order(tilts).order
    R, _, _ = ref.run_series(imgs, 1.35, order, tilts=tilts, tile=512)
    ctx = G.Context(0, 512, 0)
    mine = ctx.run_series(imgs, G.make_optics(pixel_size=1.35), order, is_tomo=True)
    ctx.close()
    for k in range(len(imgs)):
        r = mine[k]
        _close([r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score], [float(x) for x in R[k]])


def test_ctf_file_matches_reference_writer(gpu_lib, ref, tmp_path):
    """The reference's CSaveCtfResults output and gcf_write_ctf_file agree
    byte for byte on the same numbers."""
    G = gpu_lib
    tilts = [-3.0, 0.0, 3.0]
    imgs = [_img(512, 512, 1.35, (16000.0, 16300.0), 25.0, 400 + k, tilt=t)
            for k, t in enumerate(tilts)]
    order = G.series_order(tilts).order
    ref_txt = str(tmp_path / "ref.txt")
    R, _, _ = ref.run_series(imgs, 1.35, order, tilts=tilts, tile=128, names=["ts.mrc"] * 3,
                             out_ctf=ref_txt)
    results = []
    for k in range(3):
        r = G.Result()
        r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score = [float(x) for x in R[k]]
        results.append(r)
    mine_txt = str(tmp_path / "mine.txt")
    G.write_ctf_file(mine_txt, results, tilts=tilts, names=["ts.mrc"] * 3, is_tomo=True)
    assert open(mine_txt).read() == open(ref_txt).read()
    assert open(str(tmp_path / "mine_Imod.txt")).read() == open(str(tmp_path / "ref_Imod.txt")).read()


def test_background1d_matches_reference(gpu_lib, ref):
    """GBackground1D DoIt / Remove1D / Remove2D: start and background
    bit-identical to the reference; the removals to one float rounding."""
    G = gpu_lib
    img = _img(1024, 1024, 1.35, (15000.0, 15400.0), 30.0, 801)
    ctx = G.Context(0, 512, 0)
    ctx.setup(G.make_optics(pixel_size=1.35), 1024, 1024)
    ctx.gen_half_spectrum(img)
    radial = ctx.radial_average().astype(np.float32)
    half = ctx.half_spectrum(raw=True)
    x = np.arange(513, dtype=np.float64)
    curves = [radial, (1000 * np.exp(-x / 60) + 40 * np.cos(x / 4) ** 2 + 10).astype(np.float32)]
    for sp in curves:
        bg, st = ctx.background1d(sp)
        rbg, rst, rhalf, r1 = ref.background1d(sp, half=half if len(sp) == 257 else None,
                                               spec1d=sp)
        assert st == rst
        assert np.array_equal(bg, rbg)
        m1 = ctx.remove_background1d(sp, bg, st)
        assert np.allclose(m1, r1, rtol=1e-6, atol=1e-6 * np.abs(sp).max())
        if rhalf is not None:
            m2 = ctx.remove_background2d(half, bg, st)
            assert np.allclose(m2, rhalf, rtol=1e-6, atol=1e-6 * np.abs(half).max())
    ctx.close()


def test_flat_spectrum_skips_lowpass_like_reference(gpu_lib, ref):
    """CFindCtfBase::mRemoveBackground skips the lowpass when the background-
    removed spectrum's variance is below 1 (FindCTF/CFindCtfBase.cpp:170-175):
    a faint image (x 1e-4) goes down that branch in both implementations."""
    G = gpu_lib
    img = _img(1024, 1024, 1.35, (16000.0, 16500.0), 20.0, 111) * np.float32(1e-4)
    R = ref.single(img, 1.35, tile=512)
    resc, raw, ctf, full, res = _mine_single(G, img, 1.35, 512)
    C = R["ctf_half"].astype(np.float64)
    assert np.abs(ctf - C).max() <= 1e-4 * np.sqrt((C * C).mean())
    ctx = G.Context(0, 512, 0)
    r = ctx.run_series([img], G.make_optics(pixel_size=1.35), [0], is_tomo=False)[0]
    ctx.close()
    assert r.lowpassed == 0
    _close(res, [float(x) for x in R["result"]])


def test_uneven_batch_matches_reference_single_file_mode(gpu_lib, ref):
    """gcf_run_batch (independent full searches of micrographs of different
    sizes and pixel sizes in one call) against the reference run once per
    micrograph, as its single-file mode does (CInputFolder::mReadSingle)."""
    G = gpu_lib
    rng = np.random.default_rng(12)
    specs = [(2048, 2048, 0.8), (1536, 1152, 1.5), (2000, 1400, 1.0), (1024, 1024, 1.35),
             (1777, 1333, 1.2)]
    imgs, truth = [], []
    for k, (w, h, px) in enumerate(specs):
        df = float(rng.uniform(8000.0, 30000.0))
        ast = float(rng.uniform(0.0, 600.0))
        imgs.append(_img(w, h, px, (df - ast / 2, df + ast / 2), float(rng.uniform(-90, 90)), 900 + k))
    ctx = G.Context(0, 512, 0)
    mine = ctx.run_batch(imgs, [s[2] for s in specs], G.make_optics())
    ctx.close()
    for img, (w, h, px), r in zip(imgs, specs, mine):
        R, _, _ = ref.run_series([img], px, [0], is_tomo=False, tile=512)
        _close([r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score], [float(x) for x in R[0]])


def test_config0_single_micrograph_matches_reference(gpu_lib, ref):
    """The single-micrograph configuration: 4096 x 4096 at 1.0 A/px (rescaled
    to 3412 x 3412 at 1.2 A/px), 300 kV, Cs 2.7 mm, Ac 0.07, defocus
    15000 A with 300 A of astigmatism at 20 degrees, 1 e/A^2, tile 512,
    1D then 2D search."""
    G = gpu_lib
    spec = synth.MicrographSpec(width=4096, height=4096, pixel_size=1.0, df_min=14850.0,
                                df_max=15150.0, azimuth_deg=20.0, dose=1.0, seed=2024)
    img = synth.make_micrograph(spec, device="cpu").numpy().astype(np.float32)
    R, _, _ = ref.run_series([img], 1.0, [0], is_tomo=False, tile=512)
    ctx = G.Context(0, 512, 0)
    r = ctx.run_series([img], G.make_optics(pixel_size=1.0), [0], is_tomo=False)[0]
    ctx.close()
    _close([r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score], [float(x) for x in R[0]])
    assert abs(0.5 * (r.df_min + r.df_max) - 15000.0) < 150.0


def test_config2_uneven_sizes_match_reference(gpu_lib, ref):
    """The uneven batch's sizes (4096 x 4096, 5760 x 4092, 3838 x 3710) at
    pixel sizes from 0.8 to 1.5 A/px through one gcf_run_batch call, against
    the reference once per micrograph."""
    G = gpu_lib
    rng = np.random.default_rng(256)
    sizes = [(4096, 4096, 0.8), (5760, 4092, 1.5), (3838, 3710, 1.1), (5760, 4092, 0.9),
             (3838, 3710, 1.5), (4096, 4096, 1.3)]
    imgs = []
    for k, (w, h, px) in enumerate(sizes):
        df = float(rng.uniform(9000.0, 38000.0))
        ast = float(rng.uniform(0.0, 1000.0))
        spec = synth.MicrographSpec(width=w, height=h, pixel_size=px, df_min=df - ast / 2,
                                    df_max=df + ast / 2, azimuth_deg=float(rng.uniform(-90, 90)),
                                    dose=float(rng.uniform(0.5, 2.0)), seed=3000 + k)
        imgs.append(synth.make_micrograph(spec, device="cpu").numpy().astype(np.float32))
    ctx = G.Context(0, 512, 0)
    mine = ctx.run_batch(imgs, [s[2] for s in sizes], G.make_optics())
    ctx.close()
    for img, (w, h, px), r in zip(imgs, sizes, mine):
        R, _, _ = ref.run_series([img], px, [0], is_tomo=False, tile=512)
        _close([r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score], [float(x) for x in R[0]])
