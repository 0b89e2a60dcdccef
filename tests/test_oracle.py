"""CPU checks of the FP64 oracle against closed-form known answers and
independent numpy restatements (these run without a GPU).

Reference behaviour cited per check (paths within the GCtfFind tree).
"""
import math

import numpy as np
import pytest

from gctffind_b200 import synth


def test_wavelength_and_amplitude_phase():
    # CCTFTheory::mCalcWavelength (FindCTF/CCTFTheory.cpp:283-287), 300 kV
    assert abs(synth.wavelength_angstrom(300.0) - 0.019687) < 1e-5
    assert abs(synth.wavelength_angstrom(200.0) - 0.025079) < 1e-5
    # amplitude-contrast phase atan(Ac / sqrt(1 - Ac^2)) (FindCTF/CCTFTheory.cpp:83-84)
    assert abs(math.atan(0.07 / math.sqrt(1 - 0.07 ** 2)) - 0.070057) < 1e-6


def _zero_freq(n, wl, cs, df, phi):
    """n-th zero of -sin(chi + phi) (CCTFTheory::CalcFrequency,
    FindCTF/CCTFTheory.cpp:201-228): pi wl s^2 df - pi/2 wl^3 s^4 cs + phi = n pi."""
    a = -0.5 * math.pi * wl ** 3 * cs
    b = math.pi * wl * df
    c = phi - n * math.pi
    det = b * b - 4 * a * c
    s1 = (-b + math.sqrt(det)) / (2 * a)
    s2 = (-b - math.sqrt(det)) / (2 * a)
    s2v = s1 if s1 > 0 else s2
    return math.sqrt(s2v)


def test_ctf1d_zeros_match_closed_form(oracle):
    n = 257
    px = 1.35
    wl = np.float32(synth.wavelength_angstrom(300.0) / px)
    cs = np.float32(2.7e7 / px)
    phi = np.float32(math.atan(0.07 / math.sqrt(1 - 0.0049)))
    df = np.float32(20000.0 / px)
    ctf = np.zeros(n)
    oracle.lib().orc_ctf1d(n, wl, cs, phi, df, ctf)
    s = np.arange(n) * 0.5 / (n - 1)
    for k in range(1, 6):
        f = _zero_freq(k, float(wl), float(cs), float(df), float(phi))
        i = int(f / (0.5 / (n - 1)))
        assert np.sign(ctf[i]) != np.sign(ctf[i + 1]), (k, f, i)
        # linear interpolation of the crossing within 1% of a bin
        x0 = s[i] + (s[i + 1] - s[i]) * ctf[i] / (ctf[i] - ctf[i + 1])
        assert abs(x0 - f) < 0.01 * (s[1] - s[0]) * 50


def _numpy_avg_spectrum(img, tile):
    h, w = img.shape
    ov = int(tile * 0.5) // 2 * 2
    size = tile - ov
    ntx, nty = (w - ov) // size, (h - ov) // size
    offx = (w - ntx * tile + (ntx - 1) * ov) // 2
    offy = (h - nty * tile + (nty - 1) * ov) // 2
    c = tile * 0.5
    y, x = np.mgrid[0:tile, 0:tile]
    r = np.sqrt((2 * np.abs(x - c) / tile) ** 2 + (2 * np.abs(y - c) / tile) ** 2)
    wgt = np.where(r < 1, 1 - (0.5 * (1 - np.cos(np.pi * r))) ** 3, 0.0)
    acc = np.zeros((tile, tile // 2 + 1))
    for ty in range(nty):
        for tx in range(ntx):
            t = img[offy + ty * size: offy + ty * size + tile,
                    offx + tx * size: offx + tx * size + tile].astype(np.float64)
            t = (t - t.mean()) * wgt
            a = np.abs(np.fft.rfft2(t))
            acc += np.roll(a, tile // 2, axis=0)
    return acc / (ntx * nty)


def test_avg_spectrum_matches_numpy(oracle):
    rng = np.random.default_rng(0)
    img = rng.poisson(5.0, size=(200, 230)).astype(np.float32)
    got = oracle.avg_spectrum(img, 64)
    ref = _numpy_avg_spectrum(img, 64)
    assert np.allclose(got, ref, rtol=1e-10, atol=1e-9)


def test_rescale_matches_numpy_fourier_crop(oracle):
    # CRescaleImage (FindCTF/CRescaleImage.cpp:47-99) with an odd-factor size (Bluestein)
    rng = np.random.default_rng(1)
    img = rng.standard_normal((150, 170)).astype(np.float32)
    px = 0.7
    nw, nh, npx, b = oracle.rescale_dims(170, 150, px)
    assert (nw, nh) == (98, 86) and abs(npx - 1.2) < 1e-6   # float32 arithmetic: 87.99999 -> 86
    X = np.fft.rfft2(img.astype(np.float64))
    rows = [y if y <= nh // 2 else y - nh + 150 for y in range(nh)]
    crop = X[rows, : nw // 2 + 1]
    ref = np.fft.irfft(np.fft.ifft(crop, axis=0), n=nw, axis=1) * (nh * nw)
    got = oracle.rescale(img, px)
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-3 * np.abs(ref).max())


def test_background_matches_numpy(oracle):
    # GRmBackground2D (FindCTF/GRmBackground2D.cu:11-70) for tile 64 (box 7)
    rng = np.random.default_rng(2)
    tile, cx = 64, 33
    raw = rng.uniform(1.0, 5.0, size=(tile, cx))
    got = oracle.remove_background(raw, 0)
    ref = np.zeros_like(raw)
    hb, hx, hy = 3, cx - 1, tile // 2
    for y in range(tile):
        yr = y - hy
        for x in range(cx):
            fr = np.float32(np.float32(x * 0.5) / (cx - 1))
            fr = np.sqrt(np.float32(fr * fr + np.float32(yr * yr / np.float32(tile * tile))))
            if fr < 0.04:
                continue
            s = 0.0
            for k in range(-hb, hb + 1):
                for j in range(-hb, hb + 1):
                    xx, yy = x + j, yr + k
                    if xx >= hx:
                        xx -= 2 * hx
                    ix, iy = (xx, hy + yy) if xx >= 0 else (-xx, hy - yy)
                    iy %= tile
                    s += math.sqrt(raw[iy, ix])
            s /= 49.0
            ref[y, x] = raw[y, x] - s * s
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_lowpass_is_circular_gaussian_blur(oracle):
    # CFindCtfBase::mLowpass with B = 10 (FindCTF/CFindCtfBase.cpp:191-219)
    rng = np.random.default_rng(3)
    tile, cx = 64, 33
    half = rng.standard_normal((tile, cx))
    got = oracle.lowpass(half, 10.0)
    full = np.zeros((tile, tile))
    for y in range(tile):
        for X in range(tile):
            xd = X - (cx - 1)
            full[y, X] = half[y, xd] if xd >= 0 else half[(tile - y) % tile, -xd]
    ky = np.fft.fftfreq(tile) * tile
    kx = np.fft.rfftfreq(tile) * tile
    ky[tile // 2] = tile / 2
    g = np.exp(-10.0 * (kx[None, :] ** 2 + ky[:, None] ** 2) / (2.0 * tile * tile))
    lp = np.fft.irfft2(np.fft.rfft2(full) * g, s=(tile, tile))
    ref = np.array([[lp[y, (x + cx - 1) % tile] for x in range(cx)] for y in range(tile)])
    assert np.allclose(got, ref, rtol=1e-10, atol=1e-10)


def test_radial_average_matches_numpy(oracle):
    # GRadialAvg (FindCTF/GRadialAvg.cu:11-33)
    rng = np.random.default_rng(4)
    tile, cx = 64, 33
    sp = rng.uniform(size=(tile, cx))
    got = oracle.radial_average(sp)
    for r in range(cx):
        npnt = min(max(int(np.float32(3.1415926) * r + np.float32(0.5)), 1), 180)
        step = np.float32(180.0) / npnt
        s = 0.0
        for i in range(npnt):
            rad = np.float32((np.float32(-90.0) + i * step) * np.float32(0.017453))
            x = int(np.float32(r * np.cos(rad, dtype=np.float32)) + np.float32(0.5))
            y = int(np.float32(r * np.sin(rad, dtype=np.float32)) + tile // 2 + np.float32(0.5))
            s += sp[min(y, tile - 1), min(x, cx - 1)]
        assert abs(got[r] - s / npnt) < 1e-6 * max(1.0, abs(s / npnt)), r


def test_cc2d_matches_numpy(oracle):
    # GCalcCTF2D + GCC2D (FindCTF/GCalcCTF2D.cu:15-38, FindCTF/GCC2D.cu:13-170)
    rng = np.random.default_rng(5)
    tile, cx = 128, 65
    px = 1.5
    wl = np.float32(synth.wavelength_angstrom(300.0) / px)
    cs = np.float32(2.7e7 / px)
    add = np.float32(0.07)
    ctf = oracle.ctf2d(tile, wl, cs, add, np.float32(9000.0), np.float32(9600.0), np.float32(0.4))
    y, x = np.mgrid[0:tile, 0:cx]
    fx = x * 0.5 / (cx - 1)
    fy = (y - tile // 2) / tile
    s2 = fx ** 2 + fy ** 2
    th = np.arctan(fy / (fx + 1e-30))
    df = 9300.0 + 300.0 * np.cos(2 * (th - np.float64(np.float32(0.4))))
    ref = -np.sin(float(add) + np.pi * float(wl) * s2 * (df - 0.5 * s2 * float(wl) ** 2 * float(cs)))
    assert np.allclose(ctf, ref, atol=1e-9)
    sp = rng.standard_normal((tile, cx))
    lo, hi = np.float32(0.04 * tile), np.float32(0.3 * tile)
    cc = oracle.cc2d(ctf, sp, lo, hi, 16.0)
    l2, h2 = np.float32(lo / tile) ** 2, np.float32(hi / tile) ** 2
    s2f = (np.float32(0.5) * x.astype(np.float32) / np.float32(cx - 1)) ** 2 + \
        ((y.astype(np.float32) - np.float32(tile * 0.5)) / np.float32(tile)) ** 2
    band = ~((s2f < l2) | (s2f > h2))
    c = (np.abs(ctf) - 0.5) * np.exp(-16 * s2)
    ref_cc = (c * sp)[band].sum() / math.sqrt((c * c)[band].sum() * (sp * sp)[band].sum())
    assert abs(cc - ref_cc) < 1e-10


def test_search_recovers_synthetic_ctf(oracle):
    spec = synth.MicrographSpec(width=768, height=768, pixel_size=1.5, df_min=11850, df_max=12150,
                                azimuth_deg=-25.0, dose=4.0, seed=11)
    img = synth.make_micrograph(spec).numpy()
    p = oracle.params(pixel_size=1.5, tile_size=256)
    r = oracle.find_ctf_image(img, 1.5, p)
    assert abs(r.df_min - 11850) < 150 and abs(r.df_max - 12150) < 150
    d = (r.azimuth + 25.0) % 180.0
    assert min(d, 180 - d) < 4.0
    assert r.score > 0.3 and r.lowpassed == 1


def test_series_policy_refines_around_best(oracle):
    # CFindSeriesCtfs: package order[0] full, others refined; results by index
    imgs, tilts = [], [-3.0, 0.0, 3.0]
    for i, t in enumerate(tilts):
        spec = synth.MicrographSpec(width=512, height=512, pixel_size=1.5, df_min=19900,
                                    df_max=20100, azimuth_deg=10.0, dose=4.0, seed=20 + i, tilt_deg=t)
        imgs.append(synth.make_micrograph(spec).numpy())
    p = oracle.params(pixel_size=1.5, tile_size=128)
    res = oracle.series(imgs, p, [1, 0, 2], True)
    assert res[1].df_1d > 0            # full search ran on the zero tilt
    assert res[0].df_1d == 0 and res[2].df_1d == 0   # refined
    for r in res:
        assert abs(0.5 * (r.df_min + r.df_max) - 20000) < 400


def test_background1d_known_answers(oracle):
    # GBackground1D::mFindStart / DoIt (FindCTF/GBackground1D.cu:95-169):
    # a spectrum above its fitted line until bin 30 starts there; the
    # background is the centred moving average of width start/2*2-1.
    n = 257
    x = np.arange(n, dtype=np.float64)
    sp = np.where(x < 30, 1000.0 - x, 100.0 - 0.1 * x).astype(np.float32)
    bg, st = oracle.background1d(sp)
    i0, i1 = n // 5, n - n // 5
    xs = x[i0:i1]
    a, b = np.polyfit(xs, sp[i0:i1].astype(np.float64), 1)
    exp_start = next(i for i in range(2, n) if a * i + b >= sp[i])
    assert st == exp_start
    w = st // 2 * 2 - 1
    for i in (st, st + 7, n - 3):
        ks = [k if k < n else 2 * n - 1 - k for k in range(i - w // 2, i - w // 2 + w)]
        assert abs(bg[i] - sp[ks].astype(np.float64).mean()) < 1e-3
    assert np.all(bg[:st] == 0)
    r = oracle.remove_bg1d(sp, bg, st)
    assert np.all(r[:st] == 0) and np.allclose(r[st:], sp[st:] - bg[st:])


def test_work_counters():
    """orc_counts: the 1D grid points of Do1D (coarse and refine passes) are
    counted, and a reset zeroes the counters."""
    import numpy as np
    from oracle import oracle as O
    rng = np.random.default_rng(5)
    ctf = rng.random((256, 129)) - 0.5
    p = O.params(pixel_size=1.35, tile_size=256)
    O.counts(reset=True)
    O.search1d(ctf, 1.35, p)
    c2, c1 = O.counts(reset=True)
    assert c2 == 0 and c1 > 501           # two brute-force passes of up to 501 points
    assert O.counts(reset=False) == (0, 0)
