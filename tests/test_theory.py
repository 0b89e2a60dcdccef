"""CPU: CCTFTheory host math of the library against the reference's own
CCTFTheory (compiled from its sources into oracle/_ref/libgcfref.so; host
code, so no GPU) -- bit for bit -- and against closed forms."""
import math

import numpy as np
import pytest

import gctffind_b200 as G


def _ref():
    from oracle import refimpl
    if not refimpl.available():
        pytest.skip("reference build oracle/_ref/libgcfref.so not present")
    return refimpl


OPTICS = [
    # kv, cs_mm, Ac, px, ast_tol, ext_phase_rad, df_min, df_max, azimuth_rad
    (300.0, 2.7, 0.07, 1.35, 100.0, 0.0, 14000.0, 14800.0, 0.7),
    (200.0, 2.0, 0.1, 0.8, -1.0, 1.2, 5000.0, 5000.0, -1.3),
    (300.0, 0.0, 0.07, 1.0, 100.0, 4.0, 22000.0, 23000.0, 3.0),     # Cs 0, phase > pi
    (120.0, 1.4, 0.15, 2.1, 50.0, 0.5, 40000.0, 41500.0, 0.0),
]


@pytest.mark.parametrize("o", OPTICS)
def test_ctf_theory_bit_identical_to_reference(o):
    R = _ref()
    rng = np.random.default_rng(int(o[0] + o[3] * 100))
    n = 64
    freq = rng.uniform(-0.5, 0.5, n).astype(np.float32)
    az = rng.uniform(-3.2, 3.2, n).astype(np.float32)
    ph = rng.uniform(-2.0, 40.0, n).astype(np.float32)
    ref = R.ctf_theory(*o, freq, az, ph)
    t = G.CCTFTheory()
    t.Setup(*o[:6])
    t.SetDefocus(*o[6:])
    mine = np.array([getattr(t.param, k) for k, _ in G.CtfParam._fields_], np.float32)
    assert np.array_equal(mine, ref["param"])
    got = {
        "evaluate": [t.Evaluate(float(f), float(a)) for f, a in zip(freq, az)],
        "phase_shift": [t.CalcPhaseShift(float(f), float(a)) for f, a in zip(freq, az)],
        "defocus": [t.CalcDefocus(float(a)) for a in az],
        "frequency": [t.CalcFrequency(float(p), float(a)) for p, a in zip(ph, az)],
        "zeros": [t.CalcNthZero(k + 1, float(a)) for k, a in enumerate(az)],
    }
    for k, v in got.items():
        assert np.array_equal(np.asarray(v, np.float32), ref[k]), k


def test_ctf_theory_closed_forms():
    t = G.CCTFTheory()
    t.Setup(300.0, 2.7, 0.07, 1.0, 100.0, 0.0)
    # lambda(300 kV) = 12.26 / sqrt(V + 0.9784e-6 V^2) A (FindCTF/CCTFTheory.cpp:283-287)
    assert t.param.wavelength == pytest.approx(12.26 / math.sqrt(300e3 + 0.9784e-6 * 300e3 ** 2), rel=1e-6)
    assert t.param.amp_phase == pytest.approx(math.atan(0.07 / math.sqrt(1 - 0.0049)), rel=1e-6)
    assert t.param.cs == pytest.approx(2.7e7)
    t.SetDefocus(15000.0, 15600.0, 0.0)
    assert t.CalcDefocus(0.0) == pytest.approx(15600.0)
    assert t.CalcDefocus(math.pi / 2) == pytest.approx(15000.0, abs=0.01)
    # the n-th zero solves phase(s) = n pi
    for n in (1, 2, 5):
        s = t.CalcNthZero(n, 0.3)
        assert t.CalcPhaseShift(s, 0.3) == pytest.approx(n * math.pi, rel=1e-4)
        assert abs(t.Evaluate(s, 0.3)) < 1e-3
    t.SetExtPhase(200.0, True)              # kept mod pi
    assert t.GetExtPhase(True) == pytest.approx(20.0, abs=1e-3)


def test_change_pixel_size_and_equal_to():
    a = G.CCTFTheory()
    a.Setup(300.0, 2.7, 0.07, 1.0, 100.0, 0.0)
    a.SetDefocus(15000.0, 15600.0, 0.2)
    b = a.GetCopy()
    assert a.EqualTo(b, 1.0)
    b.ChangePixelSize(2.0)
    assert b.param.df_max == pytest.approx(7800.0) and b.param.pixel_size == 2.0
    assert not a.EqualTo(b, 1.0)
    c = a.GetCopy()
    c.SetDefocusInPixel(15000.0, 15600.5, 0.2)
    assert c.EqualTo(a, 1.0) and not c.EqualTo(a, 0.1)
    # the extra-phase test of CCTFTheory::EqualTo looks at the remainder of
    # the amplitude-contrast difference, so a different extra phase alone
    # still compares equal
    d = a.GetCopy()
    d.SetExtPhase(1.0, False)
    assert d.EqualTo(a, 1.0)
