"""Accuracy of the arithmetic behind k_eval2d's rotation path (CPU).

Evenly stepped line searches (mean defocus, astigmatism magnitude, phase) make
the CTF phase in turns an arithmetic sequence t0 + i * dt at every band pixel,
so the kernel forms sin(pi t_i) by rotation instead of one hardware sine per
(candidate, pixel) pair: sin and cos of pi r for |r| <= 1/2 come from their
Taylor series (coefficients (-1)^k pi^n / n!, truncated after r^13 and r^14),
and each further candidate costs one complex rotation by pi dt; two chains,
seeded at candidates 0 and 8 of a 16-candidate block, advance side by side.
This test restates that arithmetic in float32, each fused multiply-add as a
float64 product (exact for float32 operands) and sum rounded to float32 (a
true fused multiply-add but for rare double roundings), and checks it against
float64 sines: the seed within a few float32 ulps, and |sin| along a block
within 1.5e-6 beyond the rounding of t itself, the size of the error of the
fast hardware sine the other path uses.
"""
import math

import numpy as np

F = np.float32


def _fma(a, b, c):
    return F(np.float64(a) * np.float64(b) + np.float64(c))


_S = [(-1) ** k * math.pi ** (2 * k + 1) / math.factorial(2 * k + 1) for k in range(7)]
_C = [(-1) ** k * math.pi ** (2 * k) / math.factorial(2 * k) for k in range(8)]


def sincos_pi_half(r):
    """The kernel's Horner evaluation, operation by operation, in float32."""
    r = F(r)
    r2 = F(r * r)
    p = _fma(F(_S[6]), r2, F(_S[5]))
    for c in (_S[4], _S[3], _S[2], _S[1], _S[0]):
        p = _fma(p, r2, F(c))
    s = F(p * r)
    q = _fma(F(_C[7]), r2, F(_C[6]))
    for c in (_C[5], _C[4], _C[3], _C[2], _C[1]):
        q = _fma(q, r2, F(c))
    c = _fma(q, r2, F(1.0))
    return s, c


def _rint_small(t):
    m = F(12582912.0)   # 1.5 * 2^23
    return F(F(t + m) - m)


def test_seed_polynomial_accuracy():
    r = np.linspace(-0.5, 0.5, 4001)
    err_s = err_c = 0.0
    for x in r:
        s, c = sincos_pi_half(x)
        xr = float(F(x))
        err_s = max(err_s, abs(float(s) - math.sin(math.pi * xr)))
        err_c = max(err_c, abs(float(c) - math.cos(math.pi * xr)))
    assert err_s < 3e-7 and err_c < 3e-7, (err_s, err_c)


def test_rotation_chains_track_the_sine():
    rng = np.random.default_rng(7)
    worst = 0.0
    for _ in range(300):
        t0 = F(rng.uniform(-40.0, 40.0))    # CTF phase in turns at one band pixel
        dt = F(rng.uniform(-0.6, 0.6))      # its step between neighbouring candidates
        t8 = _fma(F(8.0), dt, t0)
        s = np.zeros(2, F)
        c = np.zeros(2, F)
        s[0], c[0] = sincos_pi_half(F(t0 - _rint_small(t0)))
        s[1], c[1] = sincos_pi_half(F(t8 - _rint_small(t8)))
        sd, cd = sincos_pi_half(F(dt - _rint_small(dt)))
        for i in range(8):
            for h in (0, 1):
                k = i + 8 * h
                exact = abs(math.sin(math.pi * (float(t0) + k * float(dt))))
                worst = max(worst, abs(abs(float(s[h])) - exact))
            for h in (0, 1):
                sn = _fma(s[h], cd, F(c[h] * sd))
                c[h] = _fma(c[h], cd, F(s[h] * F(-sd)))
                s[h] = sn
    # t0 + k dt itself carries float32 rounding of ~|t| * 2^-24 (the same in
    # the sine path: up to 6e-6 in sin at |t| = 40); beyond that the rotation
    # adds a few 1e-7
    assert worst < 1e-5, worst


def test_rotation_error_beyond_phase_rounding():
    """With t exactly representable steps, the rotation alone stays < 1.5e-6."""
    worst = 0.0
    for t0, dt in ((F(0.125), F(0.03125)), (F(-3.25), F(0.0625)), (F(17.5), F(-0.1875)), (F(0.0), F(0.5))):
        t8 = _fma(F(8.0), dt, t0)
        s = [None, None]
        c = [None, None]
        s[0], c[0] = sincos_pi_half(F(t0 - _rint_small(t0)))
        s[1], c[1] = sincos_pi_half(F(t8 - _rint_small(t8)))
        sd, cd = sincos_pi_half(F(dt - _rint_small(dt)))
        for i in range(8):
            for h in (0, 1):
                k = i + 8 * h
                exact = abs(math.sin(math.pi * (float(t0) + k * float(dt))))
                worst = max(worst, abs(abs(float(s[h])) - exact))
                sn = _fma(s[h], cd, F(c[h] * sd))
                c[h] = _fma(c[h], cd, F(s[h] * F(-sd)))
                s[h] = sn
    assert worst < 1.5e-6, worst
