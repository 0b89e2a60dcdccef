"""The closed forms behind the tensor-core rescale (gcf_rsgemm.cu), in FP64
against the oracle's Fourier-crop rescale (oracle/oracle.py rescale,
CRescaleImage::DoIt, FindCTF/CRescaleImage.cpp:68-99):

    out = Rh img Rw^T - a v^T + c w h,   v = Iw (b^T (img - c)),
    M[r][c] = -(-1)^r sin(pi c n_out / n_in) cot(pi (r/n_out - c/n_in))
              (n_out where r/n_out = c/n_in),
    Rw = M(nw, w), Rh = M(nh, h), a[y] = (-1)^y, b[i] = -sin(pi i nh / h),
    Iw[x][j] = (1 - (-1)^x cos(pi j nw / w)) cot(pi (x/nw - j/w))  (0 at t = 0).

The identity is exact, so the bar is float32 input rounding: max |d| <=
1e-6 x rms.  Without the rank-one term the error is several per cent, which
the second check shows (the term is needed)."""
import numpy as np
import pytest

from oracle import oracle as O


def _cot_pi(num, den):
    t = num / den
    with np.errstate(all="ignore"):
        return np.cos(np.pi * t) / np.sin(np.pi * t)


def _crop_map(n_out, n_in):
    r = np.arange(n_out)[:, None]
    c = np.arange(n_in)[None, :]
    num = r * n_in - c * n_out
    s = np.sin(np.pi * np.mod(c * n_out, 2 * n_in) / n_in)
    with np.errstate(all="ignore"):
        m = np.where(r % 2 == 1, 1.0, -1.0) * s * _cot_pi(num, n_out * n_in)
    return np.where(num == 0, float(n_out), m)


def _iw(nw, w):
    x = np.arange(nw)[:, None]
    j = np.arange(w)[None, :]
    num = x * w - j * nw
    cj = np.cos(np.pi * np.mod(j * nw, 2 * w) / w)
    with np.errstate(all="ignore"):
        m = (1.0 - np.where(x % 2 == 1, -1.0, 1.0) * cj) * _cot_pi(num, nw * w)
    return np.where(num == 0, 0.0, m)


def _maps_rescale(img, px, nyquist=True):
    h, w = img.shape
    nw, nh, _, _ = O.rescale_dims(w, h, px)
    im = img.astype(np.float64)
    c = float(im[h // 2, :256].mean())
    im = im - c
    out = _crop_map(nh, h) @ im @ _crop_map(nw, w).T + c * w * h
    if nyquist:
        b = -np.sin(np.pi * np.mod(np.arange(h) * nh, 2 * h) / h)
        v = _iw(nw, w) @ (b @ im)
        out -= np.outer((-1.0) ** np.arange(nh), v)
    return out


@pytest.mark.parametrize("w,h,px", [(46, 38, 0.9), (64, 50, 0.8), (40, 40, 1.0), (58, 62, 1.1),
                                    (301, 250, 0.85), (100, 100, 1.197)])
def test_closed_form_maps_equal_the_fourier_crop(w, h, px):
    rng = np.random.default_rng(w + 3 * h)
    img = (rng.poisson(2.0, size=(h, w)) + 50).astype(np.float32)
    ref = O.rescale(img, px).astype(np.float64)
    got = _maps_rescale(img, px)
    rms = float(np.sqrt((ref * ref).mean()))
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= 1e-6 * rms


def test_the_rank_one_nyquist_term_is_needed():
    rng = np.random.default_rng(2)
    img = rng.standard_normal((50, 64)).astype(np.float32)
    ref = O.rescale(img, 0.8).astype(np.float64)
    got = _maps_rescale(img, 0.8, nyquist=False)
    assert np.abs(got - ref).max() > 1e-2 * float(np.sqrt((ref * ref).mean()))
