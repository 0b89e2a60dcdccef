"""ctypes binding of the FP64 CPU oracle (oracle/libgcf_oracle.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg use this module as the checker.  The product package
(gctffind_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgcf_oracle.so")


class OrcResult(C.Structure):
    _fields_ = [("df_min", C.c_float), ("df_max", C.c_float), ("azimuth", C.c_float),
                ("ext_phase", C.c_float), ("score", C.c_float), ("ctf_res", C.c_float),
                ("df_1d", C.c_float), ("phase_1d", C.c_float), ("score_1d", C.c_float),
                ("lowpassed", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class OrcParams(C.Structure):
    _fields_ = [("kv", C.c_float), ("cs_mm", C.c_float), ("amp_contrast", C.c_float),
                ("pixel_size", C.c_float), ("ext_phase_deg", C.c_float),
                ("ext_phase_range", C.c_float), ("tile_size", C.c_int), ("log_spect", C.c_int),
                ("held_phase", C.c_float)]


def params(kv=300.0, cs_mm=2.7, amp_contrast=0.07, pixel_size=1.0, ext_phase_deg=0.0,
           ext_phase_range=0.0, tile_size=512, log_spect=0, held_phase=0.0) -> OrcParams:
    """held_phase: the extra phase (deg) the reference's search object holds
    when Do2D / Refine starts (0 for a freshly set-up object)."""
    return OrcParams(kv, cs_mm, amp_contrast, pixel_size, ext_phase_deg, ext_phase_range,
                     tile_size, log_spect, held_phase)


def build(force: bool = False) -> str:
    """Compile the oracle with the committed Makefile (gcc + OpenMP)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.check_call(["make", "-s", "-C", HERE, "lib"])
    return LIB_PATH


_lib = None

_F = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def lib():
    global _lib
    if _lib is not None:
        return _lib
    build()
    L = C.CDLL(LIB_PATH)
    L.orc_num_threads.argtypes = [C.c_int]
    L.orc_num_threads.restype = C.c_int
    L.orc_rescale_dims.argtypes = [C.c_int, C.c_int, C.c_float, C.POINTER(C.c_int),
                                   C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.orc_rescale.argtypes = [_F, C.c_int, C.c_int, C.c_float, _F, C.c_int]
    L.orc_tile_layout.argtypes = [C.c_int, C.c_int, C.c_int] + [C.POINTER(C.c_int)] * 5
    L.orc_avg_spectrum.argtypes = [_F, C.c_int, C.c_int, C.c_int, C.c_int, _D]
    L.orc_avg_spectrum.restype = C.c_int
    L.orc_taper.argtypes = [C.c_int, _D]
    L.orc_ctf_spectrum.argtypes = [_D, C.c_int, C.c_int, _D, C.c_void_p]
    L.orc_ctf_spectrum.restype = C.c_int
    L.orc_remove_background.argtypes = [_D, C.c_int, C.c_int, _D]
    L.orc_lowpass.argtypes = [_D, C.c_int, C.c_double, _D]
    L.orc_radial_average.argtypes = [_D, C.c_int, _D]
    L.orc_ctf1d.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, _D]
    L.orc_cc1d.argtypes = [_D, _D, C.c_int, C.c_float, C.c_float, C.c_float]
    L.orc_cc1d.restype = C.c_double
    L.orc_ctf2d.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                            C.c_float, _D]
    L.orc_cc2d.argtypes = [_D, _D, C.c_int, C.c_float, C.c_float, C.c_float]
    L.orc_cc2d.restype = C.c_double
    L.orc_find_ctf_image.argtypes = [_F, C.c_int, C.c_int, C.c_int, C.c_float,
                                     C.POINTER(OrcParams), C.c_int, C.c_void_p,
                                     C.POINTER(OrcResult), C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_find_ctf_image.restype = C.c_int
    L.orc_search.argtypes = [_D, C.c_int, C.c_float, C.POINTER(OrcParams), C.c_int, C.c_void_p,
                             C.POINTER(OrcResult)]
    L.orc_search1d.argtypes = [_D, C.c_int, C.c_float, C.POINTER(OrcParams),
                               C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.orc_refine1d.argtypes = [_D, C.c_int, C.c_float, C.POINTER(OrcParams), C.c_float, C.c_float,
                               C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.orc_background1d.argtypes = [_F, C.c_int, _F, C.POINTER(C.c_int)]
    L.orc_background1d.restype = C.c_int
    L.orc_remove_bg1d.argtypes = [_F, C.c_int, _F, C.c_int, C.c_int]
    L.orc_remove_bg1d.restype = None
    L.orc_remove_bg2d.argtypes = [_F, C.c_int, _F, C.c_int, C.c_int]
    L.orc_remove_bg2d.restype = None
    L.orc_full_spectrum.argtypes = [_D, C.c_int, C.c_float, C.POINTER(OrcParams),
                                    C.POINTER(OrcResult), _F]
    L.orc_series.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int,
                             C.POINTER(OrcParams), C.POINTER(C.c_int), C.c_int,
                             C.POINTER(OrcResult)]
    L.orc_series.restype = C.c_int
    L.orc_counts.argtypes = [C.POINTER(C.c_longlong), C.c_int]
    L.orc_counts.restype = None
    _lib = L
    return L


def num_threads(n: int = 0) -> int:
    return lib().orc_num_threads(n)


def rescale_dims(w, h, px):
    nw, nh, npx, b = C.c_int(), C.c_int(), C.c_float(), C.c_float()
    lib().orc_rescale_dims(w, h, px, C.byref(nw), C.byref(nh), C.byref(npx), C.byref(b))
    return nw.value, nh.value, npx.value, b.value


def rescale(img: np.ndarray, px: float) -> np.ndarray:
    h, w = img.shape
    nw, nh, _, _ = rescale_dims(w, h, px)
    out = np.zeros((nh, nw), np.float32)
    lib().orc_rescale(np.ascontiguousarray(img, np.float32), w, h, px, out, 0)
    return out


def tile_layout(w, h, tile):
    v = [C.c_int() for _ in range(5)]
    lib().orc_tile_layout(w, h, tile, *[C.byref(x) for x in v])
    return tuple(x.value for x in v)


def avg_spectrum(img: np.ndarray, tile: int) -> np.ndarray:
    h, w = img.shape
    out = np.zeros((tile, tile // 2 + 1), np.float64)
    n = lib().orc_avg_spectrum(np.ascontiguousarray(img, np.float32), w, h, w, tile, out)
    if n <= 0:
        raise ValueError("image smaller than one tile")
    return out


def taper(tile: int) -> np.ndarray:
    out = np.zeros((tile, tile), np.float64)
    lib().orc_taper(tile, out)
    return out


def ctf_spectrum(raw: np.ndarray, log_spect: int = 0):
    tile = raw.shape[0]
    out = np.zeros_like(raw, dtype=np.float64)
    lp = lib().orc_ctf_spectrum(np.ascontiguousarray(raw, np.float64), tile, log_spect, out, None)
    return out, lp


def remove_background(raw: np.ndarray, log_spect: int = 0) -> np.ndarray:
    out = np.zeros_like(raw, dtype=np.float64)
    lib().orc_remove_background(np.ascontiguousarray(raw, np.float64), raw.shape[0], log_spect, out)
    return out


def lowpass(spect: np.ndarray, bfactor: float = 10.0) -> np.ndarray:
    out = np.zeros_like(spect, dtype=np.float64)
    lib().orc_lowpass(np.ascontiguousarray(spect, np.float64), spect.shape[0], bfactor, out)
    return out


def radial_average(spect: np.ndarray) -> np.ndarray:
    tile = spect.shape[0]
    out = np.zeros(tile // 2 + 1, np.float64)
    lib().orc_radial_average(np.ascontiguousarray(spect, np.float64), tile, out)
    return out


def ctf2d(tile, wl_px, cs_px, add_phase, dfmin_px, dfmax_px, az_rad) -> np.ndarray:
    out = np.zeros((tile, tile // 2 + 1), np.float64)
    lib().orc_ctf2d(tile, wl_px, cs_px, add_phase, dfmin_px, dfmax_px, az_rad, out)
    return out


def cc2d(ctf, spect, lo, hi, bfac=16.0) -> float:
    return lib().orc_cc2d(np.ascontiguousarray(ctf, np.float64),
                          np.ascontiguousarray(spect, np.float64), spect.shape[0], lo, hi, bfac)


def search(ctf_spect: np.ndarray, px_n: float, p: OrcParams, mode: int = 0, refine_in=None):
    r = OrcResult()
    rin = None
    if refine_in is not None:
        arr = (C.c_float * 8)(*refine_in)
        rin = C.cast(arr, C.c_void_p)
    lib().orc_search(np.ascontiguousarray(ctf_spect, np.float64), ctf_spect.shape[0], px_n,
                     C.byref(p), mode, rin, C.byref(r))
    return r


def search1d(ctf_spect: np.ndarray, px_n: float, p: OrcParams):
    df, ph, sc = C.c_float(), C.c_float(), C.c_float()
    lib().orc_search1d(np.ascontiguousarray(ctf_spect, np.float64), ctf_spect.shape[0], px_n,
                       C.byref(p), C.byref(df), C.byref(ph), C.byref(sc))
    return df.value, ph.value, sc.value


def refine1d(ctf_spect: np.ndarray, px_n: float, p: OrcParams, init_df: float, df_range: float):
    df, ph, sc = C.c_float(), C.c_float(), C.c_float()
    lib().orc_refine1d(np.ascontiguousarray(ctf_spect, np.float64), ctf_spect.shape[0], px_n,
                       C.byref(p), init_df, df_range, C.byref(df), C.byref(ph), C.byref(sc))
    return df.value, ph.value, sc.value


def full_spectrum(ctf_spect, px_n, p, res) -> np.ndarray:
    tile = ctf_spect.shape[0]
    out = np.zeros((tile, tile), np.float32)
    lib().orc_full_spectrum(np.ascontiguousarray(ctf_spect, np.float64), tile, px_n, C.byref(p),
                            C.byref(res), out)
    return out


def find_ctf_image(img: np.ndarray, px_n: float, p: OrcParams, mode: int = 0, refine_in=None,
                   want_spectra: bool = False):
    """One package on an already-rescaled image (CFindCtf2D path)."""
    img = np.ascontiguousarray(img, np.float32)
    h, w = img.shape
    tile = p.tile_size
    r = OrcResult()
    raw = np.zeros((tile, tile // 2 + 1), np.float64) if want_spectra else None
    ctf = np.zeros((tile, tile // 2 + 1), np.float64) if want_spectra else None
    full = np.zeros((tile, tile), np.float32) if want_spectra else None
    rin = None
    if refine_in is not None:
        arr = (C.c_float * 8)(*refine_in)
        rin = C.cast(arr, C.c_void_p)

    def ptr(a):
        return None if a is None else a.ctypes.data_as(C.c_void_p)

    rc = lib().orc_find_ctf_image(img, w, h, w, px_n, C.byref(p), mode, rin, C.byref(r),
                                  ptr(raw), ptr(ctf), ptr(full))
    if rc != 0:
        raise ValueError("oracle failed (image smaller than one tile?)")
    if want_spectra:
        return r, raw, ctf, full
    return r


def series(imgs: list, p: OrcParams, order: list, is_tomo: bool):
    """CFindSeriesCtfs policy over raw images; returns results by image index."""
    arrs = [np.ascontiguousarray(a, np.float32) for a in imgs]
    h, w = arrs[0].shape
    ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    ordr = (C.c_int * len(order))(*order)
    res = (OrcResult * len(arrs))()
    rc = lib().orc_series(ptrs, len(arrs), w, h, C.byref(p), ordr, 1 if is_tomo else 0, res)
    if rc != 0:
        raise ValueError("oracle series failed")
    return [res[i] for i in range(len(arrs))]


def background1d(spectrum):
    """GBackground1D::DoIt: (background, start)."""
    sp = np.ascontiguousarray(spectrum, np.float32)
    bg = np.zeros_like(sp)
    st = C.c_int()
    lib().orc_background1d(sp, len(sp), bg, C.byref(st))
    return bg, st.value


def remove_bg1d(spectrum, bg, start):
    sp = np.array(spectrum, np.float32)
    lib().orc_remove_bg1d(sp, len(sp), np.ascontiguousarray(bg, np.float32), len(bg), int(start))
    return sp


def remove_bg2d(half, bg, start):
    sp = np.array(half, np.float32)
    lib().orc_remove_bg2d(sp, sp.shape[0], np.ascontiguousarray(bg, np.float32), len(bg), int(start))
    return sp


def counts(reset: bool = True):
    """(2D candidates, 1D grid points) evaluated since the last reset."""
    c = (C.c_longlong * 2)()
    lib().orc_counts(c, 1 if reset else 0)
    return int(c[0]), int(c[1])
