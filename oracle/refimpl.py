"""ctypes binding of the reference's own CTF path built from its sources
(oracle/_ref/libgcfref.so, recipe oracle/ref/Makefile).

TEST INFRASTRUCTURE ONLY: the parity tests, the golden-fixture script and
bench.py's reference arm use this module; the product package
(gctffind_b200) never imports it.  The library runs the reference's CUDA
kernels, so every call but ctf_theory (host math) needs a GPU.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libgcfref.so")
# the GCtfFind source tree: $GCF_REFERENCE_TREE, else a "reference" folder
# beside this repository
REF_TREE = os.environ.get("GCF_REFERENCE_TREE",
                          os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))

_lib = None
_F = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def available() -> bool:
    return os.path.exists(LIB_PATH)


def build(force: bool = False) -> bool:
    """Compile the reference sources when the source tree is present."""
    if available() and not force:
        return True
    if not os.path.isdir(os.path.join(REF_TREE, "FindCTF")):
        return False
    subprocess.check_call(["make", "-s", "-j8", "-C", os.path.join(HERE, "ref"), f"REF={REF_TREE}"])
    return available()


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not available():
        raise FileNotFoundError(f"{LIB_PATH} not built")
    L = C.CDLL(LIB_PATH)
    L.gref_run_series.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int,
                                  C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                                  C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_void_p,
                                  C.POINTER(C.c_char_p), C.c_int, _F, C.c_void_p, C.c_char_p,
                                  C.c_int, C.POINTER(C.c_double)]
    L.gref_run_series.restype = C.c_int
    L.gref_single.argtypes = [_F, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                              C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.c_void_p,
                              C.POINTER(C.c_int), C.POINTER(C.c_float), C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_void_p, _F, C.c_int]
    L.gref_single.restype = C.c_int
    L.gref_single1d.argtypes = [_F, C.c_int, C.c_int] + [C.c_float] * 6 + [C.c_int] * 4 + \
        [C.c_float, C.c_float, _F, C.c_int]
    L.gref_single1d.restype = C.c_int
    L.gref_background1d.argtypes = [_F, C.c_int, _F, C.POINTER(C.c_int), C.c_void_p, C.c_int,
                                    C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
    L.gref_background1d.restype = C.c_int
    L.gref_ctf_theory.argtypes = [C.c_float] * 9 + [C.c_int] + [_F] * 9
    L.gref_ctf_theory.restype = None
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def run_series(images, pixel_size, order, tilts=None, is_tomo=True, kv=300.0, cs_mm=2.7,
               amp_contrast=0.07, ext_phase_deg=0.0, ext_phase_range=0.0, tile=512, log_spect=0,
               gpu=0, names=None, full_spectra=False, out_ctf=None, quiet=True):
    """CFindSeriesCtfs::DoIt on host images.  Returns (results n x 5 as
    df_min, df_max, azimuth, ext_phase, score; full spectra or None;
    seconds spent in DoIt)."""
    arrs = [np.ascontiguousarray(a, np.float32) for a in images]
    n = len(arrs)
    h, w = arrs[0].shape
    ptrs = (C.c_void_p * n)(*[a.ctypes.data for a in arrs])
    ordr = (C.c_int * n)(*order)
    tl = np.ascontiguousarray(tilts if tilts is not None else np.zeros(n), np.float32)
    nm = (C.c_char_p * n)(*[(names[i] if names else "").encode() for i in range(n)])
    res = np.zeros((n, 5), np.float32)
    full = np.zeros((n, tile, tile), np.float32) if full_spectra else None
    sec = C.c_double()
    rc = lib().gref_run_series(ptrs, n, w, h, kv, cs_mm, amp_contrast, pixel_size, ext_phase_deg,
                               ext_phase_range, tile, log_spect, gpu, ordr, _ptr(tl), nm,
                               1 if is_tomo else 0, res, _ptr(full),
                               out_ctf.encode() if out_ctf else None, 1 if quiet else 0,
                               C.byref(sec))
    if rc != 0:
        raise RuntimeError(f"reference series failed: {rc}")
    return res, full, sec.value


def single(image, pixel_size, kv=300.0, cs_mm=2.7, amp_contrast=0.07, ext_phase_deg=0.0,
           ext_phase_range=0.0, tile=512, log_spect=0, gpu=0, refine=None, quiet=True):
    """One micrograph: rescale, spectra, Do2D (or Refine), full spectrum.
    Returns a dict of the reference's outputs."""
    img = np.ascontiguousarray(image, np.float32)
    h, w = img.shape
    dims = (C.c_int * 2)()
    npx = C.c_float()
    # the rescaled size is at most the raw size
    resc = np.zeros(w * h, np.float32)
    cx = tile // 2 + 1
    raw = np.zeros((tile, cx), np.float32)
    ctf = np.zeros((tile, cx), np.float32)
    full = np.zeros((tile, tile), np.float32)
    out = np.zeros(6, np.float32)
    rin = None
    if refine is not None:
        rarr = np.ascontiguousarray(refine, np.float32)
        rin = _ptr(rarr)
    rc = lib().gref_single(img, w, h, kv, cs_mm, amp_contrast, pixel_size, ext_phase_deg,
                           ext_phase_range, tile, log_spect, gpu, rin, dims, C.byref(npx),
                           _ptr(resc), _ptr(raw), _ptr(ctf), _ptr(full), out, 1 if quiet else 0)
    if rc != 0:
        raise RuntimeError(f"reference single failed: {rc}")
    nw, nh = dims[0], dims[1]
    return {"new_size": (nw, nh), "new_pixel_size": npx.value,
            "rescaled": resc[: nw * nh].reshape(nh, nw), "raw_half": raw, "ctf_half": ctf,
            "full": full, "result": out[:5], "ctf_res": float(out[5])}


def single1d(image, pixel_size, kv=300.0, cs_mm=2.7, amp_contrast=0.07, ext_phase_deg=0.0,
             ext_phase_range=0.0, tile=512, log_spect=0, gpu=0, refine=None, quiet=True):
    """CFindCtf1D::Do1D, or Refine1D(*refine) with refine = (init_df, range),
    on one micrograph.  Returns (defocus, extra phase, CC)."""
    img = np.ascontiguousarray(image, np.float32)
    h, w = img.shape
    out = np.zeros(3, np.float32)
    r0, r1 = (0.0, 0.0) if refine is None else refine
    rc = lib().gref_single1d(img, w, h, kv, cs_mm, amp_contrast, pixel_size, ext_phase_deg,
                             ext_phase_range, tile, log_spect, gpu, 0 if refine is None else 1,
                             r0, r1, out, 1 if quiet else 0)
    if rc != 0:
        raise RuntimeError(f"reference single1d failed: {rc}")
    return tuple(float(x) for x in out)


def background1d(spectrum, half=None, spec1d=None, gpu=0):
    """GBackground1D::DoIt on a 1D spectrum, then Remove2D on `half` and
    Remove1D on `spec1d`.  Returns (background, start, half_out, spec1d_out)."""
    sp = np.ascontiguousarray(spectrum, np.float32)
    n = len(sp)
    bg = np.zeros(n, np.float32)
    st = C.c_int()
    hin = None if half is None else np.ascontiguousarray(half, np.float32)
    hout = None if half is None else np.zeros_like(hin)
    s1 = None if spec1d is None else np.ascontiguousarray(spec1d, np.float32)
    s1o = None if spec1d is None else np.zeros_like(s1)
    rc = lib().gref_background1d(sp, n, bg, C.byref(st), _ptr(hin), 0 if hin is None else hin.shape[0],
                                 _ptr(hout), _ptr(s1), 0 if s1 is None else len(s1), _ptr(s1o), gpu)
    if rc != 0:
        raise RuntimeError(f"reference background1d failed: {rc}")
    return bg, st.value, hout, s1o


def ctf_theory(kv, cs_mm, amp_contrast, pixel_size, ast_tol, ext_phase_rad, df_min, df_max,
               azimuth_rad, freq, azimuth, phase):
    """The reference's CCTFTheory on arrays (host code: no GPU needed)."""
    freq = np.ascontiguousarray(freq, np.float32)
    azimuth = np.ascontiguousarray(azimuth, np.float32)
    phase = np.ascontiguousarray(phase, np.float32)
    n = len(freq)
    outs = [np.zeros(n, np.float32) for _ in range(5)]
    param = np.zeros(10, np.float32)
    lib().gref_ctf_theory(kv, cs_mm, amp_contrast, pixel_size, ast_tol, ext_phase_rad, df_min,
                          df_max, azimuth_rad, n, freq, azimuth, phase, *outs, param)
    keys = ["evaluate", "phase_shift", "defocus", "frequency", "zeros"]
    d = dict(zip(keys, outs))
    d["param"] = param
    return d
