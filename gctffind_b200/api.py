"""Python mirror of the GCtfFind CTF-estimation interface over the B200 C ABI.

The classes keep the reference's names and call shape so tests and tools
read like the reference: ``CCTFTheory.Setup`` (FindCTF/CCTFTheory.cpp:69-86),
``CFindCtf2D.Setup1/Setup2/GenHalfSpectrum/SetPhase/Do2D/Refine/
GenFullSpectrum/GetSpectSize`` (FindCTF/CFindCTFInc.h:541-623) with the
public result members ``m_fDfMin, m_fDfMax, m_fAstAng, m_fExtPhase,
m_fScore``.  All compute runs in lib/libgctf_b200.so (sm_100a); this module
only marshals arguments.  There is no CPU path: without the library (or a
GPU) every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgctf_b200.so")
CLI_PATH = os.path.join(HERE, "bin", "GCtfFind")

GCF_SPECT_FUSED = 0
GCF_SPECT_CUFFT = 1

GCF_RESCALE_CUFFT = 0
GCF_RESCALE_LINES = 1
GCF_RESCALE_GEMM = 2

GCF_SEARCH_PLAIN = 0
GCF_SEARCH_BF16 = 1
GCF_SEARCH_LEARNED = 2

# Every symbol include/gctf_b200.h declares.
EXPORTS = [
    "gcf_create", "gcf_destroy", "gcf_strerror", "gcf_last_error", "gcf_set_spectrum_impl",
    "gcf_set_fused_shape",
    "gcf_setup", "gcf_gen_half_spectrum", "gcf_set_phase", "gcf_do2d", "gcf_refine",
    "gcf_do1d", "gcf_refine1d",
    "gcf_get_spect_size", "gcf_get_half_spectrum", "gcf_gen_full_spectrum",
    "gcf_get_radial_average", "gcf_rescale_dims", "gcf_rescale", "gcf_run_series",
    "gcf_run_batch", "gcf_mrc_info", "gcf_mrc_read", "gcf_mrc_read_tilts", "gcf_mrc_write",
    "gcf_get_stage_times", "gcf_get_launch_count", "gcf_get_search_counts", "gcf_avg_spectrum_noalloc",
    "gcf_gemm_bf16", "gcf_run_batch_mode", "gcf_get_fast_counts", "gcf_get_fast_times",
    "gcf_nn_param_count", "gcf_nn_init", "gcf_nn_set_params", "gcf_nn_get_params", "gcf_nn_save",
    "gcf_nn_load", "gcf_set_learned_threshold", "gcf_set_rescale_impl", "gcf_nn_train", "gcf_nn_synth_inputs", "gcf_nn_inputs",
    "gcf_nn_forward_backward", "gcf_nn_eval_synthetic",
    "gcf_write_ctf_file", "gcf_write_ctf_file_ex", "gcf_set_package_callback", "gcf_set_graphs",
    "gcf_get_graph_info", "gcf_autotune", "gcf_mrc_load", "gcf_gemm_bf16_ex",
    "gcf_ctf_setup", "gcf_ctf_set_ext_phase", "gcf_ctf_get_ext_phase", "gcf_ctf_set_defocus",
    "gcf_ctf_set_defocus_px", "gcf_ctf_change_pixel_size", "gcf_ctf_evaluate",
    "gcf_ctf_phase_shift", "gcf_ctf_defocus", "gcf_ctf_frequency", "gcf_ctf_nth_zero",
    "gcf_ctf_equal",
    "gcf_background1d", "gcf_remove_background1d", "gcf_remove_background2d",
]


class GcfError(RuntimeError):
    pass


class Optics(C.Structure):
    _fields_ = [("kv", C.c_float), ("cs_mm", C.c_float), ("amp_contrast", C.c_float),
                ("pixel_size", C.c_float), ("ext_phase_deg", C.c_float),
                ("ext_phase_range", C.c_float)]


class Result(C.Structure):
    _fields_ = [("df_min", C.c_float), ("df_max", C.c_float), ("azimuth", C.c_float),
                ("ext_phase", C.c_float), ("score", C.c_float), ("ctf_res", C.c_float),
                ("df_1d", C.c_float), ("phase_1d", C.c_float), ("score_1d", C.c_float),
                ("lowpassed", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}

    def __repr__(self):
        return "Result(%s)" % ", ".join("%s=%.4f" % (k, v) if isinstance(v, float) else
                                        "%s=%s" % (k, v) for k, v in self.as_dict().items())


class CtfParam(C.Structure):
    """CCTFParam (FindCTF/CFindCTFInc.h:8-29): lengths in pixels, angles in radian."""
    _fields_ = [("wavelength", C.c_float), ("cs", C.c_float), ("amp_contrast", C.c_float),
                ("amp_phase", C.c_float), ("ext_phase", C.c_float), ("df_max", C.c_float),
                ("df_min", C.c_float), ("azimuth", C.c_float), ("ast_tol", C.c_float),
                ("pixel_size", C.c_float)]


class Tuning(C.Structure):
    _fields_ = [("fused_shape", C.c_int), ("gemm_tile_n", C.c_int), ("gemm_stages", C.c_int),
                ("gemm_persistent", C.c_int), ("fused_ms", C.c_float * 5), ("gemm_ms", C.c_float * 10)]

    def as_dict(self):
        return {"fused_shape": self.fused_shape, "gemm_tile_n": self.gemm_tile_n,
                "gemm_stages": self.gemm_stages, "gemm_persistent": self.gemm_persistent,
                "fused_ms": dict(zip(["8", "816", "16", "162", "168"], [round(x, 4) for x in self.fused_ms])),
                "gemm_ms": dict(zip(["256x2", "256x3", "256x4", "128x4", "128x6", "64x4", "p256x3", "p256x4",
                                     "p128x4", "p128x6"], [round(x, 4) for x in self.gemm_ms]))}


class Item(C.Structure):
    _fields_ = [("image", C.c_void_p), ("width", C.c_int), ("height", C.c_int),
                ("pixel_size", C.c_float)]


# void (*)(void* user, int done, int image, const gcf_result* result)
PACKAGE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_int, C.POINTER(Result))
GCF_CTF_COLUMN_RES = 1

_lib = None


def load_library(path: str = LIB_PATH):
    """Load the CUDA library; raises if it was not built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError("libgctf_b200.so not built: run `make -C gctffind_b200` "
                          "(or __graft_entry__.build())")
    L = C.CDLL(path)
    vp, i, f = C.c_void_p, C.c_int, C.c_float
    L.gcf_create.argtypes = [i, i, i, C.POINTER(vp)]
    L.gcf_destroy.argtypes = [vp]
    L.gcf_destroy.restype = None
    L.gcf_strerror.argtypes = [i]
    L.gcf_strerror.restype = C.c_char_p
    L.gcf_last_error.argtypes = [vp]
    L.gcf_last_error.restype = C.c_char_p
    L.gcf_set_spectrum_impl.argtypes = [vp, i]
    L.gcf_set_fused_shape.argtypes = [vp, i]
    L.gcf_setup.argtypes = [vp, C.POINTER(Optics), i, i]
    L.gcf_gen_half_spectrum.argtypes = [vp, vp, i, i]
    L.gcf_set_phase.argtypes = [vp, f, f]
    L.gcf_do2d.argtypes = [vp, C.POINTER(Result)]
    L.gcf_refine.argtypes = [vp, C.POINTER(f), C.POINTER(f), C.POINTER(f), C.POINTER(f),
                             C.POINTER(Result)]
    L.gcf_do1d.argtypes = [vp, C.POINTER(Result)]
    L.gcf_refine1d.argtypes = [vp, f, f, C.POINTER(Result)]
    L.gcf_get_spect_size.argtypes = [vp, C.POINTER(i), i]
    L.gcf_get_half_spectrum.argtypes = [vp, i, vp]
    L.gcf_gen_full_spectrum.argtypes = [vp, C.POINTER(Result), vp]
    L.gcf_get_radial_average.argtypes = [vp, vp]
    L.gcf_rescale_dims.argtypes = [i, i, f, C.POINTER(i), C.POINTER(i), C.POINTER(f)]
    L.gcf_rescale_dims.restype = None
    L.gcf_rescale.argtypes = [vp, vp, i, i, f, i, vp]
    L.gcf_run_series.argtypes = [vp, C.POINTER(vp), i, i, i, i, C.POINTER(Optics),
                                 C.POINTER(i), i, C.POINTER(Result), vp]
    L.gcf_run_batch.argtypes = [vp, C.POINTER(Item), i, i, C.POINTER(Optics), C.POINTER(Result)]
    L.gcf_mrc_info.argtypes = [C.c_char_p, C.POINTER(i), C.POINTER(i), C.POINTER(f), C.POINTER(i)]
    L.gcf_mrc_read.argtypes = [C.c_char_p, i, vp]
    L.gcf_mrc_read_tilts.argtypes = [C.c_char_p, vp, i]
    L.gcf_mrc_write.argtypes = [C.c_char_p, vp, i, i, i, f]
    L.gcf_get_stage_times.argtypes = [vp, C.POINTER(f)]
    L.gcf_get_launch_count.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.gcf_get_search_counts.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.gcf_avg_spectrum_noalloc.argtypes = [vp, i, i, i, vp, vp]
    ll = C.c_longlong
    L.gcf_gemm_bf16.argtypes = [vp, ll, vp, ll, i, i, i, vp, ll, i, i, vp]
    L.gcf_gemm_bf16_ex.argtypes = [vp, ll, vp, ll, i, i, i, vp, ll, i, i, i, vp]
    L.gcf_run_batch_mode.argtypes = [vp, C.POINTER(Item), i, i, C.POINTER(Optics), i, C.POINTER(Result)]
    L.gcf_get_fast_counts.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.gcf_get_fast_times.argtypes = [vp, C.POINTER(f)]
    ull, sz = C.c_ulonglong, C.c_size_t
    L.gcf_nn_param_count.argtypes = []
    L.gcf_nn_param_count.restype = sz
    L.gcf_nn_init.argtypes = [vp, ull]
    L.gcf_nn_set_params.argtypes = [vp, vp, sz]
    L.gcf_nn_get_params.argtypes = [vp, vp, sz]
    L.gcf_nn_save.argtypes = [vp, C.c_char_p]
    L.gcf_nn_load.argtypes = [vp, C.c_char_p]
    L.gcf_set_learned_threshold.argtypes = [vp, f]
    L.gcf_nn_train.argtypes = [vp, C.POINTER(Optics), i, i, ull, ull, f, vp]
    L.gcf_nn_synth_inputs.argtypes = [vp, C.POINTER(Optics), ull, ull, i, vp, vp, vp, vp]
    L.gcf_nn_inputs.argtypes = [vp, vp, vp, i, vp, vp]
    L.gcf_set_rescale_impl.argtypes = [vp, i]
    L.gcf_nn_forward_backward.argtypes = [vp, vp, vp, vp, i, vp, vp, vp]
    L.gcf_nn_eval_synthetic.argtypes = [vp, C.POINTER(Optics), ull, ull, i, i, C.POINTER(Result), vp]
    L.gcf_write_ctf_file.argtypes = [C.c_char_p, C.POINTER(Result), vp, vp, i, i]
    L.gcf_write_ctf_file_ex.argtypes = [C.c_char_p, C.POINTER(Result), vp, vp, i, i, i]
    L.gcf_set_package_callback.argtypes = [vp, PACKAGE_FN, vp]
    L.gcf_set_graphs.argtypes = [vp, i]
    L.gcf_mrc_load.argtypes = [vp, C.c_char_p, i, i, C.POINTER(vp)]
    L.gcf_autotune.argtypes = [vp, i, C.POINTER(Tuning)]
    L.gcf_get_graph_info.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.gcf_background1d.argtypes = [vp, vp, i, i, vp, C.POINTER(i)]
    L.gcf_remove_background1d.argtypes = [vp, vp, i, vp, i, i, i]
    L.gcf_remove_background2d.argtypes = [vp, vp, i, vp, i, i, i]
    P = C.POINTER(CtfParam)
    L.gcf_ctf_setup.argtypes = [P, f, f, f, f, f, f]
    L.gcf_ctf_set_ext_phase.argtypes = [P, f, i]
    L.gcf_ctf_get_ext_phase.argtypes = [P, i, C.POINTER(f)]
    L.gcf_ctf_set_defocus.argtypes = [P, f, f, f]
    L.gcf_ctf_set_defocus_px.argtypes = [P, f, f, f]
    L.gcf_ctf_change_pixel_size.argtypes = [P, f]
    for name in ("gcf_ctf_evaluate", "gcf_ctf_phase_shift", "gcf_ctf_frequency"):
        getattr(L, name).argtypes = [P, f, f, C.POINTER(f)]
    L.gcf_ctf_defocus.argtypes = [P, f, C.POINTER(f)]
    L.gcf_ctf_nth_zero.argtypes = [P, i, f, C.POINTER(f)]
    L.gcf_ctf_equal.argtypes = [P, P, f, C.POINTER(i)]
    for name in EXPORTS:   # every declared entry point must resolve
        getattr(L, name)
    _lib = L
    return L


def _check(status: int, ctx=None):
    if status != 0:
        L = load_library()
        msg = L.gcf_strerror(status).decode()
        if ctx is not None:
            detail = L.gcf_last_error(ctx).decode()
            if detail:
                msg += ": " + detail
        raise GcfError(msg)


def _ptr(a):
    """(pointer, is_device) of a numpy array or a torch tensor."""
    if isinstance(a, np.ndarray):
        return a.ctypes.data, 0
    if hasattr(a, "data_ptr"):
        return a.data_ptr(), 1 if a.is_cuda else 0
    raise TypeError("expected a numpy array or torch tensor")


def _as_f32(a):
    if isinstance(a, np.ndarray):
        return np.ascontiguousarray(a, dtype=np.float32)
    import torch
    if a.dtype != torch.float32 or not a.is_contiguous():
        a = a.to(torch.float32).contiguous()
    return a


def rescale_dims(w: int, h: int, px: float):
    L = load_library()
    nw, nh, npx = C.c_int(), C.c_int(), C.c_float()
    L.gcf_rescale_dims(w, h, px, C.byref(nw), C.byref(nh), C.byref(npx))
    return nw.value, nh.value, npx.value


def make_optics(kv=300.0, cs_mm=2.7, amp_contrast=0.07, pixel_size=1.0, ext_phase_deg=0.0,
                ext_phase_range=0.0) -> Optics:
    return Optics(kv, cs_mm, amp_contrast, pixel_size, ext_phase_deg, ext_phase_range)


class Context:
    """One CUDA stream + all device state (gcf_ctx)."""

    def __init__(self, gpu: int = 0, tile_size: int = 512, log_spect: int = 0,
                 spectrum_impl: int | None = None):
        L = load_library()
        h = C.c_void_p()
        _check(L.gcf_create(gpu, tile_size, log_spect, C.byref(h)))
        self._h = h
        self.tile_size = tile_size
        self.L = L
        if spectrum_impl is not None:
            _check(L.gcf_set_spectrum_impl(h, spectrum_impl), h)

    def close(self):
        if getattr(self, "_h", None):
            self.L.gcf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_spectrum_impl(self, impl: int):
        _check(self.L.gcf_set_spectrum_impl(self._h, impl), self._h)

    def set_rescale_impl(self, impl: int):
        """GCF_RESCALE_CUFFT (the reference's cuFFT calls, default),
        GCF_RESCALE_LINES (the library's line transforms: no plans to make) or
        GCF_RESCALE_GEMM (the crop as two BF16 tensor-core products)."""
        _check(self.L.gcf_set_rescale_impl(self._h, impl), self._h)

    def set_fused_shape(self, shape: int):
        """0 (auto), 8, 816, 16, 162 or 168: cluster shape of the fused tile kernel."""
        _check(self.L.gcf_set_fused_shape(self._h, shape), self._h)

    # -- CFindCtf2D shape ------------------------------------------------------
    def setup(self, optics: Optics, width: int, height: int):
        _check(self.L.gcf_setup(self._h, C.byref(optics), width, height), self._h)

    def gen_half_spectrum(self, img, pitch: int | None = None):
        img = _as_f32(img)
        p, dev = _ptr(img)
        if pitch is None:
            pitch = img.shape[-1]
        _check(self.L.gcf_gen_half_spectrum(self._h, p, pitch, dev), self._h)

    def set_phase(self, phase_deg: float, range_deg: float):
        _check(self.L.gcf_set_phase(self._h, phase_deg, range_deg), self._h)

    def do2d(self) -> Result:
        r = Result()
        _check(self.L.gcf_do2d(self._h, C.byref(r)), self._h)
        return r

    def refine(self, df_mean, ast_ratio, ast_angle, ext_phase) -> Result:
        arr = lambda v: (C.c_float * 2)(*v)
        r = Result()
        _check(self.L.gcf_refine(self._h, arr(df_mean), arr(ast_ratio), arr(ast_angle),
                                 arr(ext_phase), C.byref(r)), self._h)
        return r

    def do1d(self) -> Result:
        r = Result()
        _check(self.L.gcf_do1d(self._h, C.byref(r)), self._h)
        return r

    def refine1d(self, init_df: float, df_range: float) -> Result:
        r = Result()
        _check(self.L.gcf_refine1d(self._h, init_df, df_range, C.byref(r)), self._h)
        return r

    # -- GBackground1D (host numpy arrays) -------------------------------------
    def background1d(self, spectrum):
        """(background, start) of a 1D spectrum."""
        sp = np.ascontiguousarray(spectrum, np.float32)
        bg = np.zeros_like(sp)
        st = C.c_int()
        _check(self.L.gcf_background1d(self._h, sp.ctypes.data, len(sp), 0, bg.ctypes.data,
                                       C.byref(st)), self._h)
        return bg, st.value

    def remove_background1d(self, spectrum, background, start):
        sp = np.array(spectrum, np.float32)
        bg = np.ascontiguousarray(background, np.float32)
        _check(self.L.gcf_remove_background1d(self._h, sp.ctypes.data, len(sp), bg.ctypes.data,
                                              len(bg), int(start), 0), self._h)
        return sp

    def remove_background2d(self, half_spectrum, background, start):
        sp = np.array(half_spectrum, np.float32)
        bg = np.ascontiguousarray(background, np.float32)
        _check(self.L.gcf_remove_background2d(self._h, sp.ctypes.data, sp.shape[0], bg.ctypes.data,
                                              len(bg), int(start), 0), self._h)
        return sp

    def half_spectrum(self, raw: bool) -> np.ndarray:
        out = np.zeros((self.tile_size, self.tile_size // 2 + 1), np.float32)
        _check(self.L.gcf_get_half_spectrum(self._h, 1 if raw else 0, out.ctypes.data), self._h)
        return out

    def radial_average(self) -> np.ndarray:
        out = np.zeros(self.tile_size // 2 + 1, np.float32)
        _check(self.L.gcf_get_radial_average(self._h, out.ctypes.data), self._h)
        return out

    def full_spectrum(self, res: Result) -> np.ndarray:
        out = np.zeros((self.tile_size, self.tile_size), np.float32)
        _check(self.L.gcf_gen_full_spectrum(self._h, C.byref(res), out.ctypes.data), self._h)
        return out

    def rescale(self, img, px: float) -> np.ndarray:
        img = _as_f32(img)
        h, w = img.shape
        nw, nh, _ = rescale_dims(w, h, px)
        out = np.zeros((nh, nw), np.float32)
        p, dev = _ptr(img)
        _check(self.L.gcf_rescale(self._h, p, w, h, px, dev, out.ctypes.data), self._h)
        return out

    # -- batched paths -----------------------------------------------------------
    def run_series(self, images, optics: Optics, order=None, is_tomo: bool = True,
                   want_full: bool = False, on_package=None):
        """CFindSeriesCtfs policy over equal-sized images (gcf_run_series);
        on_package(done, image, result), if given, is called as each
        package's result becomes final, in processing order."""
        cb = None
        if on_package is not None:
            def _hook(user, done, image, r):
                on_package(done, image, Result.from_buffer_copy(r.contents))
            cb = PACKAGE_FN(_hook)
            _check(self.L.gcf_set_package_callback(self._h, cb, None), self._h)
        try:
            return self._run_series(images, optics, order, is_tomo, want_full)
        finally:
            if cb is not None:
                self.L.gcf_set_package_callback(self._h, PACKAGE_FN(), None)

    def _run_series(self, images, optics, order, is_tomo, want_full):
        imgs = [_as_f32(a) for a in images]
        n = len(imgs)
        h, w = imgs[0].shape
        ptrs = [_ptr(a) for a in imgs]
        dev = ptrs[0][1]
        if any(d != dev for _, d in ptrs):
            raise ValueError("images must all be on the host or all on the GPU")
        if order is None:
            order = list(range(n))
        parr = (C.c_void_p * n)(*[p for p, _ in ptrs])
        oarr = (C.c_int * n)(*order)
        res = (Result * n)()
        full = np.zeros((n, self.tile_size, self.tile_size), np.float32) if want_full else None
        _check(self.L.gcf_run_series(self._h, parr, n, w, h, dev, C.byref(optics), oarr,
                                     1 if is_tomo else 0, res,
                                     full.ctypes.data if want_full else None), self._h)
        out = [res[i] for i in range(n)]
        return (out, full) if want_full else out

    def run_batch(self, images, pixel_sizes, optics: Optics, mode: int = GCF_SEARCH_PLAIN):
        """Independent searches of micrographs of any size (one call);
        mode: GCF_SEARCH_PLAIN, GCF_SEARCH_BF16 or GCF_SEARCH_LEARNED."""
        imgs = [_as_f32(a) for a in images]
        n = len(imgs)
        items = (Item * n)()
        dev = None
        for k, a in enumerate(imgs):
            p, d = _ptr(a)
            dev = d if dev is None else dev
            if d != dev:
                raise ValueError("images must all be on the host or all on the GPU")
            items[k] = Item(p, a.shape[1], a.shape[0], float(pixel_sizes[k]))
        res = (Result * n)()
        _check(self.L.gcf_run_batch_mode(self._h, items, n, dev, C.byref(optics), int(mode), res), self._h)
        return [res[i] for i in range(n)]

    def mrc_load(self, path: str, z0: int = 0, n: int | None = None):
        """Sections of an MRC file converted to float on the GPU
        (gcf_mrc_load): device addresses, valid until the next load."""
        if n is None:
            n = mrc_info(path)["dims"][2] - z0
        out = (C.c_void_p * n)()
        _check(self.L.gcf_mrc_load(self._h, path.encode(), z0, n, out), self._h)
        return [out[k] for k in range(n)]

    def autotune(self, force: bool = False) -> dict:
        """Timed trials of the tile-kernel shapes and contraction tiles
        (gcf_autotune); the fastest become this context's choice."""
        t = Tuning()
        _check(self.L.gcf_autotune(self._h, 1 if force else 0, C.byref(t)), self._h)
        return t.as_dict()

    def set_graphs(self, on: bool = True):
        """CUDA graphs for repeated batch calls (gcf_set_graphs)."""
        _check(self.L.gcf_set_graphs(self._h, 1 if on else 0), self._h)

    def graph_info(self):
        """(graph launches of the last batch call, nodes and library kernels
        of the cached graph) -- gcf_get_graph_info."""
        c = (C.c_longlong * 4)()
        _check(self.L.gcf_get_graph_info(self._h, c), self._h)
        d = dict(zip(["graph_launches", "nodes", "kernels", "capture_fail"], list(c)))
        d["detail"] = self.L.gcf_last_error(self._h).decode()
        return d

    def fast_counts(self):
        """Contraction work of the last batched call (gcf_get_fast_counts)."""
        c = (C.c_longlong * 4)()
        _check(self.L.gcf_get_fast_counts(self._h, c), self._h)
        return dict(zip(["table_cand", "tensor_macs", "rescored", "fallbacks"], list(c)))

    # -- learned initialiser ------------------------------------------------------
    def nn_init(self, seed: int = 0):
        _check(self.L.gcf_nn_init(self._h, seed), self._h)

    def nn_params(self) -> np.ndarray:
        n = self.L.gcf_nn_param_count()
        out = np.zeros(n, np.float32)
        _check(self.L.gcf_nn_get_params(self._h, out.ctypes.data, n), self._h)
        return out

    def nn_set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        _check(self.L.gcf_nn_set_params(self._h, p.ctypes.data, p.size), self._h)

    def save_weights(self, path: str):
        _check(self.L.gcf_nn_save(self._h, path.encode()), self._h)

    def load_weights(self, path: str):
        _check(self.L.gcf_nn_load(self._h, path.encode()), self._h)

    def set_learned_threshold(self, tau: float):
        _check(self.L.gcf_set_learned_threshold(self._h, tau), self._h)

    def nn_train(self, optics: Optics, steps: int, batch: int, seed: int, first: int = 0, lr: float = 1e-3):
        losses = np.zeros(steps, np.float32)
        _check(self.L.gcf_nn_train(self._h, C.byref(optics), steps, batch, seed, first, lr,
                                   losses.ctypes.data), self._h)
        return losses

    def nn_synth_inputs(self, optics: Optics, seed: int, first: int, n: int):
        x1 = np.zeros((n, 256), np.float32)
        x2 = np.zeros((n, 256, 256), np.float32)
        t = np.zeros((n, 3), np.float32)
        p = np.zeros((n, 8), np.float32)
        _check(self.L.gcf_nn_synth_inputs(self._h, C.byref(optics), seed, first, n, x1.ctypes.data,
                                          x2.ctypes.data, t.ctypes.data, p.ctypes.data), self._h)
        return x1, x2, t, p

    def nn_inputs(self, spectra, pixel_sizes):
        """Network inputs (x1 n x 256, x2 n x 256 x 256) of background-removed
        half spectra (n x tile x tile/2+1, or one spectrum) of the given pixel sizes."""
        s = np.ascontiguousarray(spectra, np.float32)
        if s.ndim == 2:
            s = s[None]
        n = s.shape[0]
        px = np.ascontiguousarray(np.broadcast_to(np.asarray(pixel_sizes, np.float32), (n,)))
        x1 = np.zeros((n, 256), np.float32)
        x2 = np.zeros((n, 256, 256), np.float32)
        _check(self.L.gcf_nn_inputs(self._h, s.ctypes.data, px.ctypes.data, n, x1.ctypes.data, x2.ctypes.data),
               self._h)
        return x1, x2

    def nn_forward_backward(self, x1, x2, target):
        x1 = np.ascontiguousarray(x1, np.float32)
        x2 = np.ascontiguousarray(x2, np.float32)
        target = np.ascontiguousarray(target, np.float32)
        n = x1.shape[0]
        loss = np.zeros(1, np.float32)
        grads = np.zeros(self.L.gcf_nn_param_count(), np.float32)
        pred = np.zeros((n, 3), np.float32)
        _check(self.L.gcf_nn_forward_backward(self._h, x1.ctypes.data, x2.ctypes.data, target.ctypes.data, n,
                                              loss.ctypes.data, grads.ctypes.data, pred.ctypes.data), self._h)
        return float(loss[0]), grads, pred

    def nn_eval_synthetic(self, optics: Optics, seed: int, first: int, n: int, mode: int):
        res = (Result * n)()
        p = np.zeros((n, 8), np.float32)
        _check(self.L.gcf_nn_eval_synthetic(self._h, C.byref(optics), seed, first, n, int(mode), res,
                                            p.ctypes.data), self._h)
        return [res[i] for i in range(n)], p

    def fast_times(self):
        """Device ms of the contraction stages of the last batched call."""
        t = (C.c_float * 5)()
        _check(self.L.gcf_get_fast_times(self._h, t), self._h)
        return dict(zip(["bin", "product", "table", "finish", "network"], list(t)))

    def stage_times(self):
        t = (C.c_float * 7)()
        _check(self.L.gcf_get_stage_times(self._h, t), self._h)
        keys = ["upload", "tile_kernel", "spectrum", "post", "search1d", "search2d", "total"]
        return dict(zip(keys, list(t)))

    def search_counts(self):
        """Search work of the last batched call (gcf_get_search_counts)."""
        c = (C.c_longlong * 4)()
        _check(self.L.gcf_get_search_counts(self._h, c), self._h)
        return dict(zip(["cand2d", "pairs2d", "cand1d", "pairs1d"], list(c)))

    def launch_count(self) -> int:
        v = C.c_longlong()
        _check(self.L.gcf_get_launch_count(self._h, C.byref(v)), self._h)
        return v.value


# ---------------------------------------------------------------------------
# Reference-shaped classes
# ---------------------------------------------------------------------------
class CCTFTheory:
    """CCTFTheory (FindCTF/CCTFTheory.cpp:9-301) over the library's host CTF
    math: same method names, units and float/double arithmetic."""

    def __init__(self):
        self.param = CtfParam()
        self.param.pixel_size = 1.0
        self.optics = make_optics()

    def _f(self, fn, *args):
        out = C.c_float()
        _check(fn(C.byref(self.param), *args, C.byref(out)))
        return out.value

    def Setup(self, fKv, fCs, fAmpContrast, fPixelSize, fAstTol=100.0, fExtPhase=0.0):
        """fExtPhase in radian, as in the reference."""
        L = load_library()
        _check(L.gcf_ctf_setup(C.byref(self.param), fKv, fCs, fAmpContrast, fPixelSize, fAstTol,
                               fExtPhase))
        self.optics = make_optics(fKv, fCs, fAmpContrast, fPixelSize,
                                  float(np.float32(fExtPhase) / np.float32(0.017453)), 0.0)

    def SetExtPhase(self, fExtPhase, bDegree):
        _check(load_library().gcf_ctf_set_ext_phase(C.byref(self.param), fExtPhase, int(bDegree)))

    def GetExtPhase(self, bDegree):
        L = load_library()
        out = C.c_float()
        _check(L.gcf_ctf_get_ext_phase(C.byref(self.param), int(bDegree), C.byref(out)))
        return out.value

    def SetPixelSize(self, fPixSize):
        self.param.pixel_size = fPixSize

    def ChangePixelSize(self, fNewPixSize):
        _check(load_library().gcf_ctf_change_pixel_size(C.byref(self.param), fNewPixSize))

    def SetDefocus(self, fDefocusMin, fDefocusMax, fAstAzimuth):
        _check(load_library().gcf_ctf_set_defocus(C.byref(self.param), fDefocusMin, fDefocusMax,
                                                  fAstAzimuth))

    def SetDefocusInPixel(self, fDefocusMin, fDefocusMax, fAstAzimuth):
        _check(load_library().gcf_ctf_set_defocus_px(C.byref(self.param), fDefocusMin, fDefocusMax,
                                                     fAstAzimuth))

    def GetParam(self, bCopy=False):
        if not bCopy:
            return self.param
        c = CtfParam()
        C.pointer(c)[0] = self.param
        return c

    def SetParam(self, param: CtfParam):
        C.pointer(self.param)[0] = param

    def Evaluate(self, fFreq, fAzimuth):
        return self._f(load_library().gcf_ctf_evaluate, fFreq, fAzimuth)

    def CalcPhaseShift(self, fFreq, fAzimuth):
        return self._f(load_library().gcf_ctf_phase_shift, fFreq, fAzimuth)

    def CalcDefocus(self, fAzimuth):
        return self._f(load_library().gcf_ctf_defocus, fAzimuth)

    def CalcFrequency(self, fPhaseShift, fAzimuth):
        return self._f(load_library().gcf_ctf_frequency, fPhaseShift, fAzimuth)

    def CalcNthZero(self, iNthZero, fAzimuth):
        return self._f(load_library().gcf_ctf_nth_zero, int(iNthZero), fAzimuth)

    def EqualTo(self, other: "CCTFTheory", fDfTol):
        out = C.c_int()
        _check(load_library().gcf_ctf_equal(C.byref(self.param), C.byref(other.param), fDfTol,
                                            C.byref(out)))
        return bool(out.value)

    def GetPixelSize(self):
        return self.param.pixel_size

    def GetCopy(self):
        c = CCTFTheory()
        c.SetParam(self.param)
        c.optics = Optics(*[getattr(self.optics, k) for k, _ in Optics._fields_])
        return c


class CFindCtf2D:
    """CFindCtf2D call shape (FindCTF/CFindCTFInc.h:581-615, with the Do1D /
    Refine1D of its CFindCtf1D base) on a Context."""

    def __init__(self, tile_size: int = 512, log_spect: int = 0, gpu: int = 0, ctx=None):
        self.ctx = ctx or Context(gpu, tile_size, log_spect)
        self.m_fDfMin = self.m_fDfMax = self.m_fAstAng = 0.0
        self.m_fExtPhase = self.m_fScore = 0.0
        self._theory = None
        self._result = None

    def Setup1(self, theory: CCTFTheory):
        self._theory = theory

    def Setup2(self, img_size):
        self.ctx.setup(self._theory.optics, int(img_size[0]), int(img_size[1]))

    def SetPhase(self, fInitPhase, fPhaseRange):
        self.ctx.set_phase(fInitPhase, fPhaseRange)

    def GenHalfSpectrum(self, img):
        self.ctx.gen_half_spectrum(img)

    def _take(self, r: Result):
        self._result = r
        self.m_fDfMin, self.m_fDfMax = r.df_min, r.df_max
        self.m_fAstAng, self.m_fExtPhase, self.m_fScore = r.azimuth, r.ext_phase, r.score

    def Do2D(self):
        self._take(self.ctx.do2d())

    def Refine(self, afDfMean, afAstRatio, afAstAngle, afExtPhase):
        self._take(self.ctx.refine(afDfMean, afAstRatio, afAstAngle, afExtPhase))

    # CFindCtf1D (FindCTF/CFindCtf1D.cpp:49-67), the base of CFindCtf2D
    def Do1D(self):
        self._take(self.ctx.do1d())

    def Refine1D(self, fInitDf, fDfRange):
        self._take(self.ctx.refine1d(fInitDf, fDfRange))

    def GenFullSpectrum(self):
        return self.ctx.full_spectrum(self._result)

    def GetSpectSize(self, bHalf: bool):
        t = self.ctx.tile_size
        return (t // 2 + 1, t) if bHalf else (t, t)

    def GetHalfSpect(self, bRaw: bool):
        return self.ctx.half_spectrum(bRaw)


# ---------------------------------------------------------------------------
# MRC helpers
# ---------------------------------------------------------------------------
def mrc_info(path: str):
    L = load_library()
    dims = (C.c_int * 3)()
    mode, px, nf = C.c_int(), C.c_float(), C.c_int()
    _check(L.gcf_mrc_info(path.encode(), dims, C.byref(mode), C.byref(px), C.byref(nf)))
    return {"dims": tuple(dims), "mode": mode.value, "pixel_size": px.value, "ext_floats": nf.value}


def mrc_read(path: str, z: int = 0) -> np.ndarray:
    L = load_library()
    info = mrc_info(path)
    nx, ny, _ = info["dims"]
    out = np.zeros((ny, nx), np.float32)
    _check(L.gcf_mrc_read(path.encode(), z, out.ctypes.data))
    return out


def mrc_read_tilts(path: str, n: int) -> np.ndarray:
    L = load_library()
    out = np.zeros(n, np.float32)
    _check(L.gcf_mrc_read_tilts(path.encode(), out.ctypes.data, n))
    return out


def write_ctf_file(path: str, results, tilts=None, names=None, is_tomo: bool = False,
                   ctf_res: bool = False):
    """CSaveCtfResults::SaveCTF (+ SaveImod for tilt series); ctf_res adds
    the spectral-CC resolution as a last column (not in the reference)."""
    L = load_library()
    n = len(results)
    res = (Result * n)(*results)
    t = np.ascontiguousarray(tilts if tilts is not None else np.zeros(n), np.float32)
    nm = (C.c_char_p * n)(*[(x or "").encode() for x in (names or [""] * n)])
    _check(L.gcf_write_ctf_file_ex(path.encode(), res, t.ctypes.data, C.cast(nm, C.c_void_p), n,
                                   1 if is_tomo else 0, GCF_CTF_COLUMN_RES if ctf_res else 0))


def mrc_write(path: str, data: np.ndarray, pixel_size: float = 1.0):
    L = load_library()
    data = np.ascontiguousarray(data, np.float32)
    if data.ndim == 2:
        data = data[None]
    nz, ny, nx = data.shape
    _check(L.gcf_mrc_write(path.encode(), data.ctypes.data, nx, ny, nz, pixel_size))


@dataclass
class SeriesOrder:
    """Processing order of a tilt series: the zero tilt first, then the
    others in file order (CLoadImages::mReadTomo, MrcUtil/CLoadImages.cpp:71-91,
    CInputFolder::FindZeroTilt, CInputFolder.cpp:50-69)."""
    zero_tilt: int
    order: list


def series_order(tilts) -> SeriesOrder:
    n = len(tilts)
    if n > 1 and abs(float(tilts[0]) - float(tilts[1])) < 0.0001:
        z = n // 2
    else:
        z, fmin = -1, 10000.0
        for i, t in enumerate(tilts):
            a = abs(float(np.float32(t)))
            if a >= fmin:
                continue
            fmin, z = a, i
        if z < 0:
            z = n // 2
    return SeriesOrder(z, [z] + [i for i in range(n) if i != z])
