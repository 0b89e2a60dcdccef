"""gcf_avg_spectrum_noalloc: the spectrum entry point for callers that cannot
allocate device memory (a framework that owns every device allocation, or an
acquisition loop that must not let cudaMalloc synchronise the device).

Each case calls the entry point twice in a row on the same device image
through the C ABI, on buffers the test owns.  Both outputs must match the
context path's raw averaged spectrum and, for the small cases, the FP64
oracle's, within the spectrum tolerance used elsewhere (1e-4 relative, with
1e-5 of the mean as floor).  Between the second and a third call the
device's free memory must not change: the entry point allocates nothing
(the first calls may load kernel code, so they are not counted).
This file is collected last so a failure here leaves the other tests run.
"""
import ctypes as C

import numpy as np
import pytest

from gctffind_b200 import synth

pytestmark = pytest.mark.gpu


def _img(seed, w, h):
    spec = synth.MicrographSpec(width=w, height=h, pixel_size=1.35, df_min=15900.0,
                                df_max=16100.0, azimuth_deg=5.0, dose=3.0, seed=seed)
    return synth.make_micrograph(spec).numpy()


def _tol(ref):
    return 1e-4 * np.abs(ref) + 1e-5 * ref.mean()


def _noalloc(L, d_img, w, h, pitch, d_out):
    st = L.gcf_avg_spectrum_noalloc(C.c_void_p(d_img.data_ptr()), w, h, pitch,
                                    C.c_void_p(d_out.data_ptr()), None)
    assert st == 0, L.gcf_strerror(st)


def _check_case(G, L, ctx, img, pitch=None, oracle=None):
    import torch
    h, w = img.shape
    pitch = pitch or w
    host = np.zeros((h, pitch), np.float32)
    host[:, :w] = img
    ctx.setup(G.make_optics(pixel_size=1.35), w, h)
    ctx.gen_half_spectrum(host, pitch=pitch)
    ref = ctx.half_spectrum(raw=True).astype(np.float64)
    d_img = torch.from_numpy(host).cuda()
    outs = []
    for _ in range(2):   # two calls in a row on the same image
        d_out = torch.full((512, 257), float("nan"), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        _noalloc(L, d_img, w, h, pitch, d_out)
        torch.cuda.synchronize()
        outs.append((d_out, d_out.cpu().numpy().astype(np.float64)))
    for _, got in outs:
        assert np.all(np.abs(got - ref) <= _tol(ref)), float((np.abs(got - ref) / np.abs(ref)).max())
    if oracle is not None:
        oraw = oracle.avg_spectrum(img, 512)
        for _, got in outs:
            assert np.all(np.abs(got - oraw) <= _tol(oraw)), float((np.abs(got - oraw) / np.abs(oraw)).max())
    # no device allocation: free memory is unchanged across a further call
    free0, _ = torch.cuda.mem_get_info()
    _noalloc(L, d_img, w, h, pitch, outs[0][0])
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_matches_context_path_and_oracle(gpu_lib, oracle):
    G = gpu_lib
    L = G.load_library()
    ctx = G.Context(0, 512, 0)
    # aligned tile starts; unaligned ones (odd offset); an odd pitch (4-byte row loads)
    _check_case(G, L, ctx, _img(51, 1536, 1536), oracle=oracle)
    _check_case(G, L, ctx, _img(52, 1538, 1280), oracle=oracle)
    _check_case(G, L, ctx, _img(53, 1280, 1024), pitch=1281, oracle=oracle)
    ctx.close()


def test_noalloc_at_the_tile_limit(gpu_lib):
    """16384 x 16384 holds 63 x 63 = 3969 tiles, 16 work items of 249 or 248
    tiles: close to the 4096-tile limit of the static scratch."""
    import torch
    G = gpu_lib
    L = G.load_library()
    ctx = G.Context(0, 512, 0)
    g = torch.Generator(device="cuda").manual_seed(9)
    img = torch.poisson(torch.full((16384, 16384), 3.0, device="cuda"), generator=g).cpu().numpy()
    _check_case(G, L, ctx, img)
    ctx.close()


def test_noalloc_rejects_oversize_and_bad_args(gpu_lib):
    import torch
    L = gpu_lib.load_library()
    d = torch.zeros(16, dtype=torch.float32, device="cuda")
    p = C.c_void_p(d.data_ptr())
    # more than 4096 tiles (66 x 66 here) is beyond the static scratch
    assert L.gcf_avg_spectrum_noalloc(p, 17152, 17152, 17152, p, None) == 1
    assert L.gcf_avg_spectrum_noalloc(None, 1024, 1024, 1024, p, None) == 1
    assert L.gcf_avg_spectrum_noalloc(p, 256, 256, 256, p, None) == 1
