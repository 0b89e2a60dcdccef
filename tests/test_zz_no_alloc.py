"""gcf_avg_spectrum_noalloc: the spectrum entry point for callers that cannot
allocate device memory (a framework that owns every allocation, or a loop
that must not let cudaMalloc synchronise the device).

Called twice in a row through the C ABI on device buffers the test owns;
each output must match the context path's raw averaged spectrum within the
spectrum tolerance used elsewhere (1e-4 relative, 1e-5 of the mean as floor).
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


def test_noalloc_matches_context_path_twice(gpu_lib):
    import torch
    G = gpu_lib
    L = G.load_library()
    ctx = G.Context(0, 512, 0)
    op = G.make_optics(pixel_size=1.35)
    cases = [_img(51, 1536, 1536), _img(52, 1538, 1280)]   # aligned and unaligned tile starts
    for img in cases:
        h, w = img.shape
        ctx.setup(op, w, h)
        ctx.gen_half_spectrum(img)
        ref = ctx.half_spectrum(raw=True).astype(np.float64)
        d_img = torch.from_numpy(img).cuda()
        d_out = torch.zeros((512, 257), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        st = L.gcf_avg_spectrum_noalloc(C.c_void_p(d_img.data_ptr()), w, h, w,
                                        C.c_void_p(d_out.data_ptr()), None)
        assert st == 0, L.gcf_strerror(st)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().astype(np.float64)
        tol = 1e-4 * np.abs(ref) + 1e-5 * ref.mean()
        assert np.all(np.abs(got - ref) <= tol), float((np.abs(got - ref) / np.abs(ref)).max())


def test_noalloc_rejects_oversize_and_bad_args(gpu_lib):
    import torch
    L = gpu_lib.load_library()
    d = torch.zeros(16, dtype=torch.float32, device="cuda")
    p = C.c_void_p(d.data_ptr())
    # more than 4096 tiles (66 x 66 here) is beyond the static scratch
    assert L.gcf_avg_spectrum_noalloc(p, 17152, 17152, 17152, p, None) == 1
    assert L.gcf_avg_spectrum_noalloc(None, 1024, 1024, 1024, p, None) == 1
    assert L.gcf_avg_spectrum_noalloc(p, 256, 256, 256, p, None) == 1
