"""gcf_mrc_load: MRC sections widened to float on the GPU equal the host
conversion of CLoadImages::mToFloat (MrcUtil/CLoadImages.cpp:146-181, here
gcf_mrc_read) bit for bit, for every supported mode, both byte orders,
ragged sizes (pixel counts not a multiple of 4), a section range, and more
sections than the two staging buffers; the CLI's stack path runs on it."""
import ctypes as C

import numpy as np
import pytest

from test_library_cpu import _write_mrc

pytestmark = pytest.mark.gpu


def _cudart():
    # the runtime the library was loaded with (same soname)
    for name in ("libcudart.so.12", "libcudart.so"):
        try:
            lib = C.CDLL(name)
        except OSError:
            continue
        lib.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
        return lib
    pytest.fail("libcudart not loadable")


def _dev_to_host(ptr, ny, nx):
    out = np.empty((ny, nx), np.float32)
    assert _cudart().cudaMemcpy(out.ctypes.data, ptr, ny * nx * 4, 2) == 0   # device -> host
    return out


@pytest.mark.parametrize("mode,swap", [(0, False), (1, False), (1, True), (2, False), (2, True), (6, False),
                                       (6, True)])
def test_gpu_load_matches_host_conversion(gpu_lib, tmp_path, mode, swap):
    G = gpu_lib
    rng = np.random.default_rng(10 + mode)
    nz, ny, nx = 5, 37, 51          # 1887 pixels: not a multiple of 4
    if mode == 2:
        a = rng.normal(0, 100, size=(nz, ny, nx)).astype(np.float32)
    else:
        hi = {0: 256, 1: 32767, 6: 65535}[mode]
        lo = -32768 if mode == 1 else 0
        a = rng.integers(lo, hi, size=(nz, ny, nx))
    p = str(tmp_path / f"m{mode}{int(swap)}.mrc")
    _write_mrc(p, a, mode, swap=swap)
    ctx = G.Context(0, 512, 0)
    ptrs = ctx.mrc_load(p)
    assert len(ptrs) == nz
    for z in range(nz):
        got = _dev_to_host(ptrs[z], ny, nx)
        assert np.array_equal(got, G.mrc_read(p, z)), (mode, swap, z)
    # a section range
    ptrs = ctx.mrc_load(p, 2, 2)
    for k in range(2):
        assert np.array_equal(_dev_to_host(ptrs[k], ny, nx), G.mrc_read(p, 2 + k))
    with pytest.raises(G.GcfError):
        ctx.mrc_load(p, 4, 2)
    ctx.close()


def test_gpu_loaded_stack_runs_like_host_images(gpu_lib, tmp_path):
    """The device images of gcf_mrc_load give gcf_run_series the results of
    the same sections passed from the host (mode 1 stack, as detectors
    write it)."""
    from gctffind_b200 import synth
    G = gpu_lib
    tilts = [-3.0, 0.0, 3.0]
    imgs = np.stack([synth.make_micrograph(synth.MicrographSpec(width=1024, height=1024, pixel_size=1.35,
                                                                df_min=17000.0, df_max=17300.0,
                                                                azimuth_deg=12.0, dose=20.0, seed=900 + k,
                                                                tilt_deg=t)).numpy()
                     for k, t in enumerate(tilts)])
    ints = np.clip(np.rint(imgs), -32768, 32767).astype(np.int16)
    p = str(tmp_path / "stack16.mrc")
    _write_mrc(p, ints, 1)
    ctx = G.Context(0, 512, 0)
    op = G.make_optics(pixel_size=1.35)
    order = G.series_order(tilts).order
    host = [G.mrc_read(p, z) for z in range(3)]
    ref = ctx.run_series(host, op, order, is_tomo=True)
    dev_ptrs = ctx.mrc_load(p)
    # wrap the device addresses for the C ABI call (is_device = 1)
    L = G.load_library()
    parr = (C.c_void_p * 3)(*dev_ptrs)
    oarr = (C.c_int * 3)(*order)
    res = (G.Result * 3)()
    st = L.gcf_run_series(ctx._h, parr, 3, 1024, 1024, 1, C.byref(op), oarr, 1, res, None)
    assert st == 0, L.gcf_strerror(st)
    for r, q in zip(res, ref):
        assert r.as_dict() == q.as_dict()
    ctx.close()
