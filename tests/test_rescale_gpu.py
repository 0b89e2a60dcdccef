"""The hand-written Fourier-crop rescale (GCF_RESCALE_LINES, gcf_resize.cu)
against the cuFFT R2C + crop + C2R that the reference runs
(FindCTF/CRescaleImage.cpp:76-99, GCF_RESCALE_CUFFT, the default), on the batch's raw
sizes and on the edge cases of the line transforms: power-of-two lines
(direct FFTs) and Bluestein lines, an odd raw height, a rescale that keeps
the raw width (the Nyquist column of the raw R2C is kept), and a raw width
that is odd (not handled by the line transforms: the cuFFT path runs).

Bar: max |d| <= 1e-5 x rms of the cuFFT result, the bar the rescaled image
meets against the reference build (tests/test_ref_parity.py)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / np.sqrt((b * b).mean()))


CASES = [
    (4096, 4096, 1.0),    # 3412 x 3412: rows 2048 (direct), columns 4096 (direct) / 3412, new rows 1706
    (3838, 3710, 0.9),    # every line through Bluestein
    (5760, 4092, 0.8),    # raw rows 2880 (M = 8192)
    (1536, 1151, 0.93),   # odd raw height
    (2048, 2048, 0.6),    # 1024 x 1024: every line a power of two
    (100, 100, 1.197),    # new size = raw size: K = w/2 + 1
]


@pytest.mark.parametrize("w,h,px", CASES)
def test_line_rescale_matches_cufft(gpu_lib, w, h, px):
    G = gpu_lib
    rng = np.random.default_rng(w * 7 + h)
    img = rng.poisson(2.0, size=(h, w)).astype(np.float32)
    lines = G.Context(0, 512, 0)
    lines.set_rescale_impl(G.GCF_RESCALE_LINES)
    cufft = G.Context(0, 512, 0)
    a = lines.rescale(img, px)
    b = cufft.rescale(img, px)
    lines.close()
    cufft.close()
    assert a.shape == b.shape == G.rescale_dims(w, h, px)[1::-1]
    assert _rel(a, b) <= 1e-5, _rel(a, b)


@pytest.mark.parametrize("w,h", [(1537, 1024), (1024, 5000)])
def test_sizes_beyond_the_line_transforms_take_the_cufft_path(gpu_lib, w, h):
    """An odd raw width, and a raw height above 4096 (a column line too
    long): the cuFFT path runs, bit for bit."""
    G = gpu_lib
    img = np.random.default_rng(5).poisson(2.0, size=(h, w)).astype(np.float32)
    lines = G.Context(0, 512, 0)
    lines.set_rescale_impl(G.GCF_RESCALE_LINES)
    cufft = G.Context(0, 512, 0)
    assert np.array_equal(lines.rescale(img, 0.9), cufft.rescale(img, 0.9))
    lines.close()
    cufft.close()


def test_batch_through_line_rescale(gpu_lib):
    """A batch of micrographs below 1.2 A/px through gcf_run_batch with the
    line-transform rescale: each result within one search step of the cuFFT
    rescale's (the rescaled images differ at float rounding), and a CUDA
    graph of the call (the line kernels captured with their tables) replays
    the eager results bit for bit."""
    from gctffind_b200 import synth
    G = gpu_lib
    sizes = [(2048, 2048, 0.9), (1536, 1152, 1.0), (2000, 1400, 0.85), (1800, 1800, 1.1)]
    imgs, pxs = [], []
    for k, (w, h, px) in enumerate(sizes):
        spec = synth.MicrographSpec(width=w, height=h, pixel_size=px, df_min=14000.0 + 900 * k,
                                    df_max=14400.0 + 900 * k, azimuth_deg=15.0 * k, dose=2.0, seed=70 + k)
        imgs.append(synth.make_micrograph(spec, device="cuda"))
        pxs.append(px)
    op = G.make_optics()
    ref = G.Context(0, 512, 0)
    a = ref.run_batch(imgs, pxs, op)
    ref.close()
    ctx = G.Context(0, 512, 0)
    ctx.set_rescale_impl(G.GCF_RESCALE_LINES)
    ctx.set_graphs(True)
    b = [ctx.run_batch(imgs, pxs, op) for _ in range(3)]
    assert ctx.graph_info()["graph_launches"] == 1
    ctx.close()
    for x, y in zip(a, b[0]):
        step = max(20.0, 0.105 * 0.5 * (x.df_min + x.df_max) / 31.0)
        assert abs(x.df_min - y.df_min) <= step and abs(x.df_max - y.df_max) <= step, (x, y)
        assert abs(x.score - y.score) <= 1e-3
    assert [r.as_dict() for r in b[2]] == [r.as_dict() for r in b[0]]


def test_rescale_impl_rejects_unknown_values(gpu_lib):
    G = gpu_lib
    ctx = G.Context(0, 512, 0)
    with pytest.raises(G.GcfError):
        ctx.set_rescale_impl(7)
    ctx.close()


def test_device_views_at_odd_offsets(gpu_lib):
    """A caller's device image that starts 4 bytes past an allocation (a
    view at an odd float offset): both rescale implementations read it (the
    cuFFT path through an aligned copy, the line transforms with 4-byte
    loads) and agree with the rescale of the same pixels at an aligned
    address; so does a batch call on such views."""
    import torch
    G = gpu_lib
    w, h, px = 1536, 1152, 0.9
    rng = np.random.default_rng(11)
    host = rng.poisson(2.0, size=(h, w)).astype(np.float32)
    flat = torch.zeros(h * w + 1, device="cuda")
    view = flat[1:].view(h, w)
    view.copy_(torch.from_numpy(host).cuda())
    assert view.data_ptr() % 8 == 4
    ref = G.Context(0, 512, 0).rescale(host, px)
    for impl in (G.GCF_RESCALE_CUFFT, G.GCF_RESCALE_LINES):
        ctx = G.Context(0, 512, 0)
        ctx.set_rescale_impl(impl)
        out = ctx.rescale(view, px)
        assert _rel(out, ref) <= 1e-5, impl
        a = ctx.run_batch([view], [px], G.make_optics())[0]
        b = ctx.run_batch([torch.from_numpy(host).cuda()], [px], G.make_optics())[0]
        assert a.as_dict() == b.as_dict(), impl
        ctx.close()
