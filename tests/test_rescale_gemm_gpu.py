"""The Fourier-crop rescale as two BF16 tensor-core products
(GCF_RESCALE_GEMM, gcf_rsgemm.cu) against the cuFFT R2C + crop + C2R that the
reference runs (FindCTF/CRescaleImage.cpp:76-99, GCF_RESCALE_CUFFT).

The products take BF16 operands (8 significant bits) with FP32 accumulation,
so the result is not bit-identical to cuFFT.  Bar, relative to the standard
deviation of the cuFFT result (the fluctuations that carry the CTF, not the
image mean, which the library removes before the BF16 conversion and adds
back in FP32): rms error <= 6e-3, max error <= 8e-2.  A BF16 emulation of
the same products in numpy gives 3.1e-3 to 3.6e-3 rms on Poisson images,
with or without a 5000-count offset.  A mistake in the maps or the
rank-one Nyquist term gives errors of order 1."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    (4096, 4096, 1.0),    # 3412 x 3412
    (3838, 3710, 0.9),    # 2878 x 2782
    (5760, 4092, 0.8),    # 3840 x 2728
    (1536, 1151, 0.93),   # odd raw height
    (1537, 1024, 0.9),    # odd raw width
    (2048, 2048, 0.6),    # 1024 x 1024
    (100, 100, 1.197),    # new size = raw size
    (300, 250, 0.85),     # smaller than one product tile
]


def _errs(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    sd = float((b - b.mean()).std())
    e = a - b
    return float(np.sqrt((e * e).mean()) / sd), float(np.abs(e).max() / sd)


def _pair(G, img, px):
    gemm = G.Context(0, 512, 0)
    gemm.set_rescale_impl(G.GCF_RESCALE_GEMM)
    cufft = G.Context(0, 512, 0)
    a = gemm.rescale(img, px)
    b = cufft.rescale(img, px)
    gemm.close()
    cufft.close()
    return a, b


@pytest.mark.parametrize("w,h,px", CASES)
def test_gemm_rescale_matches_cufft(gpu_lib, w, h, px):
    G = gpu_lib
    rng = np.random.default_rng(w * 7 + h)
    img = rng.poisson(2.0, size=(h, w)).astype(np.float32)
    a, b = _pair(G, img, px)
    assert a.shape == b.shape == G.rescale_dims(w, h, px)[1::-1]
    rms, mx = _errs(a, b)
    assert rms <= 6e-3 and mx <= 8e-2, (rms, mx)


def test_large_image_mean_is_removed_before_bf16(gpu_lib):
    """A 5000-count offset (a frame stored with a pedestal): the error stays
    at the scale of the fluctuations, and the mean comes back exactly."""
    G = gpu_lib
    rng = np.random.default_rng(3)
    img = (rng.poisson(2.0, size=(1536, 1600)) + 5000).astype(np.float32)
    a, b = _pair(G, img, 0.9)
    rms, mx = _errs(a, b)
    assert rms <= 6e-3 and mx <= 8e-2, (rms, mx)
    assert abs(a.mean() - b.mean()) <= 1e-4 * abs(b.mean())


def test_gemm_rescale_matches_oracle(gpu_lib):
    """Against the FP64 oracle of the rescale (oracle/oracle.py rescale) on
    a small frame, with the same bar."""
    from oracle import oracle as O
    G = gpu_lib
    img = np.random.default_rng(9).poisson(3.0, size=(250, 300)).astype(np.float32)
    ctx = G.Context(0, 512, 0)
    ctx.set_rescale_impl(G.GCF_RESCALE_GEMM)
    a = ctx.rescale(img, 0.85)
    ctx.close()
    rms, mx = _errs(a, O.rescale(img, 0.85))
    assert rms <= 6e-3 and mx <= 8e-2, (rms, mx)


def test_sides_beyond_the_limit_take_the_cufft_path(gpu_lib):
    """A raw side above 16384: the cuFFT path runs, bit for bit."""
    G = gpu_lib
    img = np.random.default_rng(5).poisson(2.0, size=(64, 16400)).astype(np.float32)
    a, b = _pair(G, img, 0.9)
    assert np.array_equal(a, b)


def test_batch_through_gemm_rescale(gpu_lib):
    """A batch below 1.2 A/px through gcf_run_batch with the tensor-core
    rescale: each result within one search step of the cuFFT rescale's, and
    a CUDA graph of the call replays the eager results bit for bit."""
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
    ctx.set_rescale_impl(G.GCF_RESCALE_GEMM)
    ctx.set_graphs(True)
    b = [ctx.run_batch(imgs, pxs, op) for _ in range(3)]
    assert ctx.graph_info()["graph_launches"] == 1
    ctx.close()
    for x, y in zip(a, b[0]):
        step = max(20.0, 0.105 * 0.5 * (x.df_min + x.df_max) / 31.0)
        assert abs(x.df_min - y.df_min) <= step and abs(x.df_max - y.df_max) <= step, (x, y)
        assert abs(x.score - y.score) <= 5e-3
    assert [r.as_dict() for r in b[2]] == [r.as_dict() for r in b[0]]
