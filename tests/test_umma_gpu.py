"""tcgen05 BF16 tensor-core product (gcf_gemm_bf16) against a torch FP32
reference of the same product.

The BF16 inputs are exact in FP32 and so are their products; only the order
of the FP32 additions differs, so every element must agree with the FP32
reference within 1e-4 of the row's sum of |a_k b_k| (plus 1e-6 absolute).
Shapes cover full and ragged tiles in M, N and K (out-of-range rows and K
columns are zero-filled by the loads, and the stores are masked) for every
supported tile width and pipeline depth.
"""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu

CONFIGS = [(256, 2), (256, 3), (256, 4), (128, 2), (128, 4), (128, 6), (64, 2), (64, 4), (32, 2), (32, 4)]


def _run(L, a, b, tile_n, stages):
    import torch
    m, k = a.shape
    n = b.shape[0]
    d = torch.full((m, n), float("nan"), dtype=torch.float32, device="cuda")
    st = L.gcf_gemm_bf16(C.c_void_p(a.data_ptr()), a.stride(0), C.c_void_p(b.data_ptr()), b.stride(0),
                         m, n, k, C.c_void_p(d.data_ptr()), d.stride(0), tile_n, stages, None)
    assert st == 0, L.gcf_strerror(st)
    return d


def _check(a, b, d):
    import torch
    ref = a.float() @ b.float().T
    scale = a.float().abs() @ b.float().abs().T
    err = (d - ref).abs()
    assert torch.all(err <= 1e-4 * scale + 1e-6), float((err / (scale + 1e-6)).max())


@pytest.mark.parametrize("tile_n,stages", CONFIGS)
def test_gemm_matches_fp32_reference(gpu_lib, tile_n, stages):
    import torch
    L = gpu_lib.load_library()
    g = torch.Generator(device="cuda").manual_seed(tile_n * 10 + stages)
    for (m, n, k) in [(128, tile_n, 64), (256, 512, 512), (300, 200, 72), (130, 40, 200)]:
        a = torch.randn((m, k), generator=g, device="cuda").to(torch.bfloat16)
        b = torch.randn((n, k), generator=g, device="cuda").to(torch.bfloat16)
        _check(a, b, _run(L, a, b, tile_n, stages))


def test_gemm_strided_operands(gpu_lib):
    """Row pitches larger than K (a view into a wider buffer) and an output
    pitch larger than N."""
    import torch
    L = gpu_lib.load_library()
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn((384, 136), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((96, 200), generator=g, device="cuda").to(torch.bfloat16)
    a, b = A[:, :128], B[:, :128]
    D = torch.zeros((384, 100), dtype=torch.float32, device="cuda")
    st = L.gcf_gemm_bf16(C.c_void_p(a.data_ptr()), 136, C.c_void_p(b.data_ptr()), 200, 384, 96, 128,
                         C.c_void_p(D.data_ptr()), 100, 64, 2, None)
    assert st == 0
    _check(a, b, D[:, :96])


def test_gemm_rejects_unaligned(gpu_lib):
    import torch
    L = gpu_lib.load_library()
    a = torch.zeros((128, 72), dtype=torch.bfloat16, device="cuda")
    d = torch.zeros((128, 128), dtype=torch.float32, device="cuda")
    p = C.c_void_p(a.data_ptr())
    # pitch of 70 elements is 140 bytes: not a multiple of 16
    assert L.gcf_gemm_bf16(p, 70, p, 72, 128, 128, 70, C.c_void_p(d.data_ptr()), 128, 128, 2, None) == 1
    # unsupported tile width
    assert L.gcf_gemm_bf16(p, 72, p, 72, 128, 128, 64, C.c_void_p(d.data_ptr()), 128, 96, 2, None) == 1


PCONFIGS = [(256, 3), (256, 4), (128, 4), (128, 6), (64, 4), (32, 4)]


def _run_ex(L, a, b, tile_n, stages, persistent):
    import torch
    m, k = a.shape
    n = b.shape[0]
    d = torch.full((m, n), float("nan"), dtype=torch.float32, device="cuda")
    st = L.gcf_gemm_bf16_ex(C.c_void_p(a.data_ptr()), a.stride(0), C.c_void_p(b.data_ptr()), b.stride(0),
                            m, n, k, C.c_void_p(d.data_ptr()), d.stride(0), tile_n, stages, persistent, None)
    assert st == 0, L.gcf_strerror(st)
    return d


@pytest.mark.parametrize("tile_n,stages", PCONFIGS)
def test_persistent_gemm_matches_fp32_and_one_tile_per_cta(gpu_lib, tile_n, stages):
    """The persistent variant (one CTA per SM over all tiles, accumulator
    double-buffered in tensor memory) against the FP32 reference, on shapes
    with fewer tiles than SMs, with several tiles per CTA (both accumulator
    buffers reused) and ragged edges; it equals the one-tile-per-CTA kernel
    bit for bit (same MMAs, same accumulation order)."""
    import torch
    L = gpu_lib.load_library()
    g = torch.Generator(device="cuda").manual_seed(tile_n + stages)
    for (m, n, k) in [(256, 512, 512), (300, 200, 72), (2048, 4096, 512), (1100, 1000, 264)]:
        a = torch.randn((m, k), generator=g, device="cuda").to(torch.bfloat16)
        b = torch.randn((n, k), generator=g, device="cuda").to(torch.bfloat16)
        dp = _run_ex(L, a, b, tile_n, stages, 1)
        _check(a, b, dp)
        if (tile_n, stages) in CONFIGS:
            assert torch.equal(dp, _run(L, a, b, tile_n, stages))
