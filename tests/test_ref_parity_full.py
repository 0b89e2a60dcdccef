"""GPU parity at the benchmark's own sizes, against the reference's CTF path
built from its sources (oracle/_ref/libgcfref.so) and the FP64 oracle.

* The spectral-CC resolution (GSpectralCC2D, FindCTF/GSpectralCC2D.cu:12-173,
  reported by CFindDefocus2D::mCalcCtfRes, FindCTF/CFindDefocus2D.cpp:382-400)
  against the oracle's and the reference's.  The resolution is
  tile * pixel size / shell for an integer shell, so the test compares
  shells: equal, or the neighbouring shell where the shell CC lies within
  2e-3 of the 0.143 threshold (float against FP64 sums).
* The full 41-tilt series of 4096^2 micrographs at 1.35 A/px (the benchmark
  series, seed 1) through gcf_run_series against the reference's
  CFindSeriesCtfs::DoIt on the same images.
* A seeded draw of 32 micrographs with the uneven-batch distribution (sizes
  4096 x 4096, 5760 x 4092, 3838 x 3710; pixel size 0.8-1.5 A; defocus
  5000-40000 A; astigmatism 0-1000 A at an angle in 0-180 degrees; dose
  0.5-2 e/A^2) through one gcf_run_batch call against the reference once per
  micrograph (its single-file mode).  Draws outside the reference's search
  envelope -- mean defocus below the 1D search floor 3000 * px^2 A
  (FindCTF/CFindCtf1D.cpp:78-79) or an astigmatism ratio above the full
  search's 0.06 (FindCTF/CFindDefocus2D.cpp:117-118) -- are counted and left
  out of the comparison.  The same draw through the BF16 contraction and the
  learned search, and the plain search with the line-transform rescale, each
  against the reference.

Accuracy bar (the path's): defocus within one search step of the reference's
last mean-defocus line search, max(20 A, 0.105 * mean / 31); azimuth 1 degree
(mod 180) where the astigmatism exceeds 50 A; CC 1e-3.
"""
import numpy as np
import pytest

from gctffind_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle import refimpl
    if not refimpl.available():
        pytest.skip("reference build oracle/_ref/libgcfref.so not present")
    return refimpl


def _step(df_mean):
    return max(20.0, 0.105 * df_mean / 31.0)


def _ang(a, b):
    d = (a - b) % 180.0
    return min(d, 180.0 - d)


def _close(g, r):
    """g, r: (df_min, df_max, azimuth, ext_phase, score)."""
    tol = _step(0.5 * (r[0] + r[1]))
    assert abs(g[0] - r[0]) <= tol and abs(g[1] - r[1]) <= tol, (g, r, tol)
    if abs(r[1] - r[0]) > 50.0:
        assert _ang(g[2], r[2]) <= 1.0, (g, r)
    assert abs(g[4] - r[4]) <= 1e-3, (g, r)


def _shell(res_a, tile, px):
    return int(round(tile * px / res_a)) if res_a > 0 else 0


def test_ctf_res_matches_oracle_and_reference(gpu_lib, ref, oracle):
    G = gpu_lib
    cases = [(2048, 1.35, (16800.0, 17300.0), 35.0, 801, 1.0),
             (1536, 1.5, (24000.0, 24400.0), -60.0, 802, 3.0),
             (2048, 1.2, (9000.0, 9200.0), 10.0, 803, 0.7)]
    for w, px, df, az, seed, dose in cases:
        spec = synth.MicrographSpec(width=w, height=w, pixel_size=px, df_min=df[0], df_max=df[1],
                                    azimuth_deg=az, dose=dose, seed=seed)
        img = synth.make_micrograph(spec, device="cpu").numpy().astype(np.float32)
        ctx = G.Context(0, 512, 0)
        ctx.setup(G.make_optics(pixel_size=px), w, w)
        ctx.gen_half_spectrum(img)
        r = ctx.do2d()
        ctx.close()
        o = oracle.find_ctf_image(img, px, oracle.params(pixel_size=px, tile_size=512))
        R = ref.single(img, px, tile=512)
        mine, orc, rr = (_shell(x, 512, px) for x in (r.ctf_res, o.ctf_res, R["ctf_res"]))
        assert mine > 0 and rr > 0, (r, o.as_dict(), R["ctf_res"])
        assert abs(mine - orc) <= 1 and abs(mine - rr) <= 1, (mine, orc, rr)
        assert mine == rr or abs(r.ctf_res - R["ctf_res"]) / R["ctf_res"] <= 0.05, (mine, rr)


def test_full_benchmark_series_matches_reference(gpu_lib, ref):
    """41 x 4096^2 at 1.35 A/px, the benchmark series (seed 1)."""
    import torch
    G = gpu_lib
    specs = synth.tilt_series_specs(n_tilts=41, step_deg=3.0, size=4096, pixel_size=1.35, dose=3.0,
                                    df0=30000.0, seed=1)
    imgs = [synth.make_micrograph(s, device="cuda").cpu().numpy() for s in specs]
    torch.cuda.empty_cache()
    tilts = synth.tilt_angles(41, 3.0)
    order = G.series_order(tilts).order
    R, _, _ = ref.run_series(imgs, 1.35, order, tilts=tilts, tile=512)
    ctx = G.Context(0, 512, 0)
    mine = ctx.run_series(imgs, G.make_optics(pixel_size=1.35), order, is_tomo=True)
    ctx.close()
    ddf = []
    for k in range(41):
        r = mine[k]
        _close([r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score], [float(x) for x in R[k]])
        ddf.append(abs(r.df_min - float(R[k][0])) + abs(r.df_max - float(R[k][1])))
    # observed on B200: identical to float rounding
    assert float(np.median(ddf)) <= 1.0


def test_uneven_batch_draw_matches_reference(gpu_lib, ref):
    import torch
    G = gpu_lib
    specs = synth.uneven_batch_specs(32, 7)
    imgs = [synth.make_micrograph(s, device="cuda").cpu().numpy() for s in specs]
    torch.cuda.empty_cache()
    pxs = [s.pixel_size for s in specs]
    op = G.make_optics()
    ctx = G.Context(0, 512, 0)
    mine = ctx.run_batch(imgs, pxs, op)
    bf16 = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_BF16)
    G.load_learned(ctx)
    learned = ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_LEARNED)
    ctx.close()
    lines = G.Context(0, 512, 0)
    lines.set_rescale_impl(G.GCF_RESCALE_LINES)
    mine_lines = lines.run_batch(imgs, pxs, op)
    lines.close()
    checked = excluded = 0
    within = {"bf16": [], "learned": [], "lines": []}
    for k, (img, s, r) in enumerate(zip(imgs, specs, mine)):
        if not synth.inside_reference_envelope(s):
            excluded += 1
            continue
        R, _, _ = ref.run_series([img], s.pixel_size, [0], is_tomo=False, tile=512)
        ref_row = [float(x) for x in R[0]]
        _close([r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score], ref_row)
        step = max(20.0, 0.105 * 0.5 * (ref_row[0] + ref_row[1]) / 31.0)
        for name, res in (("bf16", bf16), ("learned", learned), ("lines", mine_lines)):
            f = res[k]
            within[name].append(abs(f.df_min - ref_row[0]) <= step and abs(f.df_max - ref_row[1]) <= step)
        checked += 1
    print(f"uneven batch draw: {checked} compared, {excluded} outside the reference envelope; "
          f"within one step of the reference: " + ", ".join(f"{k} {np.mean(v):.3f}" for k, v in within.items()))
    assert checked >= 24
    # the faster methods against the reference itself: the headline path's
    # accuracy bar (>= 99 % within one step on the 256-micrograph batch) at
    # this sample size allows one miss; the line-transform rescale changes
    # only rounding, so the plain search through it lands with the reference
    assert sum(not x for x in within["bf16"]) <= 1 and sum(not x for x in within["learned"]) <= 1, within
    assert all(within["lines"]), within["lines"]
