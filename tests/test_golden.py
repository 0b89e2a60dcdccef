"""CPU: the FP64 oracle pinned against golden outputs of the reference
itself (tests/golden, written by tests/golden/make_golden.py from the
reference's own CTF path built from the GCtfFind sources), plus the result
file writer against the reference's CSaveCtfResults output.

Tolerances
  rescaled image (sum, sum of squares)  : 1e-5 relative
  averaged spectrum, per pixel          : 1e-4 relative (+ 1e-5 x rms)
  background-removed, lowpassed spectrum: 5e-4 x rms away from the border
      (rows 0..8, tile-8..tile-1, columns >= tile/2 - 8).  The reference's
      B-factor lowpass reads one row past its buffer for the y = 0 row of the
      mirrored half (FindCTF/GCalcSpectrum.cu:53) and takes the x = tile/2
      column from the padding of an in-place C2R (FindCTF/CFindCtfBase.cpp:
      212-218); neither value is defined, and the blur spreads them a few
      pixels inward.  The CC band never reaches that border.
  full spectrum                         : 5e-3 x rms away from the same border
  search results                        : the same candidate, or a neighbour
      whose CC ties to 1e-5 (the reference sums CCs in float32 over ~10^4-10^5
      pixels, the oracle in FP64): df within 20 A (the smallest DfMean step),
      angle within 1 deg, extra phase within 1 deg (the largest phase step),
      CC within 1e-5
"""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, GOLD)

import make_golden as MG  # noqa: E402

META_PATH = os.path.join(GOLD, "reference_cases.json")
ARR_PATH = os.path.join(GOLD, "reference_cases.npz")

pytestmark = pytest.mark.skipif(not os.path.exists(META_PATH), reason="golden fixtures absent")


@pytest.fixture(scope="module")
def gold():
    return json.load(open(META_PATH)), np.load(ARR_PATH)


def _same_input(img, ck):
    a = img.astype(np.float64)
    if not np.allclose([a.sum(), (a * a).sum()], ck[:2], rtol=1e-9):
        pytest.skip("synthetic generator drifted from the golden inputs")
    assert np.array_equal(img.ravel()[:8], np.asarray(ck[2], np.float32))


def _border_mask(tile, k=8):
    """Half-spectrum pixels at least k + 1 rows from y = 0 and tile - 1 and
    k + 1 columns from x = tile / 2."""
    m = np.ones((tile, tile // 2 + 1), bool)
    m[: k + 1, :] = False
    m[tile - k:, :] = False
    m[:, tile // 2 - k:] = False
    return m


def _result_equal(r, ref):
    got = [r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score]
    assert abs(got[4] - ref[4]) <= 1e-5, (got, ref)
    assert abs(got[0] - ref[0]) <= 20.0 and abs(got[1] - ref[1]) <= 20.0, (got, ref)
    d = (got[2] - ref[2]) % 180.0
    assert min(d, 180.0 - d) <= 1.0, (got, ref)
    assert abs(got[3] - ref[3]) <= 1.0, (got, ref)


@pytest.mark.parametrize("name", list(MG.SINGLE_CASES))
def test_oracle_single_micrograph_matches_reference(oracle, gold, name):
    meta, arr = gold
    m = meta["cases"][name]
    ia, rk, refine = MG.SINGLE_CASES[name]
    img = MG.micrograph(**ia)
    _same_input(img, m["input_checksum"])
    px, tile = rk["pixel_size"], rk["tile"]
    nw, nh, npx, _ = oracle.rescale_dims(img.shape[1], img.shape[0], px)
    assert [nw, nh] == m["new_size"] and abs(npx - m["new_pixel_size"]) < 1e-6
    resc = oracle.rescale(img, px)
    r64 = resc.astype(np.float64)
    assert np.allclose([r64.sum(), (r64 * r64).sum()], m["rescaled_checksum"][:2], rtol=1e-5)
    p = oracle.params(pixel_size=px, tile_size=tile, log_spect=rk.get("log_spect", 0),
                      ext_phase_deg=rk.get("ext_phase_deg", 0.0),
                      ext_phase_range=rk.get("ext_phase_range", 0.0))
    r, raw, ctf, full = oracle.find_ctf_image(resc, npx, p, mode=0 if refine is None else 1,
                                              refine_in=refine, want_spectra=True)
    _result_equal(r, m["result"])
    if f"{name}/raw_half" not in arr:
        for a, key in ((raw, "raw_half_checksum"), (ctf, "ctf_half_checksum")):
            s = [a.sum(), (a * a).sum()]
            assert np.allclose(s[1], m[key][1], rtol=1e-3)
        return
    R = arr[f"{name}/raw_half"].astype(np.float64)
    rms = np.sqrt((R * R).mean())
    assert np.all(np.abs(raw - R) <= 1e-4 * np.abs(R) + 1e-5 * rms)
    C = arr[f"{name}/ctf_half"].astype(np.float64)
    mask = _border_mask(tile)
    assert np.abs(ctf - C)[mask].max() <= 5e-4 * np.sqrt((C * C).mean())
    F = arr[f"{name}/full"].astype(np.float64)
    fm = np.ones_like(F, bool)
    fm[:9, :] = fm[-8:, :] = False
    fm[:, :9] = fm[:, -8:] = False
    fm[:, tile // 2 - 8: tile // 2 + 9] = False
    assert np.abs(full - F)[fm].max() <= 5e-3 * np.sqrt((F * F).mean())


def test_oracle_series_matches_reference(oracle, gold):
    meta, _ = gold
    S = meta["series"]
    imgs, tilts = MG.series_inputs()
    for img, ck in zip(imgs, S["input_checksums"]):
        _same_input(img, ck)
    p = oracle.params(pixel_size=S["spec"]["px"], tile_size=S["spec"]["tile"])
    res = oracle.series(imgs, p, S["order"], True)
    for r, ref in zip(res, S["results"]):
        _result_equal(r, ref)


def test_oracle_phase_plate_set_matches_reference(oracle, gold):
    meta, _ = gold
    if "phase_set" not in meta:
        pytest.skip("no phase-plate case in the fixtures")
    P = meta["phase_set"]
    imgs = MG.phase_set_inputs()
    for img, ck in zip(imgs, P["input_checksums"]):
        _same_input(img, ck)
    sp = P["spec"]
    p = oracle.params(pixel_size=sp["px"], tile_size=sp["tile"], ext_phase_deg=sp["ext_phase"],
                      ext_phase_range=sp["ext_phase_range"])
    res = oracle.series(imgs, p, list(range(sp["n"])), False)
    for r, ref in zip(res, P["results"]):
        _result_equal(r, ref)


def test_ctf_file_writer_matches_reference_output(gold, tmp_path):
    """gcf_write_ctf_file (host code, no GPU) reproduces the reference's
    CSaveCtfResults files byte for byte from the same numbers."""
    import gctffind_b200 as G
    meta, _ = gold
    S = meta["series"]
    rs = []
    for v in S["results"]:
        r = G.Result()
        r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score = v
        rs.append(r)
    out = str(tmp_path / "reference_series.txt")
    G.write_ctf_file(out, rs, tilts=S["tilts"], names=["series.mrc"] * len(rs), is_tomo=True)
    assert open(out).read() == open(os.path.join(GOLD, "reference_series.txt")).read()
    assert (open(str(tmp_path / "reference_series_Imod.txt")).read()
            == open(os.path.join(GOLD, "reference_series_Imod.txt")).read())
