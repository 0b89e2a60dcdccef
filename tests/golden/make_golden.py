"""Generate the golden fixtures of tests/golden from the reference's own CTF
path (oracle/_ref/libgcfref.so, built from the GCtfFind sources by
oracle/ref/Makefile).  The reference is CUDA code, so this script needs a
GPU:

    python tests/golden/make_golden.py --out tests/golden

Inputs are seeded synthetic micrographs from gctffind_b200.synth, made on
the CPU; each case stores checksums of its input so a test can tell when
the generator drifted.  Outputs: reference_cases.npz (arrays) and
reference_cases.json (scalars), plus the reference's CSaveCtfResults files
for the tilt-series case (reference_series.txt, reference_series_Imod.txt).
Arrays are stored for the tile-128 cases only; larger cases keep checksums.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gctffind_b200 import synth  # noqa: E402


def micrograph(w, h, px, df, az, seed, dose=3.0, tilt=0.0, phase_deg=0.0):
    spec = synth.MicrographSpec(width=w, height=h, pixel_size=px, df_min=df[0], df_max=df[1],
                                azimuth_deg=az, dose=dose, seed=seed, tilt_deg=tilt,
                                ext_phase_deg=phase_deg)
    return synth.make_micrograph(spec, device="cpu").numpy().astype(np.float32)


def checksum(a):
    a64 = a.astype(np.float64)
    return [float(a64.sum()), float((a64 * a64).sum()), [float(x) for x in a.ravel()[:8]]]


# name: (image args, reference kwargs, refine or None)
SINGLE_CASES = {
    "px100_t128": (dict(w=512, h=512, px=1.0, df=(12000.0, 12400.0), az=30.0, seed=101),
                   dict(pixel_size=1.0, tile=128), None),
    "px135_t128_phase": (dict(w=512, h=448, px=1.35, df=(15000.0, 15600.0), az=-40.0, seed=102,
                              phase_deg=40.0),
                         dict(pixel_size=1.35, tile=128, ext_phase_deg=30.0,
                              ext_phase_range=60.0), None),
    "px150_t128_log": (dict(w=480, h=512, px=1.5, df=(20000.0, 20500.0), az=75.0, seed=103),
                       dict(pixel_size=1.5, tile=128, log_spect=1), None),
    "px135_t128_refine": (dict(w=512, h=512, px=1.35, df=(18000.0, 18400.0), az=10.0, seed=104),
                          dict(pixel_size=1.35, tile=128),
                          [18300.0, 9000.0, 0.011, 0.04, 12.0, 30.0, 0.0, 0.0]),
    "px135_t512": (dict(w=1024, h=1024, px=1.35, df=(25000.0, 25800.0), az=-15.0, seed=105),
                   dict(pixel_size=1.35, tile=512), None),
}

SERIES = dict(n=5, step=3.0, w=512, h=512, px=1.35, df0=16000.0, tile=128, seed=200)
# micrographs (not a tilt series) with a phase plate: refine windows of a
# non-tomo run, extra-phase search
PHASE_SET = dict(n=3, w=512, h=512, px=1.35, df=(12000.0, 12500.0), az=-20.0, phase=35.0,
                 ext_phase=30.0, ext_phase_range=60.0, tile=128, seed=210)


def series_inputs():
    tilts = [SERIES["step"] * (k - SERIES["n"] // 2) for k in range(SERIES["n"])]
    imgs = [micrograph(SERIES["w"], SERIES["h"], SERIES["px"], (SERIES["df0"] - 150.0, SERIES["df0"] + 150.0),
                       25.0, SERIES["seed"] + k, tilt=t) for k, t in enumerate(tilts)]
    return imgs, tilts


def phase_set_inputs():
    P = PHASE_SET
    return [micrograph(P["w"], P["h"], P["px"], P["df"], P["az"], P["seed"] + k, phase_deg=P["phase"])
            for k in range(P["n"])]


def zero_first_order(tilts):
    """CInputFolder::FindZeroTilt + CLoadImages::mReadTomo order."""
    n = len(tilts)
    z = n // 2 if n > 1 and tilts[0] == tilts[1] else int(np.argmin(np.abs(np.asarray(tilts))))
    return [z] + [i for i in range(n) if i != z]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    args = ap.parse_args()
    from oracle import refimpl
    if not refimpl.available():
        raise SystemExit("oracle/_ref/libgcfref.so is not built")
    os.makedirs(args.out, exist_ok=True)
    arrays, meta = {}, {"cases": {}, "series": {}}
    for name, (ia, rk, refine) in SINGLE_CASES.items():
        img = micrograph(**ia)
        out = refimpl.single(img, refine=refine, **rk)
        m = {"image": ia, "reference_args": rk, "refine": refine, "input_checksum": checksum(img),
             "new_size": list(out["new_size"]), "new_pixel_size": out["new_pixel_size"],
             "result": [float(x) for x in out["result"]],
             "rescaled_checksum": checksum(out["rescaled"])}
        if rk["tile"] <= 128:
            arrays[f"{name}/raw_half"] = out["raw_half"]
            arrays[f"{name}/ctf_half"] = out["ctf_half"]
            arrays[f"{name}/full"] = out["full"]
        else:
            m["raw_half_checksum"] = checksum(out["raw_half"])
            m["ctf_half_checksum"] = checksum(out["ctf_half"])
        meta["cases"][name] = m
        print(name, m["result"], flush=True)
    imgs, tilts = series_inputs()
    order = zero_first_order(tilts)
    ctf_path = os.path.join(args.out, "reference_series.txt")
    res, full, _ = refimpl.run_series(imgs, SERIES["px"], order, tilts=tilts, is_tomo=True,
                                      tile=SERIES["tile"], names=["series.mrc"] * len(imgs),
                                      full_spectra=True, out_ctf=ctf_path)
    meta["series"] = {"spec": SERIES, "tilts": tilts, "order": order,
                      "input_checksums": [checksum(a) for a in imgs],
                      "results": res.tolist(),
                      "full_checksums": [checksum(f) for f in full]}
    print("series", res.tolist(), flush=True)
    P = PHASE_SET
    pimgs = phase_set_inputs()
    pres, _, _ = refimpl.run_series(pimgs, P["px"], list(range(P["n"])), is_tomo=False,
                                    ext_phase_deg=P["ext_phase"], ext_phase_range=P["ext_phase_range"],
                                    tile=P["tile"])
    meta["phase_set"] = {"spec": P, "input_checksums": [checksum(a) for a in pimgs],
                         "results": pres.tolist()}
    print("phase_set", pres.tolist(), flush=True)
    np.savez_compressed(os.path.join(args.out, "reference_cases.npz"), **arrays)
    with open(os.path.join(args.out, "reference_cases.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
