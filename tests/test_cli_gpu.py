"""GPU tests of the GCtfFind command line (bin/GCtfFind): a tilt-series
stack, a single micrograph, and a folder of micrographs (-Serial 1), each
checked against the library's own results on the same images."""
import os
import subprocess

import numpy as np
import pytest

import gctffind_b200 as G
from gctffind_b200 import synth

pytestmark = pytest.mark.gpu


def _img(w, h, px, df, az, seed, tilt=0.0):
    spec = synth.MicrographSpec(width=w, height=h, pixel_size=px, df_min=df[0], df_max=df[1],
                                azimuth_deg=az, dose=3.0, seed=seed, tilt_deg=tilt)
    return synth.make_micrograph(spec, device="cpu").numpy().astype(np.float32)


def _run(*args):
    if not os.path.exists(G.CLI_PATH):
        pytest.fail("bin/GCtfFind not built")
    r = subprocess.run([G.CLI_PATH, *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r


def _rows(path):
    out = []
    for line in open(path):
        if line.startswith("#"):
            continue
        f = line.split()
        out.append([int(f[0]), float(f[1])] + [float(x) for x in f[2:7]] + [f[7]])
    return out


def test_cli_tilt_series(gpu_lib, tmp_path):
    tilts = [-6.0, -3.0, 0.0, 3.0, 6.0]
    imgs = np.stack([_img(768, 768, 1.35, (16000.0, 16400.0), 25.0, 500 + k, tilt=t)
                     for k, t in enumerate(tilts)])
    stack = str(tmp_path / "ts.mrc")
    G.mrc_write(stack, imgs, 1.35)
    out_ctf, out_mrc = str(tmp_path / "ts_ctf.txt"), str(tmp_path / "ts_ctf.mrc")
    _run("-InMrc", stack, "-OutMrc", out_mrc, "-OutCtf", out_ctf, "-PixSize", "1.35",
         "-TileSize", "256", "-TiltRange", "-6", "6")
    rows = _rows(out_ctf)
    assert [r[0] for r in rows] == list(range(5))
    assert np.allclose([r[1] for r in rows], tilts)
    ctx = G.Context(0, 256, 0)
    so = G.series_order(tilts)
    lib = ctx.run_series(list(imgs), G.make_optics(pixel_size=1.35), so.order, is_tomo=True)
    for r, l in zip(rows, lib):
        assert r[2] == pytest.approx(round(l.df_min, 2), abs=0.006)
        assert r[3] == pytest.approx(round(l.df_max, 2), abs=0.006)
        assert r[6] == pytest.approx(round(l.score, 4), abs=1.1e-4)
    info = G.mrc_info(out_mrc)
    assert info["dims"] == (256, 256, 5)
    assert os.path.exists(str(tmp_path / "ts_ctf_Imod.txt"))


def test_cli_flushes_every_21_packages_and_resolution_column(gpu_lib, tmp_path):
    """A 23-tilt stack: the package hook of gcf_run_series reports every
    package once, in processing order, with the call's own results; the
    CLI's flush after the 21st package (CFindSeriesCtfs.cpp:97-101) and its
    final write leave the complete file; -CtfRes 1 adds the resolution
    column after the reference's columns."""
    tilts = [3.0 * (k - 11) for k in range(23)]
    imgs = np.stack([_img(512, 512, 1.35, (14000.0, 14300.0), 10.0, 600 + k, tilt=t)
                     for k, t in enumerate(tilts)])
    ctx = G.Context(0, 256, 0)
    so = G.series_order(tilts)
    seen = []
    lib = ctx.run_series(list(imgs), G.make_optics(pixel_size=1.35), so.order, is_tomo=True,
                         on_package=lambda done, image, r: seen.append((done, image, r.as_dict())))
    assert [d for d, _, _ in seen] == list(range(1, 24))
    assert [i for _, i, _ in seen] == list(so.order)
    for _, i, r in seen:
        assert r == lib[i].as_dict()
    # the hook is removed after the call
    again = ctx.run_series(list(imgs), G.make_optics(pixel_size=1.35), so.order, is_tomo=True)
    assert [r.as_dict() for r in again] == [r.as_dict() for r in lib]
    ctx.close()
    stack = str(tmp_path / "ts23.mrc")
    G.mrc_write(stack, imgs, 1.35)
    out_ctf = str(tmp_path / "ts23_ctf.txt")
    _run("-InMrc", stack, "-OutCtf", out_ctf, "-PixSize", "1.35", "-TileSize", "256",
         "-TiltRange", "-33", "33", "-CtfRes", "1")
    lines = open(out_ctf).read().splitlines()
    assert lines[0].endswith("fileName  ctfRes") and len(lines) == 24
    for line, l in zip(lines[1:], lib):
        f = line.split()
        assert len(f) == 9
        assert float(f[2]) == pytest.approx(round(l.df_min, 2), abs=0.006)
        assert float(f[8]) == pytest.approx(round(l.ctf_res, 2), abs=0.006)


def test_cli_single_micrograph(gpu_lib, tmp_path):
    img = _img(1024, 1024, 1.0, (22000.0, 22600.0), -30.0, 510)
    path = str(tmp_path / "mic.mrc")
    G.mrc_write(path, img[None], 1.0)
    out_ctf, out_mrc = str(tmp_path / "mic_ctf.txt"), str(tmp_path / "mic_ctf.mrc")
    _run("-InMrc", path, "-OutMrc", out_mrc, "-OutCtf", out_ctf, "-PixSize", "1.0", "-TileSize", "256")
    rows = _rows(out_ctf)
    assert len(rows) == 1 and rows[0][1] == 0.0
    ctx = G.Context(0, 256, 0)
    lib = ctx.run_series([img], G.make_optics(pixel_size=1.0), [0], is_tomo=False)[0]
    assert rows[0][2] == pytest.approx(round(lib.df_min, 2), abs=0.006)
    assert abs(0.5 * (rows[0][2] + rows[0][3]) - 22300.0) < 300.0
    assert G.mrc_info(out_mrc)["dims"] == (256, 256, 1)
    assert not os.path.exists(str(tmp_path / "mic_ctf_Imod.txt"))


def test_cli_serial_folder(gpu_lib, tmp_path):
    d = tmp_path / "mics"
    d.mkdir()
    sizes = [(640, 640), (640, 640), (768, 640)]
    for k, (w, h) in enumerate(sizes):
        G.mrc_write(str(d / f"grid_{k + 1:03d}.mrc"), _img(w, h, 1.35, (15000.0, 15400.0), 40.0,
                                                             520 + k)[None], 1.35)
    (d / "other_001.mrc").write_bytes(b"not an mrc")
    out_ctf = str(tmp_path / "serial.txt")
    out_mrc = str(tmp_path / "spec.mrc")
    _run("-InMrc", str(d / "grid_"), "-InSuffix", ".mrc", "-Serial", "1", "-OutMrc", out_mrc,
         "-OutCtf", out_ctf, "-PixSize", "1.35", "-TileSize", "256")
    rows = _rows(out_ctf)
    assert len(rows) == 3
    assert sorted(os.path.basename(r[7]) for r in rows) == [f"grid_{k:03d}.mrc" for k in (1, 2, 3)]
    for r in rows:
        assert abs(0.5 * (r[2] + r[3]) - 15200.0) < 300.0
    spectra = sorted(p for p in os.listdir(tmp_path) if p.startswith("spec") and p.endswith(".mrc"))
    assert len(spectra) == 3
