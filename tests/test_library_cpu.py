"""CPU tests of the library surface: the C ABI loads and exports every
declared entry point, host-only entry points (MRC I/O, result files, rescale
sizes) behave like the reference, and the command line parses like CInput.
No kernel is launched here."""
import os
import re
import struct
import subprocess

import numpy as np
import pytest

import gctffind_b200 as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    src = open(os.path.join(ROOT, "include", "gctf_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gcf_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = G.load_library()
    syms = _header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(G.EXPORTS) == syms
    out = subprocess.run(["nm", "-D", "--defined-only", G.LIB_PATH], capture_output=True, text=True).stdout
    for s in syms:
        assert re.search(r"\bT %s\b" % s, out), s


def test_python_constants_match_the_header_enums():
    """Every GCF_SPECT_*, GCF_RESCALE_* and GCF_SEARCH_* value the binding
    exports equals the header's."""
    src = open(os.path.join(ROOT, "include", "gctf_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    vals = {k: int(v) for k, v in re.findall(r"\b(GCF_(?:SPECT|RESCALE|SEARCH)_[A-Z0-9]+)\s*=\s*(\d+)", src)}
    assert {"GCF_RESCALE_CUFFT", "GCF_RESCALE_LINES", "GCF_RESCALE_GEMM"} <= set(vals)
    for k, v in vals.items():
        assert getattr(G, k) == v, k


def test_strerror_codes():
    L = G.load_library()
    assert L.gcf_strerror(0) == b"ok"
    assert L.gcf_strerror(5) == b"image smaller than one tile"


def test_entry_points_reject_a_missing_context():
    """Entry points that take a context return GCF_ERR_INVALID_ARG (1) for a
    NULL one, before touching any device."""
    import ctypes as C
    L = G.load_library()
    f = (C.c_float * 8)()
    ll = (C.c_longlong * 8)()
    assert L.gcf_set_rescale_impl(None, 0) == 1
    assert L.gcf_set_fused_shape(None, 8) == 1
    assert L.gcf_set_graphs(None, 1) == 1
    assert L.gcf_get_fast_times(None, f) == 1
    assert L.gcf_get_fast_counts(None, ll) == 1
    assert L.gcf_get_stage_times(None, f) == 1
    assert L.gcf_nn_inputs(None, f, f, 1, f, f) == 1


def test_rescale_dims_like_crescaleimage():
    # CRescaleImage::Setup (FindCTF/CRescaleImage.cpp:47-66), float32 arithmetic
    assert G.rescale_dims(4096, 4096, 1.0)[:2] == (3412, 3412)
    assert G.rescale_dims(5760, 4092, 0.8)[:2] == (3840, 2728)
    assert G.rescale_dims(3838, 3710, 0.8)[:2] == (2558, 2472)
    assert G.rescale_dims(4096, 4096, 1.35) == (4096, 4096, pytest.approx(1.35))
    assert G.rescale_dims(4097, 4095, 1.5)[:2] == (4096, 4094)


def _write_mrc(path, arr, mode, ext_tilts=None, swap=False):
    nz, ny, nx = arr.shape
    hdr = bytearray(1024)
    e = ">" if swap else "<"
    struct.pack_into(e + "4i", hdr, 0, nx, ny, nz, mode)
    struct.pack_into(e + "3i", hdr, 28, nx, ny, nz)
    struct.pack_into(e + "3f", hdr, 40, nx * 1.5, ny * 1.5, nz * 1.5)
    ext = b""
    if ext_tilts is not None:
        nint, nreal = 2, 4
        struct.pack_into(e + "2h", hdr, 128, nint, nreal)
        rec = []
        for t in ext_tilts:
            rec.append(struct.pack(e + "2i4f", 7, 8, t, 1.0, 2.0, 3.0))
        ext = b"".join(rec)
    struct.pack_into(e + "i", hdr, 92, len(ext))
    dt = {0: "u1", 1: "i2", 2: "f4", 6: "u2"}[mode]
    with open(path, "wb") as f:
        f.write(bytes(hdr))
        f.write(ext)
        f.write(arr.astype((">" if swap else "<") + dt).tobytes())


@pytest.mark.parametrize("mode", [0, 1, 2, 6])
def test_mrc_modes_read_as_float(tmp_path, mode):
    # CLoadImages::mToFloat (MrcUtil/CLoadImages.cpp:146-181)
    rng = np.random.default_rng(mode)
    hi = {0: 255, 1: 3000, 2: 1000, 6: 60000}[mode]
    lo = -3000 if mode == 1 else 0
    a = rng.integers(lo, hi, size=(2, 5, 7))
    p = str(tmp_path / f"m{mode}.mrc")
    _write_mrc(p, a, mode)
    info = G.mrc_info(p)
    assert info["dims"] == (7, 5, 2) and info["mode"] == mode
    assert info["pixel_size"] == pytest.approx(1.5)
    for z in range(2):
        assert np.array_equal(G.mrc_read(p, z), a[z].astype(np.float32))


def test_mrc_byte_swapped_and_ext_header_tilts(tmp_path):
    a = np.arange(3 * 4 * 6, dtype=np.float32).reshape(3, 4, 6)
    p = str(tmp_path / "sw.mrc")
    tilts = [-3.0, 0.0, 3.0]
    _write_mrc(p, a, 2, ext_tilts=tilts, swap=True)
    assert np.array_equal(G.mrc_read(p, 2), a[2])
    assert np.allclose(G.mrc_read_tilts(p, 3), tilts)
    assert G.mrc_info(p)["ext_floats"] == 4


def test_mrc_write_round_trip_and_errors(tmp_path):
    a = np.random.default_rng(0).standard_normal((3, 16, 8)).astype(np.float32)
    p = str(tmp_path / "w.mrc")
    G.mrc_write(p, a, 1.2)
    info = G.mrc_info(p)
    assert info["dims"] == (8, 16, 3) and info["mode"] == 2
    assert info["pixel_size"] == pytest.approx(1.2)
    for z in range(3):
        assert np.array_equal(G.mrc_read(p, z), a[z])
    with pytest.raises(G.GcfError):
        G.mrc_read(str(tmp_path / "missing.mrc"))
    bad = tmp_path / "trunc.mrc"
    bad.write_bytes(open(p, "rb").read()[:1500])
    with pytest.raises(G.GcfError):
        G.mrc_read(str(bad), 2)


def _res(*v):
    r = G.Result()
    for k, x in zip(["df_min", "df_max", "azimuth", "ext_phase", "score"], v):
        setattr(r, k, x)
    return r


def test_ctf_file_format_matches_csavectfresults(tmp_path):
    # CSaveCtfResults::SaveCTF / SaveImod (CSaveCtfResults.cpp:34-117)
    rs = [_res(29700.12, 30301.5, -38.89, 0.0, 0.84431), _res(29000.0, 29500.25, 12.5, 0.0, 0.5)]
    p = str(tmp_path / "series.txt")
    G.write_ctf_file(p, rs, tilts=[0.0, -3.0], names=["ts.mrc", "ts.mrc"], is_tomo=True)
    lines = open(p).read().splitlines()
    assert lines[0] == "# Idx   tilt     dfMin      dfMax   azimuth extPhase  score    fileName"
    assert lines[1] == "   0    0.00   29700.12   30301.50  -38.89    0.00   0.8443  ts.mrc"
    assert lines[2] == "   1   -3.00   29000.00   29500.25   12.50    0.00   0.5000  ts.mrc"
    imod = open(str(tmp_path / "series_Imod.txt")).read().splitlines()
    assert imod[0] == "1  0  0.0  0.0  0.0  3"
    assert imod[1] == "   1     1     0.00     0.00   2970.01   3030.15   -38.89"
    # extra phase -> 5-column header and an extra field
    rs[0].ext_phase = 12.0
    G.write_ctf_file(str(tmp_path / "ph"), rs, tilts=[0.0, -3.0], names=["a", "b"], is_tomo=True)
    imod = open(str(tmp_path / "ph_Imod.txt")).read().splitlines()
    assert imod[0] == "5  0  0.0  0.0  0.0  3"
    assert imod[1].endswith("   12.00")
    # single micrograph: no Imod file
    G.write_ctf_file(str(tmp_path / "one.txt"), rs[:1], names=["m.mrc"], is_tomo=False)
    assert not os.path.exists(str(tmp_path / "one_Imod.txt"))


def test_ctf_file_resolution_column_is_opt_in(tmp_path):
    """gcf_write_ctf_file_ex: flags 0 writes the reference's file byte for
    byte; GCF_CTF_COLUMN_RES appends the spectral-CC resolution after the
    file name, so the reference's columns keep their positions."""
    rs = [_res(29700.12, 30301.5, -38.89, 0.0, 0.84431), _res(29000.0, 29500.25, 12.5, 0.0, 0.5)]
    rs[0].ctf_res, rs[1].ctf_res = 4.21, 11.5
    a, b = str(tmp_path / "a.txt"), str(tmp_path / "b.txt")
    G.write_ctf_file(a, rs, tilts=[0.0, -3.0], names=["ts.mrc", "ts.mrc"], is_tomo=True)
    G.write_ctf_file(b, rs, tilts=[0.0, -3.0], names=["ts.mrc", "ts.mrc"], is_tomo=True, ctf_res=True)
    la, lb = open(a).read().splitlines(), open(b).read().splitlines()
    assert lb[0] == la[0] + "  ctfRes"
    assert lb[1] == la[1] + "     4.21"
    assert lb[2] == la[2] + "    11.50"
    # the Imod file does not change
    assert open(str(tmp_path / "a_Imod.txt")).read() == open(str(tmp_path / "b_Imod.txt")).read()
    L = G.load_library()
    assert L.gcf_write_ctf_file_ex(b.encode(), (G.Result * 1)(rs[0]), None, None, 1, 0, 2) == 1


def test_series_order_zero_tilt_first():
    # CInputFolder::FindZeroTilt + CLoadImages::mReadTomo
    so = G.series_order([-6, -3, 0.0, 3, 6])
    assert so.zero_tilt == 2 and so.order == [2, 0, 1, 3, 4]
    so = G.series_order([0.0, 0.0, 0.0, 0.0])          # equal first two -> n / 2
    assert so.zero_tilt == 2
    so = G.series_order([-1.0, 0.5, -0.5, 2.0])       # first strict minimum of |tilt|
    assert so.zero_tilt == 1


def _cli(*args):
    if not os.path.exists(G.CLI_PATH):
        pytest.skip("CLI not built")
    return subprocess.run([G.CLI_PATH, *args], capture_output=True, text=True, timeout=60)


def test_cli_help_version_and_usage():
    r = _cli()
    assert r.returncode == 0 and "--help" in r.stdout
    r = _cli("--help")
    assert r.returncode == 0
    for tag in ["-InMrc", "-OutMrc", "-OutCtf", "-AngFile", "-TiltRange", "-kV", "-Cs",
                "-AmpContrast", "-PixSize", "-ExtPhase", "-TileSize", "-LogSpect", "-InSuffix",
                "-Serial", "-Gpu"]:
        assert tag in r.stdout, tag
    assert _cli("--version").returncode == 0


def test_cli_parses_like_cinput():
    # CParseArgs (Util/CParseArgs.cpp:25-94): case-insensitive tags, numeric runs,
    # -TiltRange clamped to +-70.1, negative -ExtPhase range -> 0
    r = _cli("-inmrc", "in.mrc", "-OUTCTF", "out.txt", "-PixSize", "1.35", "7", "-ExtPhase", "10",
             "-5", "-TiltRange", "-80", "75", "-TileSize", "256", "-Gpu", "9999")
    out = r.stdout
    assert re.search(r"-InMrc\s+in.mrc", out) and re.search(r"-OutCtf\s+out.txt", out)
    assert re.search(r"-PixSize\s+1.350000", out)
    assert re.search(r"-ExtPhase\s+10.000000\s+0.000000", out)
    assert re.search(r"-TiltRange\s+-70.10\s+70.10", out)
    assert re.search(r"-TileSize\s+256", out)
    assert r.returncode == 1            # GPU 9999 does not exist: error, no crash


def test_cli_rejects_same_input_and_output():
    r = _cli("-InMrc", "a.mrc", "-OutCtf", "A.MRC")
    assert r.returncode == 1 and "same name" in r.stderr
