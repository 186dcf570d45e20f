"""The TOML-driven drivers (recon_lamino, recon_tomo, forward_scalar) and their file formats.

CPU tests run the drivers with --dry-run, which parses the config, loads and
prepares the inputs exactly as a reconstruction would and prints a summary,
and check what they read against the reference's conventions
(include/config.h): degrees to radians, the negated gamma, odd recon_dims,
shift broadcast and files, alignment overrides, error cases.  TIFF and .npy
round trips go through lc_convert against a TIFF writer and reader written
here in Python.  The GPU tests reconstruct through the drivers and compare
with the Python API on the same data."""
import json
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "laminocam_b200", "bin")


@pytest.fixture(scope="module")
def bins():
    from laminocam_b200 import build
    build.build()
    return {k: os.path.join(BIN, k) for k in ("recon_lamino", "recon_tomo", "forward_scalar", "lc_convert")}


def write_tiff(path, vol, big_endian=False, rows_per_strip=None, dtype=np.float32):
    """Minimal multi-page TIFF writer (test side): uncompressed, one sample."""
    e = ">" if big_endian else "<"
    vol = np.asarray(vol, dtype=dtype)
    n, h, w = vol.shape
    rps = rows_per_strip or h
    bits = vol.dtype.itemsize * 8
    fmt = 3 if vol.dtype.kind == "f" else 1
    out = bytearray(b"MM" if big_endian else b"II")
    out += struct.pack(e + "HI", 42, 8)
    for i in range(n):
        page = vol[i].astype(vol.dtype.newbyteorder(e)).tobytes()
        nstrips = (h + rps - 1) // rps
        strip_bytes = [min(rps, h - s * rps) * w * vol.dtype.itemsize for s in range(nstrips)]
        ifd_at = len(out)
        nent = 10
        arrays_at = ifd_at + 2 + 12 * nent + 4
        offs_at = arrays_at
        cnts_at = arrays_at + 4 * nstrips
        data_at = cnts_at + 4 * nstrips
        next_at = data_at + len(page) if i + 1 < n else 0
        ent = [(256, 4, 1, w), (257, 4, 1, h), (258, 3, 1, bits), (259, 3, 1, 1), (262, 3, 1, 1),
               (273, 4, nstrips, data_at if nstrips == 1 else offs_at), (277, 3, 1, 1),
               (278, 4, 1, rps), (279, 4, nstrips, strip_bytes[0] if nstrips == 1 else cnts_at),
               (339, 3, 1, fmt)]
        out += struct.pack(e + "H", nent)
        for tag, typ, cnt, val in ent:
            if typ == 3 and cnt == 1:
                out += struct.pack(e + "HHIHH", tag, typ, cnt, val, 0)
            else:
                out += struct.pack(e + "HHII", tag, typ, cnt, val)
        out += struct.pack(e + "I", next_at)
        starts = [data_at + sum(strip_bytes[:s]) for s in range(nstrips)]
        out += struct.pack(e + "%dI" % nstrips, *starts)
        out += struct.pack(e + "%dI" % nstrips, *strip_bytes)
        out += page
    with open(path, "wb") as f:
        f.write(bytes(out))


def read_tiff(path):
    """Minimal reader for the drivers' own output: little-endian float32 pages."""
    b = open(path, "rb").read()
    assert b[:2] == b"II" and struct.unpack("<H", b[2:4])[0] == 42
    pages, at = [], struct.unpack("<I", b[4:8])[0]
    while at:
        n = struct.unpack("<H", b[at:at + 2])[0]
        tags = {}
        for k in range(n):
            tag, typ, cnt, val = struct.unpack("<HHII", b[at + 2 + 12 * k: at + 14 + 12 * k])
            tags[tag] = val & 0xFFFF if typ == 3 else val
        w, h = tags[256], tags[257]
        assert tags[258] == 32 and tags[339] == 3 and tags[259] == 1
        pages.append(np.frombuffer(b, "<f4", w * h, tags[273]).reshape(h, w))
        at = struct.unpack("<I", b[at + 2 + 12 * n: at + 6 + 12 * n])[0]
    return np.stack(pages)


def dry(exe, cfg):
    r = subprocess.run([exe, "--dry-run", cfg], capture_output=True, text=True)
    return r.returncode, (json.loads(r.stdout) if r.returncode == 0 else None), r.stderr


def lamino_case(tmp_path, nproj=12, rows=18, cols=20, extra_input="", params_extra="",
                regularizer=True):
    rng = np.random.default_rng(1)
    projs = rng.random((nproj, rows, cols)).astype(np.float32)
    projs[0, 0, 0] = np.nan
    write_tiff(tmp_path / "projs.tiff", projs)
    ang = np.arange(nproj) * 360.0 / nproj
    np.savetxt(tmp_path / "angles.txt", ang)
    reg = ("[recon_params.regularizer]\nmethod = \"split_bregman\"\n"
           "[recon_params.regularizer.split_bregman]\nlambda = 0.25 # TV weight\nmu = 8\n"
           "inner_iters = 2\n") if regularizer else ""
    cfg = f"""# test config
[[input]]
filename = "projs.tiff"
angles = 'angles.txt'
angle_units = "deg"
gamma = 30
{extra_input}

[output]
filename = "out/recon.tiff"
formats = ["tiff", "tiff"]

[recon_params]
max_iters = 7
tol = 1e-4
recon_dims = [6, 16, 17]
{params_extra}
{reg}"""
    (tmp_path / "cfg.toml").write_text(cfg)
    return projs, ang


def test_lamino_config_parsing(bins, tmp_path):
    projs, ang = lamino_case(tmp_path)
    rc, d, err = dry(bins["recon_lamino"], str(tmp_path / "cfg.toml"))
    assert rc == 0, err
    trimmed = np.nan_to_num(projs[:, :17, :19], nan=0.0)  # even sizes lose their last row/column
    assert d["projections"] == [12, 17, 19]
    assert abs(d["sum"] - trimmed.astype(np.float64).sum()) < 1e-3
    assert abs(d["theta_last"] - np.deg2rad(ang[-1])) < 1e-12
    assert abs(d["gamma"] + np.deg2rad(30.0)) < 1e-12 and d["beta"] == 0
    assert d["recon_dims"] == [5, 15, 17] and d["max_iters"] == 7
    assert d["method"] == 1 and abs(d["lambda"] - 0.25) < 1e-7 and d["mu"] == 8 and d["inner_iters"] == 2
    assert abs(d["tol"] - 1e-4) < 1e-10 and abs(d["xtol"] - 1e-5) < 1e-10
    assert d["any_shift"] is False and d["output"] == "out/recon.tiff" and d["tiff"]


def test_lamino_shifts_and_alignment(bins, tmp_path):
    lamino_case(tmp_path, extra_input='cor-offset = [1.5, -2]')
    rc, d, err = dry(bins["recon_lamino"], str(tmp_path / "cfg.toml"))
    assert rc == 0, err
    assert d["shift0"] == [1.5, -2.0] and d["any_shift"] is True
    np.savetxt(tmp_path / "shifts.txt", np.column_stack([np.arange(12) * 0.5, -np.arange(12.0)]))
    lamino_case(tmp_path, extra_input='shifts = "shifts.txt"\ncor-offset = [9, 9]')
    rc, d, err = dry(bins["recon_lamino"], str(tmp_path / "cfg.toml"))
    assert rc == 0, err
    assert d["shift0"] == [0.0, 0.0] and d["any_shift"] is True
    al = ("gamma_deg = 20.0\nbeta_deg = 1.0\ncorrected_angles_deg = [" +
          ", ".join(str(1.0 + 30 * k) for k in range(12)) + "]\nshifts_px = [" +
          ", ".join("[%d, 0.25]" % k for k in range(12)) + ",\n]\n")
    (tmp_path / "align.toml").write_text(al)
    lamino_case(tmp_path, extra_input='alignment = "align.toml"')
    rc, d, err = dry(bins["recon_lamino"], str(tmp_path / "cfg.toml"))
    assert rc == 0, err
    assert abs(d["gamma"] + np.deg2rad(20.0)) < 1e-12 and abs(d["beta"] - np.deg2rad(1.0)) < 1e-12
    assert abs(d["theta0"] - np.deg2rad(1.0)) < 1e-12 and d["shift0"] == [0.0, 0.25]


def test_lamino_unconstrained_and_warnings(bins, tmp_path):
    lamino_case(tmp_path, regularizer=False, params_extra="num_gpus = 2\nbogus = 1")
    rc, d, err = dry(bins["recon_lamino"], str(tmp_path / "cfg.toml"))
    assert rc == 0, err
    assert d["method"] == 0
    assert "unknown key 'bogus'" in err
    assert "recon_dims[0] / recon_dims[2]" in err  # 5/17 > 0.15: the thickness warning


@pytest.mark.parametrize("mutate,msg", [
    (lambda c: c.replace('[output]', '[outputs]'), "Missing [output]"),
    (lambda c: c.replace("recon_dims = [6, 16, 17]", "recon_dims = [6, 16]"), "recon_dims"),
    (lambda c: c.replace("recon_dims = [6, 16, 17]", "recon_dims = [0, 16, 17]"), "positive integer"),
    (lambda c: c.replace('angles = \'angles.txt\'', ''), "'angles' is required"),
    (lambda c: c.replace('"projs.tiff"', '"missing.tiff"'), "does not exist"),
    (lambda c: c.replace('"projs.tiff"', '"projs.h5"'), "HDF5"),
    (lambda c: c.replace('method = "split_bregman"', 'method = "tv"'), "must be 'split_bregman'"),
    (lambda c: c.replace('formats = ["tiff", "tiff"]', 'formats = ["png"]'), "invalid format"),
    (lambda c: c.replace('angle_units = "deg"', 'angle_units = "grad"'), "angle_units"),
    (lambda c: c.replace("max_iters = 7", "max_iters = 7 7"), "after a value"),
    (lambda c: c.replace("max_iters = 7", "max_iters = 07"), "leading zero"),
    (lambda c: c.replace("tol = 1e-4", "tol = 1e-4\ntol = 2"), "duplicate key"),
])
def test_lamino_config_errors(bins, tmp_path, mutate, msg):
    lamino_case(tmp_path)
    p = tmp_path / "cfg.toml"
    if "projs.h5" in mutate(p.read_text()):
        (tmp_path / "projs.h5").write_bytes(b"\x89HDF\r\n")
    p.write_text(mutate(p.read_text()))
    rc, d, err = dry(bins["recon_lamino"], str(p))
    assert rc == 2 and msg in err, err


def test_lamino_angle_count_mismatch(bins, tmp_path):
    lamino_case(tmp_path)
    np.savetxt(tmp_path / "angles.txt", np.arange(11.0))
    rc, _, err = dry(bins["recon_lamino"], str(tmp_path / "cfg.toml"))
    assert rc == 2 and "has 12 pages" in err and "11 entries" in err


def test_no_config_writes_template(bins, tmp_path):
    for exe in ("recon_lamino", "recon_tomo"):
        r = subprocess.run([bins[exe]], capture_output=True, text=True, cwd=tmp_path)
        assert r.returncode == 1 and "Usage" in r.stderr
        tmpl = (tmp_path / "config_template.toml").read_text()
        assert "[recon_params]" in tmpl and "[[input]]" in tmpl


def test_tomo_prepares_sinogram(bins, tmp_path):
    rng = np.random.default_rng(2)
    a = rng.random((10, 9, 13)).astype(np.float32)
    b = rng.random((6, 9, 13)).astype(np.float32) * 3
    np.save(tmp_path / "a.npy", a)
    np.save(tmp_path / "b.npy", b.astype(np.float64))
    np.savetxt(tmp_path / "ta.txt", np.linspace(0, np.pi, 10, endpoint=False))
    np.save(tmp_path / "tb.npy", np.linspace(0, 90, 6))
    cfg = """[[input]]
filename = "a.npy"
angles = "ta.txt"
angle_units = "rad"
[[input]]
filename = "b.npy"
angles = "tb.npy"
[output]
filename = "r.tiff"
[recon_params]
recon_dims = [9, 12, 12]
"""
    (tmp_path / "t.toml").write_text(cfg)
    rc, d, err = dry(bins["recon_tomo"], str(tmp_path / "t.toml"))
    assert rc == 0, err
    stacked = np.concatenate([a, b]).astype(np.float64)
    assert d["sinogram"] == [9, 16, 13]
    assert abs(d["max_before"] - stacked.max()) < 1e-5
    assert abs(d["sum"] - (stacked / stacked.max()).sum()) < 1e-3
    assert abs(d["theta_last"] - np.deg2rad(90.0)) < 1e-12 and d["recon_dims"] == [9, 11, 11]
    (tmp_path / "t.toml").write_text(cfg.replace("[9, 12, 12]", "[7, 12, 12]"))
    rc, _, err = dry(bins["recon_tomo"], str(tmp_path / "t.toml"))
    assert rc == 2 and "detector row count" in err
    (tmp_path / "t.toml").write_text(cfg.replace('angle_units = "rad"', 'angle_units = "rad"\ngamma = 5'))
    rc, _, err = dry(bins["recon_tomo"], str(tmp_path / "t.toml"))
    assert rc == 2 and "recon_lamino" in err


@pytest.mark.parametrize("big,rps,dtype", [(False, None, np.float32), (True, 3, np.float32),
                                           (False, 2, np.float64), (True, None, np.uint16)])
def test_tiff_read_variants_and_odd_trim(bins, tmp_path, big, rps, dtype):
    rng = np.random.default_rng(3)
    v = (rng.random((3, 8, 10)) * 1000).astype(dtype)
    write_tiff(tmp_path / "v.tiff", v, big_endian=big, rows_per_strip=rps)
    r = subprocess.run([bins["lc_convert"], str(tmp_path / "v.tiff"), str(tmp_path / "v.npy")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    np.testing.assert_array_equal(np.load(tmp_path / "v.npy"), v[:, :7, :9].astype(np.float32))
    r = subprocess.run([bins["lc_convert"], "--no-trim", str(tmp_path / "v.tiff"), str(tmp_path / "w.npy")],
                       capture_output=True, text=True)
    assert r.returncode == 0 and np.load(tmp_path / "w.npy").shape == (3, 8, 10)


def test_tiff_write_round_trip(bins, tmp_path):
    v = np.random.default_rng(4).standard_normal((4, 7, 9)).astype(np.float32)
    np.save(tmp_path / "v.npy", v)
    r = subprocess.run([bins["lc_convert"], str(tmp_path / "v.npy"), str(tmp_path / "v.tiff")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    np.testing.assert_array_equal(read_tiff(tmp_path / "v.tiff"), v)


def test_tiff_rejects_compressed(bins, tmp_path):
    write_tiff(tmp_path / "c.tiff", np.ones((1, 3, 3), np.float32))
    b = bytearray((tmp_path / "c.tiff").read_bytes())
    at = b.index(struct.pack("<HHI", 259, 3, 1))
    b[at + 8:at + 10] = struct.pack("<H", 5)
    (tmp_path / "c.tiff").write_bytes(bytes(b))
    r = subprocess.run([bins["lc_convert"], str(tmp_path / "c.tiff"), str(tmp_path / "c.npy")],
                       capture_output=True, text=True)
    assert r.returncode == 2 and "compressed" in r.stderr


@pytest.mark.gpu
def test_recon_lamino_matches_python_api(bins, tmp_path, cuda):
    import laminocam_b200 as lc
    from laminocam_b200.synthetic import ellipsoid_phantom
    from oracle import oracle as O
    nth, dims = 40, (7, 31, 31)
    th = np.arange(nth) * 360.0 / nth
    g = -np.deg2rad(30.0)
    pg = lc.PolarGrid(np.deg2rad(th), np.full(nth, g), np.zeros(nth), 31, 31)
    p = lc.forward(ellipsoid_phantom(dims, 6, 7), pg).cpu().numpy().astype(np.float32)
    write_tiff(tmp_path / "p.tiff", p)
    np.savetxt(tmp_path / "a.txt", th)
    (tmp_path / "c.toml").write_text("""[[input]]
filename = "p.tiff"
angles = "a.txt"
gamma = 30
[output]
filename = "o/r.tiff"
[recon_params]
max_iters = 3
tol = 0
xtol = 0
recon_dims = [7, 31, 31]
[recon_params.regularizer]
method = "split_bregman"
[recon_params.regularizer.split_bregman]
lambda = 0.1
mu = 10
""")
    r = subprocess.run([bins["recon_lamino"], str(tmp_path / "c.toml")], capture_output=True, text=True,
                       cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stderr
    got = read_tiff(tmp_path / "o" / "r.tiff")
    ref = lc.MBIR([lc.Dataset(p, np.deg2rad(th), g, 0.0)],
                  lc.ReconParams(regularizer="split_bregman", recon_dims=dims, max_iters=3, tol=0, xtol=0))
    assert O.rel_l2(got, ref) < 1e-4


@pytest.mark.gpu
def test_recon_tomo_matches_python_api(bins, tmp_path, cuda):
    import laminocam_b200 as lc
    from laminocam_b200.synthetic import ellipse_phantom
    from oracle import oracle as O
    n, nth, rows = 63, 60, 3
    th = np.arange(nth) * 180.0 / nth
    imgs = np.stack([ellipse_phantom(n, 8, 10 + k) for k in range(rows)])
    sino = lc.forward2d(imgs, lc.PolarGrid2D(np.deg2rad(th), n)).cpu().numpy()  # {rows, nth, n}
    projs = np.ascontiguousarray(np.transpose(sino, (1, 0, 2)), dtype=np.float32)  # {nth, rows, n}
    np.save(tmp_path / "p.npy", projs)
    np.savetxt(tmp_path / "a.txt", th)
    (tmp_path / "c.toml").write_text("""[[input]]
filename = "p.npy"
angles = "a.txt"
[output]
filename = "r.npy"
[recon_params]
max_iters = 5
tol = 0
xtol = 0
recon_dims = [3, 63, 63]
""")
    r = subprocess.run([bins["recon_tomo"], str(tmp_path / "c.toml")], capture_output=True, text=True,
                       cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stderr
    got = np.load(tmp_path / "r.npy")
    prepared = np.ascontiguousarray(sino / sino.max(), dtype=np.float32)
    ref = lc.MBIR2D(prepared, np.deg2rad(th),
                    lc.ReconParams(regularizer="unconstrained", recon_dims=(3, n, n), max_iters=5, tol=0, xtol=0))
    assert O.rel_l2(got, ref) < 1e-4


FORWARD_CFG = """[input]
filename = "vol.tiff"
[output]
basedir = "fwd"
pad_factor = 1.5
proj_angles = { min = -90, max = 90, n = 30 }
[[projections]]
gamma = 0
filename = "g0.tiff"
[[projections]]
gamma = 25.5
filename = "sub/g25.tiff"
"""


def test_forward_scalar_config(bins, tmp_path):
    """src/radon.cpp: [min, max) in n float steps, every axis padded to
    int(n pad) forced odd, one output file per [[projections]] entry."""
    vol = np.random.default_rng(4).random((9, 21, 23)).astype(np.float32)
    write_tiff(tmp_path / "vol.tiff", vol)
    (tmp_path / "f.toml").write_text(FORWARD_CFG)
    rc, out, err = dry(bins["forward_scalar"], str(tmp_path / "f.toml"))
    assert rc == 0, err
    assert out["volume"] == [9, 21, 23]
    assert out["padded"] == [13, 31, 33]  # int(1.5 n) -> 13, 31, 34 -> 33
    assert out["angles"] == 30 and out["angle0"] == -90.0 and out["angle_last"] == 84.0
    assert [p["gamma"] for p in out["projections"]] == [0.0, 25.5]
    assert out["projections"][1]["file"].endswith("fwd/sub/g25.tiff")
    assert abs(out["sum"] - float(vol.astype(np.float64).sum())) < 1e-3 * vol.size
    (tmp_path / "g.toml").write_text("[output]\nbasedir = 'x'\n")
    rc, _, err = dry(bins["forward_scalar"], str(tmp_path / "g.toml"))
    assert rc != 0 and "input and output sections are required" in err


@pytest.mark.gpu
def test_forward_scalar_matches_python_api(bins, tmp_path, cuda):
    """The tool's files against lc.forward of the same padded volume, cropped."""
    import laminocam_b200 as lc
    from oracle import oracle as O
    vol = np.random.default_rng(5).random((9, 21, 23)).astype(np.float32)
    write_tiff(tmp_path / "vol.tiff", vol)
    (tmp_path / "f.toml").write_text(FORWARD_CFG)
    r = subprocess.run([bins["forward_scalar"], str(tmp_path / "f.toml")], capture_output=True, text=True,
                       cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stderr
    ang = np.loadtxt(tmp_path / "fwd" / "angles.txt")
    assert ang.shape == (30,) and ang[0] == -90 and ang[-1] == 84
    vp = np.zeros((13, 31, 33), np.float32)
    vp[2:11, 5:26, 5:28] = vol
    th = (np.float32(-90) + np.arange(30, dtype=np.float32) * np.float32(6)) * np.float32(np.pi) / np.float32(180)
    for gamma, name in ((0.0, "g0.tiff"), (25.5, "sub/g25.tiff")):
        g = np.float32(gamma) * np.float32(np.pi) / np.float32(180)
        pg = lc.PolarGrid(th.astype(np.float64), np.full(30, float(g)), np.zeros(30), 31, 33)
        want = lc.forward(vp, pg).cpu().numpy()[:, 5:26, 5:28]
        got = read_tiff(tmp_path / "fwd" / name)
        assert got.shape == (30, 21, 23)
        assert O.rel_l2(got, want) < 1e-6, name
