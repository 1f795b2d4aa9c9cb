"""Host-side image output (no GPU): the PPM / PFM writers of the C ABI read
back exactly, and the oracle's filmic tone map behaves as the reference's
curve (imagen.h:193-204) and 8-bit conversion (imagen_utils.h:59-62)."""
import numpy as np

from oracle import oracle as orc
from tfg_b200 import pathtracer as pt


def _read_ppm(path):
    data = open(path, "rb").read()
    magic, w, h, mx, rest = data.split(maxsplit=4)
    assert magic == b"P6" and mx == b"255"
    return np.frombuffer(rest, np.uint8).reshape(int(h), int(w), 3)


def _read_pfm(path):
    data = open(path, "rb").read()
    magic, dims, scale, rest = data.split(b"\n", 3)
    w, h = map(int, dims.split())
    assert magic == b"PF" and float(scale) < 0          # little-endian
    return np.frombuffer(rest, "<f4").reshape(h, w, 3)[::-1]   # stored bottom row first


def test_ppm_and_pfm_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    rgb8 = rng.integers(0, 256, (7, 11, 3), dtype=np.uint8)
    hdr = rng.normal(size=(7, 11, 3)).astype(np.float32) * 10
    pt.write_ppm(tmp_path / "a.ppm", rgb8)
    pt.write_pfm(tmp_path / "a.pfm", hdr)
    np.testing.assert_array_equal(_read_ppm(tmp_path / "a.ppm"), rgb8)
    np.testing.assert_array_equal(_read_pfm(tmp_path / "a.pfm"), hdr)


def test_oracle_filmic_curve():
    n = 6
    s = np.array([0, 0, 0, 1e-3, 0.1, 0.5, 1, 2, 4, 100, 1e6, -3, np.nan, 0.25, 0.75, 1.5, 3, 8], np.float32)
    hdr = np.zeros(3 * n, np.float32)
    b = np.zeros(3 * n, np.uint8)
    orc.cpu.orc_tonemap_filmic(orc.p(s), 2, n, orc.p(hdr), orc.p(b))
    np.testing.assert_array_equal(hdr[~np.isnan(s)], (s * np.float32(0.5))[~np.isnan(s)])
    assert b[0] == 0 and b[10] == 255                       # black, saturated white
    # the reference's rational curve is not clamped below: -1.5 maps above 1,
    # i.e. white (the renderer never produces negative radiance)
    assert b[11] == 255
    x = (s[:10] * np.float32(0.5)).astype(np.float64) * 0.6
    f = np.clip(x * (2.51 * x + 0.03) / (x * (2.43 * x + 0.59) + 0.14), 0, 1)
    assert np.abs(b[:10].astype(int) - np.round(f * 255)).max() <= 1
    assert (np.diff(b[:10].astype(int)) >= 0).all()          # monotone in the input
