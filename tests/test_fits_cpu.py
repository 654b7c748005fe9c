"""FITS boundary of the library (host only) against the reference's files."""
import os
import tempfile

import numpy as np
import pytest

from conftest import load_case
from hcgrid_b200 import api, synth
from oracle import oracle as O
import fitsutil

REF_DATA = O.reference_data()


def test_read_input_map_matches_golden():
    """The reference's input1.fits as read_input_map sees it (values from the
    primary HDU, lon then lat from the second), recorded in the golden case."""
    c = load_case("input1_target1")
    path = os.path.join(REF_DATA, "input1.fits")
    if not os.path.exists(path):
        pytest.skip("reference fixture not present")
    lon, lat, vals = api.fits_read_samples(path)
    np.testing.assert_array_equal(lon, c["lon"])
    np.testing.assert_array_equal(lat, c["lat"])
    np.testing.assert_array_equal(vals[0].astype(np.float64), c["values"][:, 0])


def test_header_and_cube_roundtrip():
    hdr = synth.sin_header(12, 10, 30.0, 40.0, 0.01, nz=3)
    with tempfile.TemporaryDirectory() as d:
        t = os.path.join(d, "t.fits")
        fitsutil.write_header_only(t, hdr)
        h = api.fits_read_header(t)
        assert h.startswith("SIMPLE") and "RA---SIN" in h and h.rstrip().endswith("END")
        assert len(h) % 80 == 0
        nx, ny, x, y = api.header_coords(h)
        assert (nx, ny) == (12, 10)
        rng = np.random.default_rng(0)
        cube = rng.normal(size=(3, 120)).astype(np.float32)
        cube[1, 5] = np.nan
        w = rng.uniform(size=120).astype(np.float32)
        out = os.path.join(d, "o.fits")
        api.fits_write_cube("!" + out, h, 12, 10, cube, w, bitpix=-64)
        hd = fitsutil.read_fits(out)
        assert hd[0][0]["NAXIS1"] == "12" and hd[0][0]["NAXIS3"] == "3" and hd[0][0]["CTYPE1"] == "RA---SIN"
        np.testing.assert_array_equal(hd[0][1].reshape(3, 120), cube.astype(np.float64))
        assert hd[1][0]["EXTNAME"] == "WEIGHTS"
        np.testing.assert_array_equal(hd[1][1], w.astype(np.float64))


def test_missing_file_is_an_io_error():
    with pytest.raises(api.HcgError) as e:
        api.fits_read_samples("/nonexistent/input.fits")
    assert e.value.status == 5


def _card(k, v):
    return ("%-8s= %20s" % (k, v)).ljust(80)


def _hdu(cards, data_be):
    s = "".join(cards + ["END".ljust(80)]).encode("ascii")
    s += b" " * ((-len(s)) % 2880)
    return s + data_be + b"\0" * ((-len(data_be)) % 2880)


@pytest.mark.parametrize("bitpix", [8, 16, 32, 64, -32, -64])
def test_read_every_bitpix_scaled_and_threaded(bitpix):
    """Values of every BITPIX, with BSCALE/BZERO on the integer types, over
    enough samples that several threads and 4 MB pieces share the data unit;
    the sample positions as 32-bit integers scaled to degrees. Each value is
    the big-endian number times BSCALE plus BZERO, as read_input_map reads it."""
    n, z = 300_007, 8
    rng = np.random.default_rng(abs(bitpix))
    dt = fitsutil._DT[bitpix]
    if bitpix > 0:
        info = np.iinfo(np.dtype(dt).newbyteorder("="))
        raw = rng.integers(max(info.min, -(1 << 40)), min(info.max, 1 << 40), size=z * n, endpoint=True)
        scale, zero = 0.5, 3.0
    else:
        raw = rng.normal(size=z * n)
        scale, zero = 1.0, 0.0
    data = np.asarray(raw).astype(dt)
    pos = rng.integers(-(1 << 30), 1 << 30, size=2 * n).astype(">i4")
    prim = [_card("SIMPLE", "T"), _card("BITPIX", bitpix), _card("NAXIS", 3), _card("NAXIS1", 1),
            _card("NAXIS2", n), _card("NAXIS3", z), _card("EXTEND", "T")]
    if bitpix > 0:
        prim += [_card("BSCALE", scale), _card("BZERO", zero)]
    ext = [("%-8s= %-20s" % ("XTENSION", "'IMAGE   '")).ljust(80), _card("BITPIX", 32), _card("NAXIS", 2),
           _card("NAXIS1", n), _card("NAXIS2", 2), _card("PCOUNT", 0), _card("GCOUNT", 1),
           _card("BSCALE", 1e-7), _card("BZERO", 10.0)]
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "in.fits")
        with open(path, "wb") as f:
            f.write(_hdu(prim, data.tobytes()))
            f.write(_hdu(ext, pos.tobytes()))
        lon, lat, vals = api.fits_read_samples(path)
    want = data.astype(np.float64)
    if bitpix > 0:
        want = want * scale + zero
    np.testing.assert_array_equal(vals.reshape(-1), want.astype(np.float32))
    p = pos.astype(np.float64) * 1e-7 + 10.0
    np.testing.assert_array_equal(lon, p[:n])
    np.testing.assert_array_equal(lat, p[n:])


def test_large_cube_write_roundtrip():
    """A cube of several 64 MB conversion rounds (-64) written and read back."""
    nx, ny, nz = 1024, 1024, 9
    hdr = synth.sin_header(nx, ny, 30.0, 40.0, 0.001, nz=nz)
    rng = np.random.default_rng(5)
    cube = rng.normal(size=(nz, nx * ny)).astype(np.float32)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "o.fits")
        api.fits_write_cube("!" + out, hdr, nx, ny, cube, None, bitpix=-64)
        assert os.path.getsize(out) % 2880 == 0
        hd = fitsutil.read_fits(out)
    np.testing.assert_array_equal(hd[0][1].reshape(nz, -1), cube.astype(np.float64))


def test_truncated_data_unit_is_an_io_error():
    rng = np.random.default_rng(1)
    n = 1000
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "in.fits")
        fitsutil.write_input_map(path, rng.normal(size=n), rng.uniform(size=n), rng.uniform(size=n))
        b = open(path, "rb").read()
        open(path, "wb").write(b[:len(b) - 2880])  # the coordinate unit cut short
        with pytest.raises(api.HcgError) as e:
            api.fits_read_samples(path)
    assert e.value.status == 5
