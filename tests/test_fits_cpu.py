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
