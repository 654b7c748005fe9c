"""CPU-only checks of the native library: it loads, exports every symbol the
C header declares, its host-side WCS agrees with wcslib, and the device
HEALPix arithmetic (built for the host) reproduces the reference's keys."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, load_case
from hcgrid_b200 import api, synth
from oracle import oracle as O

HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(hcg_\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_loads_and_exports_every_declared_symbol():
    L = api.load(build_if_missing=True)
    names = declared_symbols()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # the binding covers the whole header
    assert set(names) <= set(api.EXPORTS), set(names) - set(api.EXPORTS)


# The reference's C++ names (HCGrid/gmap.h, gridding.h, healpix.h) and
# globals: a driver compiled against the reference's headers links to these.
REFERENCE_CXX = ["_Healpix_init(unsigned long, unsigned int)",
                 "_prepare_grid_kernel(unsigned int, double*, double, double)",
                 "read_input_map(char const*)", "read_output_map(char const*)", "set_WCS()",
                 "write_output_map(char const*)", "write_ordered_map(char const*, char const*)",
                 "init_input_with_cpu(int const&)", "init_input_with_thrust(int const&)", "init_output()",
                 "data_alloc()", "data_h2d()", "data_d2h()", "data_free()",
                 "solve_gridding(char const*, char const*, char const*, char const*, int const&, int const&)"]
REFERENCE_GLOBALS = ["h_GMaps", "h_Healpix", "h_lons", "h_lats", "h_data", "h_weights", "h_hpx_idx", "h_start_ring",
                     "h_header", "h_zyx", "h_xwcs", "h_ywcs", "h_datacube", "h_weightscube", "h_kernel_params",
                     "last_sphere_radius", "last_hpxmaxres"]


def test_reference_cxx_names_and_globals_are_exported():
    api.load(build_if_missing=True)
    out = subprocess.run(["nm", "-DC", api.lib_path()], capture_output=True, text=True, check=True).stdout
    defined = set()
    for line in out.splitlines():
        parts = line.split(None, 2)
        if len(parts) == 3 and parts[1] in ("T", "B", "D"):
            defined.add(parts[2])
    missing = [n for n in REFERENCE_CXX + REFERENCE_GLOBALS if n not in defined]
    assert not missing, missing


def test_status_strings_and_no_device_errors():
    L = api.load()
    for s in range(8):
        assert L.hcg_status_string(s)
    h = C.c_void_p()
    st = L.hcg_context_create(-1, None, C.byref(h))
    assert st == 4  # HCG_EDEVICE: no such device, no exit()
    assert L.hcg_grid(None, None, None, None, 0, None, 0, 0) == 1  # HCG_EINVAL
    assert L.hcg_field_band_samples(None, None, None, 0, 0, None, None) == 1
    assert L.hcg_grid_planes(None, None, None, None, 0, None, 1, None, 0, 0) == 1
    assert L.hcg_autotune_layout(None, 0) == 1


def _reference_header(path):
    b = open(path, "rb").read()
    cards = []
    i = 0
    while True:
        c = b[i * 80:(i + 1) * 80].decode()
        cards.append(c)
        i += 1
        if c.startswith("END"):
            return "".join(cards)


WCS_CASES = [(30, 40, 300, 60 / 3600), (0.3, 10, 40, 90 / 3600), (120, 76, 40, 72 / 3600),
             (250, -25, 64, 0.01), (180, 30, 120, 1 / 60), (45, 85, 64, 0.02)]


@pytest.mark.skipif(not O.have_ref(), reason="reference host build (oracle/_ref) not present")
@pytest.mark.parametrize("case", WCS_CASES + ["target1"])
def test_header_coords_match_wcslib(case):
    import fitsutil
    if case == "target1":
        hdr = _reference_header(os.path.join(O.reference_data(), "target1.fits"))
    else:
        ra, dec, nx, pix = case
        hdr = synth.sin_header(nx, nx, ra, dec, pix)
    nx1, ny1, x, y = api.header_coords(hdr)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "t.fits")
        fitsutil.write_header_only(p, hdr)
        rx, ry, rz, xw, yw = O.ref_target_wcs(p)
    assert (nx1, ny1) == (rx, ry)
    dx = np.abs(((x - xw + 180.0) % 360.0) - 180.0)
    assert dx.max() < 1e-10 and np.abs(y - yw).max() < 1e-10


def test_header_coords_golden_target():
    """target1.fits coordinates recorded from the reference's set_WCS."""
    c = load_case("input1_target1")
    hdr = synth.sin_header(90, 90, 60.0, 30.0, 0.055555555555556)
    nx, ny, x, y = api.header_coords(hdr)
    assert (nx, ny) == (int(c["nx"]), int(c["ny"]))
    assert np.abs(x - c["xwcs"]).max() < 1e-10 and np.abs(y - c["ywcs"]).max() < 1e-10


def test_header_rejects_other_projections():
    hdr = synth.sin_header(8, 8, 10, 10, 0.1).replace("RA---SIN", "RA---TAN").replace("DEC--SIN", "DEC--TAN")
    with pytest.raises(api.HcgError) as e:
        api.header_coords(hdr)
    assert e.value.status == 6


@pytest.fixture(scope="module")
def hostmath():
    d = tempfile.mkdtemp()
    so = os.path.join(d, "hostmath.so")
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC",
                    "-I", os.path.join(ROOT, "hcgrid_b200", "csrc"), os.path.join(ROOT, "tests", "hostmath.cpp"),
                    "-o", so, "-lquadmath", "-lm"], check=True)
    L = C.CDLL(so)
    f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    u64 = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
    L.hm_ang2pix.argtypes = [C.c_uint64, C.c_long, f64, f64, u64, C.POINTER(C.c_long)]
    L.hm_cos_check.argtypes = [C.c_long, f64] + [C.POINTER(C.c_long)] * 4
    return L


def test_correctly_rounded_cos(hostmath):
    rng = np.random.default_rng(7)
    th = np.concatenate([rng.uniform(0, np.pi, 400_000), np.ldexp(rng.uniform(0.5, 1, 50_000),
                                                                   -rng.integers(0, 60, 50_000))])
    bc, bs, dl, hd = (C.c_long() for _ in range(4))
    hostmath.hm_cos_check(len(th), th, C.byref(bc), C.byref(bs), C.byref(dl), C.byref(hd))
    assert bc.value == 0 and bs.value == 0 and hd.value == 0
    # host libm's cos is not correctly rounded on a small fraction of inputs
    assert dl.value < 0.005 * len(th)


@pytest.mark.parametrize("nside", [1, 4, 64, 4096, 8192, 32768])
def test_device_ang2pix_matches_reference_keys(hostmath, nside):
    """Random and ring-boundary inputs: the device arithmetic gives the
    reference's pixels (recorded golden keys and the oracle's host-libm
    keys); any difference must come from host libm's misrounded cos."""
    rng = np.random.default_rng(nside)
    th = np.concatenate([rng.uniform(0, np.pi, 200_000), np.array([0.0, np.pi, -1e-9, np.nan, 0.01, np.pi - 0.01])])
    ph = np.concatenate([rng.uniform(-7, 14, 200_000), np.zeros(6)])
    out = np.empty(len(th), np.uint64)
    hd = C.c_long()
    hostmath.hm_ang2pix(nside, len(th), th, ph, out, C.byref(hd))
    ref = O.ang2pix(O.healpix(nside), th, ph)
    np.testing.assert_array_equal(out, ref)


def test_device_ang2pix_on_golden_boundary_vectors(hostmath):
    g = np.load(os.path.join(ROOT, "tests", "golden", "healpix.npz"))
    for nside in (1, 2, 4, 64, 1024, 8192, 32768):
        th, ph, keys = g["n%d_theta" % nside], g["n%d_phi" % nside], g["n%d_keys" % nside]
        out = np.empty(len(th), np.uint64)
        hd = C.c_long()
        hostmath.hm_ang2pix(nside, len(th), np.ascontiguousarray(th), np.ascontiguousarray(ph), out, C.byref(hd))
        bad = np.nonzero(out != keys)[0]
        for i in bad:  # only where libm's cos is not the correctly rounded value
            assert np.cos(th[i]) != float(np.float64(np.cos(np.longdouble(th[i])))), (nside, th[i])
        assert len(bad) <= 2, (nside, len(bad))
