"""The reference-named C++ layer and the coarsening factor, on the GPU.

* tests/compat_sequence.cpp calls the reference's lower-level names in the
  order of the reference's solve_gridding (read_input_map, read_output_map,
  set_WCS, init_output, init_input_with_cpu, data_alloc, data_h2d, data_d2h,
  write_output_map, write_ordered_map, data_free) and dumps the globals each
  step leaves; they are compared with the golden vectors made by running the
  reference itself on its input1/target1 fixture: kernel setup, sorted keys,
  ring table, sorted coordinates exactly; target pixels within 1e-9 deg;
  the unnormalised sums and weight sums within 1e-6 relative.
* The coarsening factor (h_GMaps.factor 2 and 3) against the reference's own
  kernel body built for the host (oracle/_ref), every engine: the FP64
  single-channel kernel (1e-6), the FP32 and FP16 hi/lo tensor-core
  multi-channel engines (1e-5, relative to each channel plane's largest
  value)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import fitsutil
from conftest import ROOT, load_case
from hcgrid_b200 import api, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LIBDIR = os.path.join(ROOT, "hcgrid_b200", "lib")


@pytest.fixture(scope="module")
def driver():
    d = tempfile.mkdtemp()
    exe = os.path.join(d, "compat_sequence")
    r = subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "compat_sequence.cpp"), "-o", exe, "-L", LIBDIR,
                        "-lhcgrid_b200", "-Wl,-rpath," + LIBDIR], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def run_sequence(exe, c, header, factor=1):
    d = tempfile.mkdtemp()
    fitsutil.write_input_map(os.path.join(d, "in.fits"), c["values"][:, 0], c["lon"], c["lat"])
    fitsutil.write_header_only(os.path.join(d, "tar.fits"), header)
    dump = os.path.join(d, "dump")
    os.makedirs(dump)
    r = subprocess.run([exe, d + "/in.fits", d + "/tar.fits", "!" + d + "/out.fits", "!" + d + "/sorted.fits", dump,
                        repr(float(c["sigma"])), repr(float(c["sphere_radius"])), repr(float(c["hpx_max_res"])),
                        str(factor)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr

    def rd(name, dt):
        return np.fromfile(os.path.join(dump, name + ".bin"), dt)
    return d, rd


def test_reference_call_sequence_leaves_the_reference_globals(driver):
    c = load_case("input1_target1")
    n = len(c["lon"])
    header = synth.sin_header(90, 90, 60.0, 30.0, 0.055555555555556)
    d, rd = run_sequence(driver, c, header)
    setup = rd("setup", np.float64)
    assert setup[0] == c["kparam"] and setup[1] == c["disc_size"]  # _prepare_grid_kernel, bit for bit
    assert rd("healpix", np.uint64)[0] == c["nside"]
    np.testing.assert_array_equal(rd("in_lons", np.float64), c["lon"])  # read_input_map, input order
    np.testing.assert_array_equal(rd("zyx", np.uint32), [1, 90, 90])
    assert np.abs(rd("xwcs", np.float64) - c["xwcs"]).max() < 1e-9  # set_WCS
    assert np.abs(rd("ywcs", np.float64) - c["ywcs"]).max() < 1e-9
    np.testing.assert_array_equal(rd("hpx_idx", np.uint64), c["keys"])  # init_input_with_cpu
    np.testing.assert_array_equal(rd("start_ring", np.uint32), c["lut"])
    np.testing.assert_array_equal(rd("rings", np.uint64), [c["firstring"], c["usedrings"]])
    np.testing.assert_array_equal(rd("sorted_lons", np.float64), c["lon"][c["perm"]])
    np.testing.assert_array_equal(rd("sorted_lats", np.float64), c["lat"][c["perm"]])
    np.testing.assert_array_equal(rd("sorted_data", np.float64), c["values"][c["perm"], 0])
    cube, wts = rd("datacube", np.float64), rd("weightscube", np.float64)  # data_d2h: the kernel's sums
    ok = c["wts"] > 0
    assert np.array_equal(wts > 0, ok)
    assert np.abs(wts[ok] - c["wts"][ok]).max() <= 1e-6 * c["wts"].max()
    ref = c["cube"][:, 0][ok] / c["wts"][ok]
    assert np.abs(cube[ok] / wts[ok] - ref).max() <= 1e-6 * np.abs(ref).max()
    # write_output_map normalised in place and wrote the map; write_ordered_map the sorted samples
    got = fitsutil.read_fits(os.path.join(d, "out.fits"))[0][1].reshape(-1)
    assert np.array_equal(np.isnan(got), ~ok)
    assert np.abs(got[ok] - ref).max() <= 1e-6 * np.abs(ref).max()
    lon_s, lat_s, vals_s = api.fits_read_samples(os.path.join(d, "sorted.fits"))
    np.testing.assert_array_equal(lon_s, c["lon"][c["perm"]])
    np.testing.assert_array_equal(vals_s[0], c["values"][c["perm"], 0].astype(np.float32))
    assert n == len(lon_s)


def reference_coarsened(c, factor):
    """The reference's kernel body (host build) with h_GMaps.factor = factor,
    per channel: normalised cube [npix, nchan] and weights."""
    O.ref_prepare(float(c["sigma"]), float(c["sphere_radius"]), float(c["hpx_max_res"]))
    nx, ny = int(c["nx"]), int(c["ny"])
    cubes, w = [], None
    for ch in range(c["values"].shape[1]):
        keys, sl, sb, sd, fr, ur, lut = O.ref_presort(c["lon"], c["lat"], c["values"][:, ch], 2)
        cube, w = O.ref_grid(keys, sl, sb, sd, lut, fr, ur, nx, ny, c["xwcs"], c["ywcs"], factor=factor)
        cubes.append(cube)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.stack(cubes, 1) / w[:, None], w


@pytest.mark.skipif(not O.have_ref(), reason="reference host build (oracle/_ref) not present")
@pytest.mark.parametrize("case", ["synth_dec40", "synth_polar"])
@pytest.mark.parametrize("factor", [2, 3])
def test_coarsening_factor_matches_reference(case, factor):
    c = load_case(case)
    ref, rw = reference_coarsened(c, factor)
    ctx = api.Context(0)
    ctx.prepare_grid_kernel(api.GAUSS1D, np.array([float(c["sigma"]), 0.0, 0.0]), float(c["sphere_radius"]),
                            float(c["hpx_max_res"]))
    ctx.set_coarsening_factor(factor)
    t = ctx.target(int(c["nx"]), int(c["ny"]), c["xwcs"], c["ywcs"])
    nchan = c["values"].shape[1]
    outs = {}
    for ch in range(nchan):  # the FP64 single-channel kernel
        f = ctx.field(c["lon"], c["lat"])
        f.set_spectra(np.ascontiguousarray(c["values"][:, ch], np.float32))
        cube, w = ctx.grid(f, t)
        outs.setdefault("fp64", []).append(cube[:, 0])
        f.close()
    f = ctx.field(c["lon"], c["lat"])
    f.set_spectra(np.ascontiguousarray(c["values"] if nchan > 1 else c["values"][:, 0], np.float32))
    if nchan > 1:
        outs["fp32"], w32 = ctx.grid(f, t, engine=api.ENGINE_FP32)
        f.split_spectra(api.ENGINE_TC_F16)
        outs["tc"], wtc = ctx.grid(f, t, engine=api.ENGINE_TC_F16)
        np.testing.assert_array_equal(w32, wtc)
    outs["fp64"] = np.stack(outs["fp64"], 1)
    ok = rw > 0
    assert np.abs(w[ok] - rw[ok]).max() <= 1e-6 * rw.max()
    for name, cube in outs.items():
        assert np.array_equal(np.isnan(cube), np.isnan(ref)), name
        tol = 1e-6 if name == "fp64" else 1e-5
        for ch in range(nchan):
            r = ref[ok, ch]
            assert np.abs(cube[ok, ch] - r).max() <= tol * np.abs(r).max(), (name, ch)
    # away from the poles a factor changes the result (near them every pixel of
    # a row takes whole rings over the same ring range, with or without it)
    ctx.set_coarsening_factor(1)
    plain, _ = ctx.grid(f, t, engine=api.ENGINE_FP32 if nchan > 1 else api.ENGINE_AUTO)
    if case != "synth_polar":
        assert not np.allclose(plain[ok], outs["fp64"][ok], rtol=1e-9, equal_nan=True)
    with pytest.raises(api.HcgError):
        ctx.set_coarsening_factor(4)
    f.close()
    t.close()
    ctx.close()
