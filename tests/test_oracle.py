"""The CPU restatement (oracle/) against the reference's golden vectors and,
where the reference build is present, against the reference itself."""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle as O


@pytest.fixture(scope="module")
def hpx_golden():
    z = np.load(os.path.join(GOLDEN, "healpix.npz"))
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("nside", [1, 2, 4, 64, 1024, 8192, 32768])
def test_healpix_functions_match_reference(hpx_golden, nside):
    g = hpx_golden
    h = O.healpix(nside)
    u = g["n%d_state_u" % nside]
    d = g["n%d_state_d" % nside]
    assert [h.nside, h.order, h.nrings, h.npface, h.ncap, h.npix] == [int(x) for x in u[:6]]
    assert [h.fact1, h.fact2, h.resolution, h.omega] == list(d)
    keys = O.ang2pix(h, g["n%d_theta" % nside], g["n%d_phi" % nside])
    np.testing.assert_array_equal(keys, g["n%d_keys" % nside])
    pix = g["n%d_pix" % nside]
    np.testing.assert_array_equal(O.pix2ring(h, pix), g["n%d_pix2ring" % nside])
    th, ph = O.pix2ang(h, pix)
    np.testing.assert_array_equal(th, g["n%d_pix2ang_theta" % nside])
    np.testing.assert_array_equal(ph, g["n%d_pix2ang_phi" % nside])


def test_optimal_nside_matches_reference(hpx_golden):
    for k, v in hpx_golden.items():
        if k.startswith("nside_for_"):
            res = float(k[len("nside_for_"):])
            assert O.lib().orc_set_optimal_nside(np.deg2rad(res)) == int(v)


def test_prepare_grid_kernel(golden_case):
    c = golden_case
    g = O.prepare_grid_kernel(float(c["sigma"]), float(c["sphere_radius"]), float(c["hpx_max_res"]))
    assert g.params[0] == float(c["kparam"])
    assert g.disc_size == float(c["disc_size"])
    assert g.hpx.nside == int(c["nside"])


def test_presort_and_lut_match_reference(golden_case):
    c = golden_case
    h = O.healpix(int(c["nside"]))
    ps = O.presort(h, c["lon"], c["lat"])
    np.testing.assert_array_equal(ps.keys, c["keys"])
    np.testing.assert_array_equal(ps.perm, c["perm"])
    assert ps.firstring == int(c["firstring"]) and ps.usedrings == int(c["usedrings"])
    np.testing.assert_array_equal(ps.lut, c["lut"])


def test_grid_matches_reference_bitexact(golden_case):
    """FP64 cube and weights identical to the reference kernel body."""
    c = golden_case
    g = O.prepare_grid_kernel(float(c["sigma"]), float(c["sphere_radius"]), float(c["hpx_max_res"]))
    ps = O.presort(g.hpx, c["lon"], c["lat"])
    perm = ps.perm
    cube, wts, st = O.grid(g, ps, c["lon"][perm], c["lat"][perm], c["values"][perm], c["xwcs"], c["ywcs"])
    assert st.a3_events == 0
    np.testing.assert_array_equal(wts, c["wts"])
    np.testing.assert_array_equal(cube, c["cube"])


def test_exact_disc_contains_compat(golden_case):
    """Exact-disc selection is a superset of the reference's ring windows."""
    c = golden_case
    g = O.prepare_grid_kernel(float(c["sigma"]), float(c["sphere_radius"]), float(c["hpx_max_res"]))
    ps = O.presort(g.hpx, c["lon"], c["lat"])
    perm = ps.perm
    args = (g, ps, c["lon"][perm], c["lat"][perm], c["values"][perm, 0], c["xwcs"], c["ywcs"])
    _, w0, s0 = O.grid(*args, mode=0)
    _, w1, s1 = O.grid(*args, mode=1)
    assert s1.pairs_within >= s0.pairs_within
    assert np.all(w1 >= w0 * (1 - 1e-12))


@pytest.mark.skipif(not O.have_ref(), reason="reference host build (oracle/_ref) not present")
@pytest.mark.parametrize("nside", [8192, 32768])
def test_ang2pix_random_vs_reference(nside):
    rng = np.random.default_rng(nside)
    n = 200_000
    th = rng.uniform(0, np.pi, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    O.ref().ref_healpix_init(nside)
    rk = np.empty(n, np.uint64)
    O.ref().ref_ang2pix(n, th, ph, rk)
    np.testing.assert_array_equal(O.ang2pix(O.healpix(nside), th, ph), rk)


@pytest.mark.skipif(not O.have_ref(), reason="reference host build (oracle/_ref) not present")
def test_config1_reduced_vs_reference():
    """A reduced config-1 raster through the live reference build."""
    from hcgrid_b200 import synth
    job = synth.config1(n=40_000, nx=64)
    import fitsutil
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "t.fits")
        fitsutil.write_header_only(p, job.header)
        nx, ny, nz, xw, yw = O.ref_target_wcs(p)
    params, disc, st = O.ref_prepare(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    vals = job.values.astype(np.float64)
    keys, slon, slat, sdat, fr, ur, lut = O.ref_presort(job.lon, job.lat, vals, 2)
    cube_r, wts_r = O.ref_grid(keys, slon, slat, sdat, lut, fr, ur, nx, ny, xw, yw)
    g = O.prepare_grid_kernel(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    ps = O.presort(g.hpx, job.lon, job.lat)
    np.testing.assert_array_equal(ps.keys, keys)
    np.testing.assert_array_equal(ps.lut, lut)
    cube, wts, s = O.grid(g, ps, job.lon[ps.perm], job.lat[ps.perm], vals[ps.perm], xw, yw)
    np.testing.assert_array_equal(wts, wts_r)
    np.testing.assert_array_equal(cube, cube_r)


# ---------------------------------------------------------------------------
# GAUSS2D and TAPERED_SINC grid kernels (HCGrid/gridding.cu:237-257)

@pytest.fixture(scope="module")
def kernels_golden():
    z = np.load(os.path.join(GOLDEN, "kernels.npz"))
    return {k: z[k] for k in z.files}


def _kernel_grid(z, kt, params, weights=None, want_abs=False):
    g = O.prepare_grid_kernel(float(z["sigma"]), float(z["sphere_radius"]), float(z["hpx_max_res"]), kt, params)
    ps = O.presort(g.hpx, z["lon"], z["lat"])
    w = None if weights is None else weights[ps.perm]
    return O.grid(g, ps, z["lon"][ps.perm], z["lat"][ps.perm], z["values"][ps.perm], z["xwcs"], z["ywcs"],
                  weights=w, want_abs=want_abs)


@pytest.mark.parametrize("name", ["gauss2d_pa04", "gauss2d_pa_neg", "sinc"])
def test_kernel_types_match_reference_bitexact(kernels_golden, name):
    z = kernels_golden
    cube, wts, st = _kernel_grid(z, int(z[name + "_type"]), z[name + "_params"])
    assert st.a3_events == 0 and st.pairs_within > 0
    np.testing.assert_array_equal(wts, z[name + "_wts"])
    np.testing.assert_array_equal(cube, z[name + "_cube"])


def test_kernel_types_match_reference_build(kernels_golden):
    """Fresh parameters against the reference's own kernel body (host build)."""
    if not O.have_ref():
        pytest.skip("reference host build not present")
    z = kernels_golden
    rng = np.random.default_rng(3)
    s = float(z["sigma"])
    cases = [(O.GAUSS2D, [s * rng.uniform(0.5, 2), s * rng.uniform(0.5, 2), rng.uniform(-3, 3)]) for _ in range(2)]
    cases += [(O.TAPERED_SINC, [s * rng.uniform(0.7, 1.5), rng.uniform(2, 12), rng.uniform(1, 3)]) for _ in range(2)]
    for kt, params in cases:
        cube, wts, _ = _kernel_grid(z, kt, params)
        O.ref_prepare(s, float(z["sphere_radius"]), float(z["hpx_max_res"]), kt, params)
        keys, slon, slat, sdat, fr, ur, lut = O.ref_presort(z["lon"], z["lat"], z["values"][:, 0], 2)
        rc, rw = O.ref_grid(keys, slon, slat, sdat, lut, fr, ur, int(z["nx"]), int(z["ny"]), z["xwcs"], z["ywcs"])
        np.testing.assert_array_equal(wts, rw)
        np.testing.assert_array_equal(cube[:, 0], rc)


def _hav_deg(l1, b1, l2, b2):
    l1, b1, l2, b2 = map(np.deg2rad, (l1, b1, l2, b2))
    return np.rad2deg(2 * np.arcsin(np.sqrt(np.sin((b1 - b2) / 2) ** 2 + np.cos(b1) * np.cos(b2) *
                                            np.sin((l1 - l2) / 2) ** 2)))


def test_kernel_formulas_single_pairs():
    """One sample, one pixel: the weight map is the kernel itself. GAUSS2D
    with its bearing, TAPERED_SINC in the reference's form exp(+(arg/a)^2)
    and, with TAPER_FIX, exp(-(arg/a)^2)."""
    sigma = 0.02
    r = 3 * sigma
    lon0, lat0 = 50.0, 20.0
    ang = np.linspace(0, 2 * np.pi, 13)[:-1]
    dist = np.linspace(0.002, 0.055, 12)
    lon = lon0 + dist * np.sin(ang) / np.cos(np.deg2rad(lat0))
    lat = lat0 + dist * np.cos(ang)
    for kt, params in [(O.GAUSS2D, [0.03, 0.015, 0.7]), (O.TAPERED_SINC, [0.02, 2.52, 1.55]),
                       (O.TAPERED_SINC | O.TAPER_FIX, [0.02, 2.52, 1.55])]:
        for i in range(len(lon)):
            g = O.prepare_grid_kernel(sigma, r, sigma / 2, kt, params)
            ps = O.presort(g.hpx, np.array([lon[i]]), np.array([lat[i]]))
            _, w, st = O.grid(g, ps, np.array([lon[i]]), np.array([lat[i]]), np.ones(1), np.array([lon0]),
                              np.array([lat0]))
            d = _hav_deg(lon0, lat0, lon[i], lat[i])
            if kt == O.GAUSS2D:
                l1, b1, l2, b2 = map(np.deg2rad, (lon0, lat0, lon[i], lat[i]))
                bear = np.arctan2(np.cos(b2) * np.sin(l2 - l1),
                                  np.cos(b1) * np.sin(b2) - np.sin(b1) * np.cos(b2) * np.cos(l2 - l1))
                p0, p1, pa = params
                ell = p0 ** 2 * np.sin(bear - pa) ** 2 + p1 ** 2 * np.cos(bear - pa) ** 2
                want = np.exp(-((d / p0 / p1) ** 2) / 2 * ell)
            else:
                arg = np.pi * d / params[0]
                x = arg / params[2]
                t = (arg / params[1]) ** 2
                want = np.sin(x) / x * np.exp(-t if kt & O.TAPER_FIX else t)
            if st.pairs_within == 0:
                assert w[0] == 0.0  # the reference's window missed the sample (quirk A1)
                continue
            np.testing.assert_allclose(w[0], want, rtol=1e-12)
    # the flag is TAPERED_SINC's only
    g = O.GMaps()
    assert O.lib().orc_prepare_grid_kernel(ctypes.byref(g), O.GAUSS2D | O.TAPER_FIX, np.zeros(3), r, sigma / 2) == -1


def test_sum_abs_weights_is_the_conditioning(kernels_golden):
    """Sum |w| per pixel: equal to sum w for positive weights (GAUSS1D), at
    least |sum w| with the sinc's negative lobes."""
    z = kernels_golden
    s = float(z["sigma"])
    _, w1, _, a1 = _kernel_grid(z, O.GAUSS1D, [s, 0.0, 0.0], want_abs=True)
    np.testing.assert_allclose(a1, w1, rtol=1e-12)
    _, w2, _, a2 = _kernel_grid(z, O.TAPERED_SINC, [s, 9.0, 1.55], want_abs=True)
    assert np.all(a2 >= np.abs(w2) * (1 - 1e-12)) and np.any(a2 > np.abs(w2) * 1.01)
