"""Generate the golden vectors in tests/golden/ from the reference itself.

Run from the repository root where the reference tree is available:

    python tests/golden/make_golden.py

It builds oracle/_ref (the reference's own HCGrid sources compiled for the
host, see oracle/Makefile) and records, for each case, the inputs and what
the reference's functions return: HEALPix pixel/ring values
(HCGrid/healpix.cu), sorted keys, permutation and ring lookup table
(HCGrid/gridding.cu:70-136, order_arg 2), target pixel coordinates from
set_WCS through wcslib (HCGrid/gmap.cpp:183-250), and the FP64 datacube and
weight map of the `hcgrid` kernel body (HCGrid/gridding.cu:277-403).
Multi-channel cases run the reference kernel once per channel, as HCGrid+
does (HCGrid+/gridding-omp.cu:616-626). kernels.npz holds the same kernel
body with the GAUSS2D and TAPERED_SINC grid kernels (HCGrid/gridding.cu:
237-257, parameters as _prepare_grid_kernel leaves them, gmap.cpp:73-80).

`python tests/golden/make_golden.py kernels` writes kernels.npz alone.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from hcgrid_b200 import synth  # noqa: E402
sys.path.insert(0, os.path.join(ROOT, "tests"))
import fitsutil as F  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
REF_DATA = O.reference_data()


def target_coords(header: str):
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "t.fits")
        F.write_header_only(p, header)
        return O.ref_target_wcs(p)


def grid_case(name, lon, lat, vals, sigma, r, res, nx, ny, xw, yw):
    """Reference presort + kernel for one or more channels."""
    vals = np.asarray(vals, np.float64)
    vals2 = vals.reshape(len(lon), -1)
    params, disc, st = O.ref_prepare(sigma, r, res)
    keys, slon, slat, sdat, fr, ur, lut = O.ref_presort(lon, lat, vals2[:, 0], 2)
    # The reference permutes lon/lat/data with a stable sort of the unsorted
    # keys (gridding.cu:77-114); recompute those keys with its h_ang2pix.
    theta = np.pi / 2 - (np.pi / 180.0) * lat
    phi = (np.pi / 180.0) * lon
    k0 = np.empty(len(lon), np.uint64)
    O.ref().ref_ang2pix(len(lon), np.ascontiguousarray(theta), np.ascontiguousarray(phi), k0)
    perm = np.argsort(k0, kind="stable").astype(np.uint32)
    assert np.array_equal(lon[perm], slon) and np.array_equal(lat[perm], slat)
    assert np.array_equal(vals2[perm, 0], sdat)
    cubes = []
    wts = None
    for c in range(vals2.shape[1]):
        cube, w = O.ref_grid(keys, slon, slat, np.ascontiguousarray(vals2[perm, c]), lut, fr, ur, nx, ny, xw, yw)
        cubes.append(cube)
        if wts is None:
            wts = w
        else:
            assert np.array_equal(wts, w)
    return dict(name=name, lon=lon, lat=lat, values=vals2.astype(np.float64), sigma=sigma, sphere_radius=r,
                hpx_max_res=res, kparam=params[0], disc_size=disc, nside=int(st[0][0]), keys=keys, perm=perm,
                firstring=fr, usedrings=ur, lut=lut, nx=nx, ny=ny, xwcs=xw, ywcs=yw,
                cube=np.stack(cubes, axis=1), wts=wts)


def healpix_vectors():
    rng = np.random.default_rng(123)
    out = {}
    for nside in (1, 2, 4, 64, 1024, 8192, 32768):
        O.ref().ref_healpix_init(nside)
        u, d = O.ref_state()
        npix = int(u[5])
        theta = rng.uniform(0, np.pi, 3000)
        phi = rng.uniform(-7, 14, 3000)
        # ring-boundary thetas: pixel centres of ring starts and their neighbours in ulps
        rings = rng.integers(1, 4 * nside, 200).astype(np.uint64)
        sp = np.empty(200, np.uint64); npr = np.empty(200, np.uint64); sh = np.empty(200, np.int32)
        O.ref().ref_ring_info(200, rings, sp, npr, sh)
        th_c = np.empty(200); ph_c = np.empty(200)
        O.ref().ref_pix2ang(200, sp, th_c, ph_c)
        th_b = np.concatenate([th_c, np.nextafter(th_c, 0), np.nextafter(th_c, 4)])
        ph_b = np.concatenate([ph_c, ph_c, ph_c])
        special = np.array([0.0, 1e-300, 0.005, 0.01, np.nextafter(0.01, 0), np.pi - 0.01, np.pi, np.nextafter(np.pi, 0),
                            np.arccos(2 / 3), np.nextafter(np.arccos(2 / 3), 0), np.nextafter(np.arccos(2 / 3), 4),
                            -1e-9, np.pi + 1e-9, np.nan, np.pi / 2])
        th = np.concatenate([theta, th_b, special])
        ph = np.concatenate([phi, ph_b, rng.uniform(0, 6.3, len(special))])
        keys = np.empty(len(th), np.uint64)
        O.ref().ref_ang2pix(len(th), th, ph, keys)
        ncap = int(u[4])
        edges = [p for p in (0, 1, ncap - 1, ncap, npix - ncap - 1, npix - ncap, npix - 1) if 0 <= p < npix]
        pix = np.concatenate([rng.integers(0, npix, 2000).astype(np.uint64), np.array(edges, np.uint64)])
        pr = np.empty(len(pix), np.uint64)
        O.ref().ref_pix2ring(len(pix), pix, pr)
        pt = np.empty(len(pix)); pp = np.empty(len(pix))
        O.ref().ref_pix2ang(len(pix), pix, pt, pp)
        out["n%d_theta" % nside] = th
        out["n%d_phi" % nside] = ph
        out["n%d_keys" % nside] = keys
        out["n%d_pix" % nside] = pix
        out["n%d_pix2ring" % nside] = pr
        out["n%d_pix2ang_theta" % nside] = pt
        out["n%d_pix2ang_phi" % nside] = pp
        out["n%d_state_u" % nside] = u
        out["n%d_state_d" % nside] = d
    for res_deg in (0.001, 0.0042, 0.0106, 0.0177, 0.1, 1.0):
        out["nside_for_%g" % res_deg] = np.uint64(O.ref().ref_set_optimal_nside(np.deg2rad(res_deg)))
    np.savez_compressed(os.path.join(OUT, "healpix.npz"), **out)


def save(case):
    np.savez_compressed(os.path.join(OUT, case["name"] + ".npz"), **case)
    print("wrote", case["name"], "n=%d" % len(case["lon"]), "pix=%d" % (case["nx"] * case["ny"]),
          "chan=%d" % case["values"].shape[1], "nside=%d" % case["nside"])


def input1_case():
    h = F.read_fits(os.path.join(REF_DATA, "input1.fits"))
    data = h[0][1].reshape(-1).astype(np.float64)
    coords = h[1][1].reshape(-1).astype(np.float64)
    n = len(data)
    lon, lat = coords[:n], coords[n:]
    nx, ny, nz, xw, yw = O.ref_target_wcs(os.path.join(REF_DATA, "target1.fits"))
    fwhm = 180 / 3600.0
    sigma = fwhm / np.sqrt(8 * np.log(2))
    # HCGrid.cpp:146-151: sphere_radius = 5 sigma, hpx_max_res = sigma / 2
    save(grid_case("input1_target1", lon, lat, data, sigma, 5 * sigma, sigma / 2, nx, ny, xw, yw))


def synth_case(name, n, ra, dec, size, nx, pix_arcsec, fwhm, nchan, seed):
    rng = np.random.default_rng(seed)
    lon, lat = synth.raster_scan(n, ra, dec, size, 2.0, rng)
    src = synth.make_sources(12, ra, dec, size, rng)
    if nchan == 1:
        vals = synth.continuum(lon, lat, src, 1.0, 0.05, rng)
    else:
        G, L = synth.line_factors(lon, lat, src, nchan, rng)
        vals = synth.spectra_cpu(G, L, 0.05, rng)
    hdr = synth.sin_header(nx, nx, ra, dec, pix_arcsec / 3600.0)
    tx, ty, tz, xw, yw = target_coords(hdr)
    sigma = fwhm / 3600.0 * synth.FWHM_TO_SIGMA
    case = grid_case(name, lon, lat, vals, sigma, 3 * sigma, sigma / 2, tx, ty, xw, yw)
    case["header"] = np.array(hdr)
    save(case)


# (name, kernel type, parameters in units of sigma except the angle PA in
# radians): GAUSS2D (sigma_maj, sigma_min, PA), TAPERED_SINC (sigma, a, b)
KERNEL_CASES = [
    ("gauss2d_pa04", O.GAUSS2D, (1.3, 0.8, 0.4)),
    ("gauss2d_pa_neg", O.GAUSS2D, (0.7, 1.1, -1.2)),
    ("sinc", O.TAPERED_SINC, (1.0, 9.0, 1.55)),
]


def kernel_cases():
    rng = np.random.default_rng(15)
    ra, dec, size = 30.0, 40.0, 0.6
    lon, lat = synth.raster_scan(6000, ra, dec, size, 2.0, rng)
    vals = np.stack([rng.normal(1.0, 0.3, len(lon)), rng.normal(0.0, 1.0, len(lon))], axis=1)
    hdr = synth.sin_header(24, 24, ra, dec, 60.0 / 3600.0)
    nx, ny, nz, xw, yw = target_coords(hdr)
    sigma = 180.0 / 3600.0 * synth.FWHM_TO_SIGMA
    r, res = 3 * sigma, sigma / 2
    out = dict(lon=lon, lat=lat, values=vals, sigma=sigma, sphere_radius=r, hpx_max_res=res, nx=nx, ny=ny,
               xwcs=xw, ywcs=yw, header=np.array(hdr), names=np.array([c[0] for c in KERNEL_CASES]))
    for name, kt, p in KERNEL_CASES:
        params = np.array([p[0] * sigma, p[1] * sigma if kt == O.GAUSS2D else p[1], p[2]])
        pr, disc, st = O.ref_prepare(sigma, r, res, kt, params)
        assert np.array_equal(pr, params)  # GAUSS2D / TAPERED_SINC parameters are not transformed
        keys, slon, slat, sdat, fr, ur, lut = O.ref_presort(lon, lat, vals[:, 0], 2)
        theta = np.pi / 2 - (np.pi / 180.0) * lat
        phi = (np.pi / 180.0) * lon
        k0 = np.empty(len(lon), np.uint64)
        O.ref().ref_ang2pix(len(lon), np.ascontiguousarray(theta), np.ascontiguousarray(phi), k0)
        perm = np.argsort(k0, kind="stable").astype(np.uint32)
        cubes, wts = [], None
        for c in range(vals.shape[1]):
            cube, w = O.ref_grid(keys, slon, slat, np.ascontiguousarray(vals[perm, c]), lut, fr, ur, nx, ny, xw, yw)
            cubes.append(cube)
            assert wts is None or np.array_equal(wts, w)
            wts = w
        out[name + "_type"] = np.uint32(kt)
        out[name + "_params"] = params
        out[name + "_cube"] = np.stack(cubes, axis=1)
        out[name + "_wts"] = wts
    np.savez_compressed(os.path.join(OUT, "kernels.npz"), **out)
    print("wrote kernels", ", ".join(c[0] for c in KERNEL_CASES))


def main():
    O.build(with_ref=True)
    if sys.argv[1:] == ["kernels"]:
        kernel_cases()
        return
    healpix_vectors()
    input1_case()
    synth_case("synth_dec40", 20000, 30.0, 40.0, 1.2, 48, 60.0, 180.0, 4, 10)
    synth_case("synth_polar", 16000, 120.0, 76.0, 1.0, 40, 72.0, 180.0, 1, 11)
    synth_case("synth_wrap", 16000, 0.3, 10.0, 1.2, 40, 90.0, 180.0, 1, 12)
    synth_case("synth_south", 16000, 250.0, -25.0, 1.0, 40, 72.0, 300.0, 2, 13)
    synth_case("synth_fwhm60", 12000, 80.0, 55.0, 0.3, 32, 20.0, 60.0, 1, 14)
    kernel_cases()


if __name__ == "__main__":
    main()
