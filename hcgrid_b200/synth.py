"""Seeded synthetic single-dish workloads for the gridder.

The reference ships no benchmark data (its fixtures are 10k samples), so the
workloads are generated here with numpy's PCG64 from a stated seed:

* raster drift scans: rows along RA stepping in Dec, the RA extent scaled by
  1/cos(dec) so a field is square in true angle (the layout of the
  reference's HCGrid/Create_input_file.py:68-73), Gaussian position jitter;
* continuum values: Gaussian sources with log-uniform amplitudes, a constant
  offset and Gaussian noise (float32);
* spectral cubes: the same sources carrying Gaussian line profiles along the
  channel axis plus noise;
* SIN target headers centred on the field with CRPIX = NAXIS/2 (as in the
  reference's Creat_target_file.py:75-76).

Sample counts are kept exact: a raster of `n` samples uses
round(sqrt(n/2)) rows (keeping the reference's 2:1 row:sample spacing ratio)
and truncates the last row.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

ARCSEC = 1.0 / 3600.0
FWHM_TO_SIGMA = 1.0 / math.sqrt(8.0 * math.log(2.0))


def raster_scan(n: int, ra0: float, dec0: float, size_deg: float, jitter_arcsec: float,
                rng: np.random.Generator) -> tuple[np.ndarray, np.ndarray]:
    """Return (lon, lat) in degrees (float64) of an n-sample raster scan."""
    rows = max(1, int(round(math.sqrt(n / 2.0))))
    per_row = -(-n // rows)
    row_step = size_deg / rows
    samp_step = size_deg / per_row
    dec_rows = dec0 - size_deg / 2 + (np.arange(rows) + 0.5) * row_step
    x = -size_deg / 2 + (np.arange(per_row) + 0.5) * samp_step
    dec = np.repeat(dec_rows, per_row)[:n]
    xt = np.tile(x, rows)[:n]
    j = jitter_arcsec * ARCSEC
    dec = dec + rng.normal(0.0, j, n)
    cosd = np.cos(np.deg2rad(dec))
    ra = ra0 + (xt + rng.normal(0.0, j, n)) / cosd
    ra = np.mod(ra, 360.0)
    return ra.astype(np.float64), dec.astype(np.float64)


@dataclasses.dataclass
class Sources:
    ra: np.ndarray
    dec: np.ndarray
    amp: np.ndarray
    sigma_deg: np.ndarray


def make_sources(nsrc: int, ra0: float, dec0: float, size_deg: float, rng: np.random.Generator) -> Sources:
    dec = dec0 + rng.uniform(-size_deg / 2, size_deg / 2, nsrc)
    ra = ra0 + rng.uniform(-size_deg / 2, size_deg / 2, nsrc) / np.cos(np.deg2rad(dec))
    amp = np.exp(rng.uniform(np.log(0.1), np.log(10.0), nsrc))
    fwhm = rng.uniform(1.0, 10.0, nsrc) / 60.0
    return Sources(ra, dec, amp, fwhm * FWHM_TO_SIGMA)


def source_profile(lon: np.ndarray, lat: np.ndarray, src: Sources, k: int) -> np.ndarray:
    """Spatial Gaussian of source k at the samples (small-angle, cos-dec scaled)."""
    dx = (lon - src.ra[k] + 180.0) % 360.0 - 180.0
    dx = dx * np.cos(np.deg2rad(src.dec[k]))
    dy = lat - src.dec[k]
    return np.exp(-(dx * dx + dy * dy) / (2.0 * src.sigma_deg[k] ** 2))


def continuum(lon: np.ndarray, lat: np.ndarray, src: Sources, offset: float, noise: float,
              rng: np.random.Generator) -> np.ndarray:
    v = np.full(len(lon), offset, np.float64)
    for k in range(len(src.amp)):
        v += src.amp[k] * source_profile(lon, lat, src, k)
    v += rng.normal(0.0, noise, len(lon))
    return v.astype(np.float32)


def line_factors(lon: np.ndarray, lat: np.ndarray, src: Sources, nchan: int,
                 rng: np.random.Generator) -> tuple[np.ndarray, np.ndarray]:
    """Spectral cube as a low-rank product: values = G @ L + noise, with
    G[n, nsrc] the spatial source profiles and L[nsrc, nchan] the Gaussian
    line profiles (centre U(0.1, 0.9)*nchan, width U(0.01, 0.05)*nchan)."""
    nsrc = len(src.amp)
    G = np.empty((len(lon), nsrc), np.float32)
    for k in range(nsrc):
        G[:, k] = src.amp[k] * source_profile(lon, lat, src, k)
    c0 = rng.uniform(0.1, 0.9, nsrc) * nchan
    w = rng.uniform(0.01, 0.05, nsrc) * nchan
    ch = np.arange(nchan)
    L = np.exp(-((ch[None, :] - c0[:, None]) ** 2) / (2.0 * w[:, None] ** 2)).astype(np.float32)
    return G, L


def spectra_cpu(G: np.ndarray, L: np.ndarray, noise: float, rng: np.random.Generator) -> np.ndarray:
    s = G @ L
    s += rng.normal(0.0, noise, s.shape).astype(np.float32)
    return s.astype(np.float32)


def sin_header(nx: int, ny: int, ra0: float, dec0: float, pix_deg: float, nz: int = 1) -> str:
    """FITS header (80-char cards, ending with END) of a RA---SIN/DEC--SIN
    target grid, laid out like the reference's target files."""
    def card(key, val, comment=""):
        if isinstance(val, str):
            v = "'%-8s'" % val
            s = "%-8s= %-20s" % (key, v)
        elif isinstance(val, bool):
            s = "%-8s= %20s" % (key, "T" if val else "F")
        elif isinstance(val, int):
            s = "%-8s= %20d" % (key, val)
        else:
            s = "%-8s= %20s" % (key, repr(float(val)))
        if comment:
            s += " / " + comment
        return s[:80].ljust(80)
    cards = [
        card("SIMPLE", True), card("BITPIX", -32), card("NAXIS", 3), card("NAXIS1", nx), card("NAXIS2", ny),
        card("NAXIS3", nz), card("WCSAXES", 3), card("CRPIX1", nx / 2.0), card("CRPIX2", ny / 2.0),
        card("CRPIX3", 0.0), card("CDELT1", -pix_deg), card("CDELT2", pix_deg), card("CDELT3", 1.0),
        card("CUNIT1", "deg"), card("CUNIT2", "deg"), card("CTYPE1", "RA---SIN"), card("CTYPE2", "DEC--SIN"),
        card("CRVAL1", float(ra0)), card("CRVAL2", float(dec0)), card("CRVAL3", 0.0), card("LONPOLE", 180.0),
        card("LATPOLE", float(dec0)), card("RADESYS", "ICRS"),
    ]
    return "".join(cards) + "END".ljust(80)


@dataclasses.dataclass
class GridJob:
    """One gridding job: samples, values, kernel and target."""
    name: str
    lon: np.ndarray
    lat: np.ndarray
    nchan: int
    values: np.ndarray | None        # [n] or [n, nchan] float32 (None: build lazily from factors)
    factors: tuple | None            # (G, L, noise) for large cubes
    nx: int
    ny: int
    header: str
    fwhm_arcsec: float
    seed: int

    @property
    def n(self) -> int:
        return len(self.lon)

    @property
    def sigma_deg(self) -> float:
        return self.fwhm_arcsec * ARCSEC * FWHM_TO_SIGMA

    @property
    def sphere_radius(self) -> float:
        return 3.0 * self.sigma_deg

    @property
    def hpx_max_res(self) -> float:
        return self.sigma_deg / 2.0


def config1(n: int = 200_000, nx: int = 300, seed: int = 0) -> GridJob:
    """Plain single-channel gridding: 5x5 deg raster at (30, 40), FWHM 180",
    300x300 SIN target with 60" pixels (sizes overridable for tests)."""
    rng = np.random.default_rng(seed)
    lon, lat = raster_scan(n, 30.0, 40.0, 5.0, 2.0, rng)
    src = make_sources(50, 30.0, 40.0, 5.0, rng)
    vals = continuum(lon, lat, src, 1.0, 0.05, rng)
    pix = 60.0 * ARCSEC * (300.0 / nx)
    return GridJob("config1", lon, lat, 1, vals, None, nx, nx, sin_header(nx, nx, 30.0, 40.0, pix), 180.0, seed)


def config2(n: int = 4_000_000, nchan: int = 1024, nx: int = 1200, seed: int = 1, size_deg: float = 20.0,
            build_values: bool = False) -> GridJob:
    """Plain multi-channel gridding at scale: 20x20 deg raster at (180, 30),
    1024 channels of line profiles + N(0, 0.05) noise, 1200x1200 SIN target
    with 60" pixels. Values are returned as low-rank factors (G, L) unless
    build_values is set, so a 16 GB cube can be formed on the device."""
    rng = np.random.default_rng(seed)
    lon, lat = raster_scan(n, 180.0, 30.0, size_deg, 2.0, rng)
    src = make_sources(50, 180.0, 30.0, size_deg, rng)
    G, L = line_factors(lon, lat, src, nchan, rng)
    pix = size_deg / nx
    job = GridJob("config2", lon, lat, nchan, None, (G, L, 0.05), nx, nx,
                  sin_header(nx, nx, 180.0, 30.0, pix), 180.0, seed)
    if build_values:
        job.values = spectra_cpu(G, L, 0.05, rng)
    return job


def config4_shapes(nblocks: int = 256, seed: int = 2):
    """Shapes of the batched form: sample counts log-uniform in [1e4, 2e6],
    fields 1-15 deg at Dec U[-30, 80], grids 64^2..2048^2 (pixel = field /
    grid), channels from {1, 64, 256, 1024, 2048}, FWHM from {60, 180, 300}"."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(nblocks):
        n = int(round(math.exp(rng.uniform(math.log(1e4), math.log(2e6)))))
        size = float(rng.uniform(1.0, 15.0))
        dec = float(rng.uniform(-30.0, 80.0))
        ra = float(rng.uniform(20.0, 340.0))
        grid = int(2 ** rng.integers(6, 12))
        nchan = int(rng.choice([1, 64, 256, 1024, 2048]))
        fwhm = float(rng.choice([60.0, 180.0, 300.0]))
        out.append(dict(block=b, n=n, size_deg=size, ra=ra, dec=dec, grid=grid, nchan=nchan, fwhm=fwhm,
                        seed=int(rng.integers(0, 2**31 - 1))))
    return out


def block_job(shape: dict, build_values: bool = True) -> GridJob:
    """Materialise one config-4 style scan block."""
    rng = np.random.default_rng(shape["seed"])
    lon, lat = raster_scan(shape["n"], shape["ra"], shape["dec"], shape["size_deg"], 2.0, rng)
    src = make_sources(20, shape["ra"], shape["dec"], shape["size_deg"], rng)
    nchan = shape["nchan"]
    g = shape["grid"]
    hdr = sin_header(g, g, shape["ra"], shape["dec"], shape["size_deg"] / g)
    if nchan == 1:
        vals = continuum(lon, lat, src, 1.0, 0.05, rng)
        return GridJob("block%d" % shape["block"], lon, lat, 1, vals, None, g, g, hdr, shape["fwhm"], shape["seed"])
    G, L = line_factors(lon, lat, src, nchan, rng)
    job = GridJob("block%d" % shape["block"], lon, lat, nchan, None, (G, L, 0.05), g, g, hdr, shape["fwhm"],
                  shape["seed"])
    if build_values:
        job.values = spectra_cpu(G, L, 0.05, rng)
    return job


def job_work(shape: dict) -> float:
    """Estimated multiply-adds of one job: pixels x candidates x channels
    (candidates = density x disc area x 1.4 for the ring windows)."""
    sig = shape["fwhm"] / 3600.0 * FWHM_TO_SIGMA
    r = 3.0 * sig
    dens = shape["n"] / shape["size_deg"] ** 2
    return shape["grid"] ** 2 * math.pi * r * r * dens * 1.4 * shape["nchan"]


def config5_requests(njobs: int = 2000, seed: int = 3, reuse: float = 0.3, max_grid: int = 2048,
                     max_values: int = 1 << 62, max_work: float = float("inf"), max_cube: int = 1 << 62):
    """Request stream of the served form: shapes drawn as in config 4 (seed
    `seed`), a fraction `reuse` of requests re-gridding an earlier request's
    field (same samples, new spectra). Caps, when given, redraw shapes whose
    grid, sample-channel count, cube size or estimated work exceed them. Returns dicts
    with the shape, the field id it uses and the seed of its spectra."""
    rng = np.random.default_rng(seed)
    shapes = []
    draws = config4_shapes(nblocks=max(4 * njobs, 64), seed=seed)
    for s in draws:
        if (s["grid"] > max_grid or s["n"] * s["nchan"] > max_values or job_work(s) > max_work
                or s["grid"] ** 2 * s["nchan"] > max_cube):
            continue
        shapes.append(s)
    out = []
    fields = []
    k = 0
    for i in range(njobs):
        if fields and rng.uniform() < reuse:
            fid = int(rng.integers(0, len(fields)))
            shape = dict(fields[fid])
        else:
            shape = dict(shapes[k % len(shapes)])
            k += 1
            fid = len(fields)
            fields.append(shape)
        out.append(dict(request=i, field=fid, shape=shape, spectra_seed=int(rng.integers(0, 2**31 - 1))))
    return out
