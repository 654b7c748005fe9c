"""ctypes access to the parity checker -- TEST INFRASTRUCTURE ONLY.

Two libraries, both built by ``oracle/Makefile``:

* ``lib/liboracle.so``      -- the C restatement of HCGrid's gridding path
  (``hcg_oracle.c``; each function cites the reference file:line it follows).
* ``_ref/libhcgrid_ref.so`` -- the reference's own HCGrid sources compiled
  for the host (present only where the reference tree was available at
  build time, or where the built file travelled with the repository).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this module; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "lib", "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libhcgrid_ref.so")
REF_CLI = os.path.join(HERE, "_ref", "HCGrid")

GAUSS1D, GAUSS2D, TAPERED_SINC = 1, 2, 3
TAPER_FIX = 0x100  # OR'd into TAPERED_SINC: taper exp(-(arg/a)^2) instead of the reference's exp(+(arg/a)^2)
MAX_Y = 1 << 30

_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def reference_root() -> str:
    """Where the reference tree lies: $HCG_REFERENCE, else the REF default
    that oracle/Makefile's recipe reads it from (one place holds that path)."""
    env = os.environ.get("HCG_REFERENCE")
    if env:
        return env
    with open(os.path.join(HERE, "Makefile")) as fh:
        for line in fh:
            m = re.match(r"\s*REF\s*\?=\s*(\S+)", line)
            if m:
                return m.group(1)
    return ""


def reference_data() -> str:
    """The reference's test fixtures (input1.fits, target1.fits)."""
    return os.path.join(reference_root(), "test_data")


def build(with_ref: bool = True, dropin: bool = False) -> None:
    """Compile the restatement (and the reference build when its tree
    exists); `dropin` also links the reference's own driver, unchanged,
    against the B200 library (the relink check of the C++ boundary)."""
    targets = ["oracle"] + (["ref"] if with_ref else []) + (["dropin"] if dropin and with_ref else [])
    env = dict(os.environ, REF=reference_root())
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True, env=env)


class Healpix(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("nside", "order", "nrings", "npface", "ncap", "npix")] + [
        (n, C.c_double) for n in ("fact1", "fact2", "resolution", "omega")
    ]


class GMaps(C.Structure):
    _fields_ = [
        ("hpx", Healpix),
        ("kernel_type", C.c_uint32),
        ("params", C.c_double * 3),
        ("sphere_radius", C.c_double),
        ("disc_size", C.c_double),
        ("bearing_needed", C.c_int),
        ("taper_fix", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [("pairs_visited", C.c_longlong), ("pairs_within", C.c_longlong), ("a3_events", C.c_longlong)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_ORACLE):
            build(with_ref=False)
        L = C.CDLL(LIB_ORACLE)
        L.orc_healpix_init.argtypes = [C.POINTER(Healpix), C.c_uint64]
        L.orc_ang2pix.argtypes = [C.POINTER(Healpix), C.c_double, C.c_double]
        L.orc_ang2pix.restype = C.c_uint64
        L.orc_pix2ring.argtypes = [C.POINTER(Healpix), C.c_uint64]
        L.orc_pix2ring.restype = C.c_uint64
        L.orc_set_optimal_nside.argtypes = [C.c_double]
        L.orc_set_optimal_nside.restype = C.c_uint64
        L.orc_prepare_grid_kernel.argtypes = [C.POINTER(GMaps), C.c_uint32, _f64p, C.c_double, C.c_double]
        L.orc_prepare_grid_kernel.restype = C.c_int
        L.orc_sample_keys.argtypes = [C.POINTER(Healpix), C.c_long, _f64p, _f64p, _u64p]
        L.orc_stable_sort.argtypes = [C.c_long, _u64p, _u64p, _u32p]
        L.orc_ring_lut.argtypes = [C.POINTER(Healpix), C.c_long, _u64p, C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_uint64), _u32p, C.c_long]
        L.orc_ring_lut.restype = C.c_long
        L.orc_grid.argtypes = [C.POINTER(GMaps), C.c_long, _u64p, _u32p, C.c_uint64, C.c_uint64, _f64p, _f64p,
                               _f64p, _f64p, C.c_long, C.c_long, _f64p, _f64p, C.c_int, _f64p, _f64p,
                               C.POINTER(Stats)]
        L.orc_grid_ex.argtypes = [C.POINTER(GMaps), C.c_long, _u64p, _u32p, C.c_uint64, C.c_uint64, _f64p, _f64p,
                                  _f64p, _f64p, C.c_long, C.c_long, _f64p, _f64p, C.c_int, _f64p, _f64p, _f64p,
                                  C.POINTER(Stats)]
        L.orc_pixel_windows.argtypes = [C.POINTER(GMaps), C.c_long, _u64p, _u32p, C.c_uint64, C.c_uint64,
                                        C.c_double, C.c_double, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                        _u32p, _u32p, C.c_long, C.POINTER(C.c_long)]
        L.orc_pixel_windows.restype = C.c_long
        L.orc_ang2pix_many.argtypes = [C.POINTER(Healpix), C.c_long, _f64p, _f64p, _u64p]
        L.orc_pix2ring_many.argtypes = [C.POINTER(Healpix), C.c_long, _u64p, _u64p]
        L.orc_pix2ang_many.argtypes = [C.POINTER(Healpix), C.c_long, _u64p, _f64p, _f64p]
        L.orc_ring_info_many.argtypes = [C.POINTER(Healpix), C.c_long, _u64p, _u64p, _u64p]
        _lib = L
    return _lib


def healpix(nside: int) -> Healpix:
    h = Healpix()
    lib().orc_healpix_init(C.byref(h), nside)
    return h


def prepare_grid_kernel(sigma_deg: float, sphere_radius: float, hpx_max_res: float, kernel_type: int = GAUSS1D,
                        params=None) -> GMaps:
    """gmap.cpp:64-99. GAUSS1D takes sigma_deg; GAUSS2D and TAPERED_SINC take
    `params` (three values, used as given)."""
    g = GMaps()
    p = np.array([sigma_deg, 0.0, 0.0]) if params is None else np.array(params, np.float64).copy()
    rc = lib().orc_prepare_grid_kernel(C.byref(g), kernel_type, p, sphere_radius, hpx_max_res)
    assert rc == 0
    return g


def ang2pix(h: Healpix, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    theta = np.ascontiguousarray(theta, np.float64)
    phi = np.ascontiguousarray(phi, np.float64)
    out = np.empty(len(theta), np.uint64)
    lib().orc_ang2pix_many(C.byref(h), len(theta), theta, phi, out)
    return out


def pix2ring(h: Healpix, pix: np.ndarray) -> np.ndarray:
    pix = np.ascontiguousarray(pix, np.uint64)
    out = np.empty(len(pix), np.uint64)
    lib().orc_pix2ring_many(C.byref(h), len(pix), pix, out)
    return out


def pix2ang(h: Healpix, pix: np.ndarray):
    pix = np.ascontiguousarray(pix, np.uint64)
    th = np.empty(len(pix))
    ph = np.empty(len(pix))
    lib().orc_pix2ang_many(C.byref(h), len(pix), pix, th, ph)
    return th, ph


def ring_info(h: Healpix, rings: np.ndarray):
    rings = np.ascontiguousarray(rings, np.uint64)
    sp = np.empty(len(rings), np.uint64)
    npr = np.empty(len(rings), np.uint64)
    lib().orc_ring_info_many(C.byref(h), len(rings), rings, sp, npr)
    return sp, npr


def sample_keys(h: Healpix, lons: np.ndarray, lats: np.ndarray) -> np.ndarray:
    lons = np.ascontiguousarray(lons, np.float64)
    lats = np.ascontiguousarray(lats, np.float64)
    keys = np.empty(len(lons), np.uint64)
    lib().orc_sample_keys(C.byref(h), len(lons), lons, lats, keys)
    return keys


class Presorted:
    """Sorted keys (with the npix sentinel), permutation and ring LUT."""

    def __init__(self, keys, perm, firstring, usedrings, lut):
        self.keys, self.perm, self.firstring, self.usedrings, self.lut = keys, perm, firstring, usedrings, lut


def presort(h: Healpix, lons: np.ndarray, lats: np.ndarray) -> Presorted:
    keys = sample_keys(h, lons, lats)
    n = len(keys)
    sk = np.empty(n + 1, np.uint64)
    perm = np.empty(n, np.uint32)
    lib().orc_stable_sort(n, keys, sk, perm)
    sk[n] = h.npix
    fr, ur = C.c_uint64(), C.c_uint64()
    cap = 4 * h.nside + 2
    lut = np.empty(cap, np.uint32)
    m = lib().orc_ring_lut(C.byref(h), n, sk, C.byref(fr), C.byref(ur), lut, cap)
    assert m > 0
    return Presorted(sk, perm, fr.value, ur.value, lut[:m].copy())


def grid(g: GMaps, ps: Presorted, lons, lats, data, xwcs, ywcs, weights=None, mode=0, want_abs=False):
    """FP64 gridding of sorted inputs. data: [n] or [n, C] in SORTED order.
    Returns (cube[npix, C], weights[npix], stats) unnormalised, and with
    want_abs the per-pixel sum of |weight| as a fourth item."""
    n = len(lons)
    data = np.asarray(data, np.float64)
    squeeze = data.ndim == 1
    data2 = np.ascontiguousarray(data.reshape(n, -1))
    nchan = data2.shape[1]
    if weights is None:
        weights = np.ones(n)
    npix = len(xwcs)
    cube = np.empty((npix, nchan))
    wts = np.empty(npix)
    wabs = np.empty(npix)
    st = Stats()
    lib().orc_grid_ex(C.byref(g), n, ps.keys, ps.lut, ps.firstring, ps.usedrings,
                      np.ascontiguousarray(lons, np.float64), np.ascontiguousarray(lats, np.float64),
                      np.ascontiguousarray(weights, np.float64), data2, nchan, npix,
                      np.ascontiguousarray(xwcs, np.float64), np.ascontiguousarray(ywcs, np.float64), mode,
                      cube, wts, wabs, C.byref(st))
    out = (cube[:, 0] if squeeze else cube), wts, st
    return out + (wabs,) if want_abs else out


def pixel_windows(g: GMaps, ps: Presorted, xw: float, yw: float, cap: int = 4096):
    lo = np.empty(cap, np.uint32)
    hi = np.empty(cap, np.uint32)
    ur, dr, a3 = C.c_uint64(), C.c_uint64(), C.c_long()
    k = lib().orc_pixel_windows(C.byref(g), len(ps.keys) - 1, ps.keys, ps.lut, ps.firstring, ps.usedrings,
                                float(xw), float(yw), C.byref(ur), C.byref(dr), lo, hi, cap, C.byref(a3))
    assert k >= 0
    return ur.value, dr.value, lo[:k].copy(), hi[:k].copy(), a3.value


# ---------------------------------------------------------------------------
# The reference's own code (host build)

_ref = None


def have_ref() -> bool:
    return os.path.exists(LIB_REF)


def ref():
    global _ref
    if _ref is None:
        R = C.CDLL(LIB_REF)
        R.ref_healpix_init.argtypes = [C.c_uint64]
        R.ref_healpix_state.argtypes = [_u64p, _f64p]
        R.ref_prepare_grid_kernel.argtypes = [C.c_uint32, _f64p, C.c_double, C.c_double, _f64p,
                                              C.POINTER(C.c_double), C.POINTER(C.c_double)]
        R.ref_ang2pix.argtypes = [C.c_long, _f64p, _f64p, _u64p]
        R.ref_loc2pix.argtypes = [C.c_long, _f64p, _f64p, _f64p, _i32p, _u64p]
        R.ref_pix2ring.argtypes = [C.c_long, _u64p, _u64p]
        R.ref_ring_info.argtypes = [C.c_long, _u64p, _u64p, _u64p, _i32p]
        R.ref_pix2ang.argtypes = [C.c_long, _u64p, _f64p, _f64p]
        R.ref_set_optimal_nside.argtypes = [C.c_double]
        R.ref_set_optimal_nside.restype = C.c_uint64
        R.ref_presort.argtypes = [C.c_uint32, _f64p, _f64p, _f64p, C.c_int, _u64p, _f64p, _f64p, _f64p,
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), _u32p, C.c_uint32]
        R.ref_presort.restype = C.c_int
        R.ref_grid.argtypes = [C.c_uint32, _u64p, _f64p, _f64p, _f64p, _f64p, _u32p, C.c_uint64, C.c_uint64,
                               C.c_uint32, C.c_uint32, _f64p, _f64p, C.c_uint32, _f64p, _f64p]
        R.ref_grid.restype = C.c_int
        R.ref_solve_gridding.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_uint32]
        R.ref_target_wcs.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                     C.POINTER(C.c_uint32), _f64p, _f64p, C.c_long]
        R.ref_target_wcs.restype = C.c_int
        _ref = R
    return _ref


def ref_prepare(sigma_deg: float, sphere_radius: float, hpx_max_res: float, kernel_type: int = GAUSS1D,
                params=None):
    """HCGrid.cpp:137-151 sequence: _Healpix_init(1, RING), then
    _prepare_grid_kernel. Returns (params_after, disc_size, healpix_state)."""
    R = ref()
    R.ref_healpix_init(1)
    out = np.zeros(3)
    ds, sr = C.c_double(), C.c_double()
    p = np.array([sigma_deg, 0.0, 0.0]) if params is None else np.array(params, np.float64).copy()
    R.ref_prepare_grid_kernel(kernel_type, p, sphere_radius, hpx_max_res, out, C.byref(ds), C.byref(sr))
    return out, ds.value, ref_state()


def ref_state():
    u = np.zeros(8, np.uint64)
    d = np.zeros(4)
    ref().ref_healpix_state(u, d)
    return u, d


def ref_presort(lons, lats, data, order_arg=2):
    n = len(lons)
    keys = np.empty(n + 1, np.uint64)
    lo, la, da = np.empty(n), np.empty(n), np.empty(n)
    fr, ur = C.c_uint64(), C.c_uint64()
    cap = 1 << 20
    lut = np.empty(cap, np.uint32)
    rc = ref().ref_presort(n, np.ascontiguousarray(lons, np.float64), np.ascontiguousarray(lats, np.float64),
                           np.ascontiguousarray(data, np.float64), order_arg, keys, lo, la, da, C.byref(fr),
                           C.byref(ur), lut, cap)
    assert rc == 0
    return keys, lo, la, da, fr.value, ur.value, lut[: ur.value + 1].copy()


def ref_grid(keys, lons, lats, data, lut, firstring, usedrings, nx, ny, xwcs, ywcs, weights=None, factor=1):
    """The reference's kernel body on the host (one channel, square maps);
    `factor` is its coarsening factor h_GMaps.factor (1-3)."""
    n = len(lons)
    if weights is None:
        weights = np.ones(n)
    num = nx * ny
    cube = np.empty(num)
    wts = np.empty(num)
    ref().ref_grid(n, keys, np.ascontiguousarray(lons, np.float64), np.ascontiguousarray(lats, np.float64),
                   np.ascontiguousarray(data, np.float64), np.ascontiguousarray(weights, np.float64), lut,
                   firstring, usedrings, nx, ny, np.ascontiguousarray(xwcs, np.float64),
                   np.ascontiguousarray(ywcs, np.float64), factor, cube, wts)
    return cube, wts


def ref_target_wcs(path: str, cap: int = 1 << 24):
    nx, ny, nz = C.c_uint32(), C.c_uint32(), C.c_uint32()
    xw = np.empty(cap)
    yw = np.empty(cap)
    ok = ref().ref_target_wcs(path.encode(), C.byref(nx), C.byref(ny), C.byref(nz), xw, yw, cap)
    assert ok == 1
    num = nx.value * ny.value
    return nx.value, ny.value, nz.value, xw[:num].copy(), yw[:num].copy()


def ref_header_coords(header: str):
    """Target pixel centres of a FITS header through the reference's own
    read_output_map + set_WCS (wcslib's wcsp2s, HCGrid/gmap.cpp:151-250):
    the header is written as a header-only FITS file and read back by the
    reference's host build. Returns (nx, ny, xwcs, ywcs) in degrees."""
    import tempfile
    assert len(header) % 80 == 0
    cards = [header[i:i + 80] for i in range(0, len(header), 80)]
    kv = {c[:8].strip(): c[10:].split("/")[0].strip() for c in cards if c[8:10] == "= "}
    n = 1
    for i in range(1, int(kv["NAXIS"]) + 1):
        n *= int(kv["NAXIS%d" % i])
    nb = n * abs(int(kv["BITPIX"])) // 8
    h = header.encode("ascii")
    h += b" " * ((-len(h)) % 2880)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "target.fits")
        with open(p, "wb") as fh:
            fh.write(h)
            fh.write(b"\0" * (nb + (-nb) % 2880))
        nx, ny, _, xw, yw = ref_target_wcs(p, cap=max(1 << 20, n))
    return nx, ny, xw, yw
