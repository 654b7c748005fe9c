"""CUDA path against the reference (golden vectors) and the oracle, through
the C ABI. Tolerances: keys, permutation, LUT and candidate counts are
bit-exact; the normalised cube is within 1e-5 of the reference's FP64 cube
relative to the largest |value| of each channel plane (single channel:
1e-6); weights within 1e-6 relative."""
import numpy as np
import pytest

from conftest import load_case
from hcgrid_b200 import api, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CUBE_TOL = 1e-5
CUBE_TOL_1CHAN = 1e-6
WTS_TOL = 1e-6


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def prepare(ctx, sigma, r, res):
    kp = np.array([sigma, 0.0, 0.0])
    ctx.prepare_grid_kernel(api.GAUSS1D, kp, r, res)
    return kp


def assert_cube_close(cube, ref, tol):
    """cube, ref: [npix, nchan]; NaN where the reference has 0/0."""
    nan_ref = np.isnan(ref)
    assert np.array_equal(np.isnan(cube), nan_ref)
    for c in range(ref.shape[1]):
        r = ref[:, c][~nan_ref[:, c]]
        g = cube[:, c][~nan_ref[:, c]].astype(np.float64)
        if r.size == 0:
            continue
        err = np.abs(g - r).max() / max(np.abs(r).max(), 1e-30)
        assert err <= tol, (c, err)


def test_field_sort_and_lut_bitexact(ctx, golden_case):
    c = golden_case
    kp = prepare(ctx, float(c["sigma"]), float(c["sphere_radius"]), float(c["hpx_max_res"]))
    assert kp[0] == float(c["kparam"])
    inf = ctx.info()
    assert inf.nside == int(c["nside"]) and inf.disc_size == float(c["disc_size"])
    f = ctx.field(c["lon"], c["lat"])
    keys, perm, lut, fr, ur = f.sorted()
    np.testing.assert_array_equal(keys, c["keys"])
    np.testing.assert_array_equal(perm, c["perm"])
    assert (fr, ur) == (int(c["firstring"]), int(c["usedrings"]))
    np.testing.assert_array_equal(lut, c["lut"])


@pytest.mark.parametrize("layout", [api.SAMPLE_MAJOR, api.CHANNEL_MAJOR])
def test_grid_matches_reference(ctx, golden_case, layout):
    c = golden_case
    prepare(ctx, float(c["sigma"]), float(c["sphere_radius"]), float(c["hpx_max_res"]))
    f = ctx.field(c["lon"], c["lat"])
    vals = c["values"].astype(np.float32)
    nchan = vals.shape[1]
    if layout == api.SAMPLE_MAJOR:
        f.set_spectra(np.ascontiguousarray(vals))
    else:
        f.set_spectra(np.ascontiguousarray(vals.T), layout=api.CHANNEL_MAJOR)
    t = ctx.target(int(c["nx"]), int(c["ny"]), c["xwcs"], c["ywcs"])
    cube, w = ctx.grid(f, t, layout=layout)
    if layout == api.CHANNEL_MAJOR:
        cube = cube.T
    ref = c["cube"] / c["wts"][:, None]
    assert_cube_close(cube, ref, CUBE_TOL_1CHAN if nchan == 1 else CUBE_TOL)
    ok = c["wts"] > 0
    assert np.abs(w[ok] - c["wts"][ok]).max() / c["wts"].max() <= WTS_TOL
    assert np.all(w[~ok] == 0)
    st = ctx.stats()
    # same candidate pairs as the reference kernel visits
    g = O.prepare_grid_kernel(float(c["sigma"]), float(c["sphere_radius"]), float(c["hpx_max_res"]))
    ps = O.presort(g.hpx, c["lon"], c["lat"])
    _, _, ost = O.grid(g, ps, c["lon"][ps.perm], c["lat"][ps.perm], vals[ps.perm, 0].astype(np.float64),
                       c["xwcs"], c["ywcs"])
    assert st.pairs_within == ost.pairs_within
    assert st.pairs_candidate == ost.pairs_visited
    assert st.ring_skips == 0 and st.hard_roundings == 0


def test_target_from_header_device_matches_host(ctx):
    job = synth.config1(n=20_000, nx=48)
    prepare(ctx, job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    t = ctx.target_from_header(job.header)
    x, y = t.coords()
    nx, ny, hx, hy = api.header_coords(job.header)
    assert (t.nx, t.ny) == (nx, ny)
    # device SIN (CUDA libm) vs host SIN (host libm): same formulas
    assert np.abs(((x - hx + 180.0) % 360.0) - 180.0).max() < 1e-10
    assert np.abs(y - hy).max() < 1e-10


def test_config1_full_size_vs_oracle(ctx):
    """Config 1 (200k samples, 300x300, FWHM 180"): keys/LUT bit-exact,
    cube within tolerance of the FP64 oracle, identical pair counts."""
    job = synth.config1()
    prepare(ctx, job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    t = ctx.target_from_header(job.header)
    xw, yw = t.coords()
    cube, w = ctx.grid(f, t)
    st = ctx.stats()
    g = O.prepare_grid_kernel(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    ps = O.presort(g.hpx, job.lon, job.lat)
    keys, perm, lut, fr, ur = f.sorted()
    np.testing.assert_array_equal(keys, ps.keys)
    np.testing.assert_array_equal(perm, ps.perm)
    np.testing.assert_array_equal(lut, ps.lut)
    oc, ow, ost = O.grid(g, ps, job.lon[ps.perm], job.lat[ps.perm], job.values[ps.perm].astype(np.float64), xw, yw)
    assert st.pairs_within == ost.pairs_within and st.pairs_candidate == ost.pairs_visited
    assert_cube_close(cube, (oc / ow)[:, None], CUBE_TOL_1CHAN)


def test_multichannel_reduced_config2_vs_oracle(ctx):
    """Config-2 generator at reduced size: 300k samples, 3x3 deg, 128
    channels, 180x180 map; FP32 channel sums against the FP64 oracle."""
    job = synth.config2(n=300_000, nchan=128, nx=180, size_deg=3.0, build_values=True)
    prepare(ctx, job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    t = ctx.target_from_header(job.header)
    xw, yw = t.coords()
    cube, w = ctx.grid(f, t)
    st = ctx.stats()
    g = O.prepare_grid_kernel(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    ps = O.presort(g.hpx, job.lon, job.lat)
    oc, ow, ost = O.grid(g, ps, job.lon[ps.perm], job.lat[ps.perm], job.values[ps.perm].astype(np.float64), xw, yw)
    assert st.pairs_within == ost.pairs_within
    assert_cube_close(cube, oc / ow[:, None], CUBE_TOL)


def test_entry_budget_chunks_give_identical_cube(ctx):
    """Splitting the multi-channel work into runs of tile rows (small entry
    budget) changes nothing: same entries, same per-group sums."""
    job = synth.config2(n=120_000, nchan=64, nx=96, size_deg=1.6, build_values=True)
    prepare(ctx, job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    t = ctx.target_from_header(job.header)
    c1, w1 = ctx.grid(f, t)
    ctx.set_entry_budget(200_000)
    try:
        c2, w2 = ctx.grid(f, t)
    finally:
        ctx.set_entry_budget(4 << 30)
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(w1, w2)


@pytest.mark.parametrize("nchan", [1, 64])
def test_ring_pixel_tables_match_binary_searches(ctx, monkeypatch, nchan):
    """The per-ring pixel tables give the windows the binary searches over the
    sorted keys give: same candidates, same pairs, bit-identical cube."""
    job = synth.config2(n=150_000, nchan=nchan, nx=120, size_deg=2.0, build_values=True)
    prepare(ctx, job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    t = ctx.target_from_header(job.header)
    out = []
    for cap in ("0", None):
        if cap is None:
            monkeypatch.delenv("HCG_RING_TABLE_MAX", raising=False)
        else:
            monkeypatch.setenv("HCG_RING_TABLE_MAX", cap)
        f = ctx.field(job.lon, job.lat)
        f.set_spectra(job.values)
        cube, w = ctx.grid(f, t)
        st = ctx.stats()
        out.append((cube, w, st.pairs_candidate, st.pairs_within))
        f.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    assert out[0][2:] == out[1][2:]


@pytest.mark.parametrize("ra", [120.0, 0.4])
@pytest.mark.parametrize("engine,weights", [(api.ENGINE_FP32, api.TC_WEIGHTS_AUTO),
                                            (api.ENGINE_TC_F16, api.TC_WEIGHTS_ENTRIES),
                                            (api.ENGINE_TC_F16, api.TC_WEIGHTS_DIRECT)])
def test_polar_multichannel_vs_oracle(ctx, ra, engine, weights):
    """Pixels within 20 deg of the pole, where the reference takes whole
    rings. The multi-channel path narrows each ring to the pixels that can
    hold a sample within the radius: the accepted pairs, the candidate count
    the reference reports and the cube (within tolerance) stay the
    reference's. RA 0.4: the field crosses RA 0, so windows there wrap and
    keep the whole ring."""
    shape = dict(block=0, n=40_000, size_deg=1.5, ra=ra, dec=78.0, grid=64, nchan=8, fwhm=180.0, seed=11)
    job = synth.block_job(shape)
    prepare(ctx, job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    if engine != api.ENGINE_FP32:
        f.split_spectra(engine)
    t = ctx.target_from_header(job.header)
    xw, yw = t.coords()
    ctx.tc_set_weights(weights)
    try:
        cube, w = ctx.grid(f, t, engine=engine)
    finally:
        ctx.tc_set_weights(api.TC_WEIGHTS_AUTO)
    st = ctx.stats()
    g = O.prepare_grid_kernel(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    ps = O.presort(g.hpx, job.lon, job.lat)
    oc, ow, ost = O.grid(g, ps, job.lon[ps.perm], job.lat[ps.perm], job.values[ps.perm].astype(np.float64), xw, yw)
    assert st.pairs_within == ost.pairs_within
    assert st.pairs_candidate == ost.pairs_visited
    assert_cube_close(cube, oc / ow[:, None], CUBE_TOL)
    ok = ow > 0
    assert np.abs(w[ok] - ow[ok]).max() / ow.max() <= WTS_TOL
    f.close()
    t.close()


def test_invalid_inputs_are_rejected(ctx):
    prepare(ctx, 0.02, 0.06, 0.01)
    lon = np.array([10.0, 10.1, 10.2])
    with pytest.raises(api.HcgError) as e:
        ctx.field(lon, np.array([10.0, np.nan, 10.2]))
    assert e.value.status == 1
    with pytest.raises(api.HcgError) as e:
        ctx.field(lon, np.array([10.0, 95.0, 10.2]))
    assert e.value.status == 1
    f = ctx.field(lon, np.array([10.0, 10.05, 10.1]))
    t = ctx.target(2, 2, np.array([10.0, 10.1, 10.0, 10.1]), np.array([10.0, 10.0, 10.1, 10.1]))
    with pytest.raises(api.HcgError) as e:
        ctx.grid(f, t)  # no spectra yet
    assert e.value.status == 7
    # a field grids with the kernel set up when it was created
    lat = np.array([10.0, 10.05, 10.1])
    ctx.prepare_grid_kernel(api.GAUSS2D, np.array([0.02, 0.01, 0.3]), 0.06, 0.01)
    f2 = ctx.field(lon, lat)
    f2.set_spectra(np.ones(3, np.float32))
    prepare(ctx, 0.02, 0.06, 0.01)
    f1 = ctx.field(lon, lat)
    f1.set_spectra(np.ones(3, np.float32))
    xw, yw = t.coords()
    for f, kt, params in ((f2, O.GAUSS2D, [0.02, 0.01, 0.3]), (f1, O.GAUSS1D, None)):
        _, w = ctx.grid(f, t)
        g = O.prepare_grid_kernel(0.02, 0.06, 0.01, kt, params)
        ps = O.presort(g.hpx, lon, lat)
        _, ow, _ = O.grid(g, ps, lon[ps.perm], lat[ps.perm], np.ones(3), xw, yw)
        np.testing.assert_allclose(w, ow, rtol=1e-6)
    # HCG_TAPER_FIX is TAPERED_SINC's flag; unknown kernel types are refused
    for kt in (api.GAUSS2D | api.TAPER_FIX, 7):
        with pytest.raises(api.HcgError) as e:
            ctx.prepare_grid_kernel(kt, np.array([0.02, 0.01, 0.3]), 0.06, 0.01)
        assert e.value.status == 1
    # outputs declared as device memory must be writable by the context's
    # device: pageable host memory is refused before anything is launched
    import ctypes as C
    host = np.zeros(4, np.float32)
    st = ctx.L.hcg_grid(ctx.h, f1.h, t.h, host.ctypes.data_as(C.c_void_p), api.SAMPLE_MAJOR, None,
                        api.MEM_DEVICE, api.ENGINE_AUTO)
    assert st == 1 and b"device memory" in ctx.L.hcg_last_error(ctx.h)
    assert np.all(host == 0)


def test_empty_pixels_are_nan_and_single_sample_weight(ctx):
    """One sample seen by a row of pixels: weights are exp(-d^2 p0) inside
    the radius, NaN (0/0) outside. A second sample far to the north occupies
    the first used ring, which the reference's search never grids."""
    sigma = 0.02
    r = 3 * sigma
    prepare(ctx, sigma, r, sigma / 2)
    lon = np.array([30.0, 30.0])
    lat = np.array([40.0, 41.0])
    vals = np.array([2.5, -7.0], np.float32)
    f = ctx.field(lon, lat)
    f.set_spectra(vals)
    xs = 30.0 + np.linspace(-0.1, 0.1, 21) / np.cos(np.deg2rad(40.0))
    ys = np.full(21, 40.0)
    t = ctx.target(21, 1, xs, ys)
    cube, w = ctx.grid(f, t)
    g = O.prepare_grid_kernel(sigma, r, sigma / 2)
    ps = O.presort(g.hpx, lon, lat)
    oc, ow, _ = O.grid(g, ps, lon[ps.perm], lat[ps.perm], vals[ps.perm].astype(np.float64), xs, ys)
    has = ow > 0
    assert has.sum() >= 5 and (~has).sum() >= 5
    np.testing.assert_allclose(w, ow, rtol=1e-6)
    d = np.rad2deg(2 * np.arcsin(np.sqrt(np.sin(np.deg2rad(ys - 40.0) / 2) ** 2 + np.cos(np.deg2rad(ys)) *
                                         np.cos(np.deg2rad(40.0)) * np.sin(np.deg2rad(xs - 30.0) / 2) ** 2)))
    np.testing.assert_allclose(w[has], np.exp(-d[has] ** 2 * (0.5 / sigma ** 2)), rtol=1e-6)
    assert np.all(np.isnan(cube[~has, 0])) and np.allclose(cube[has, 0], 2.5)


@pytest.mark.parametrize("layout", [api.SAMPLE_MAJOR, api.CHANNEL_MAJOR])
def test_chunked_host_upload_equals_device_spectra(ctx, layout):
    """Host spectra above twice the upload chunk go up in chunks through two
    staging buffers, each chunk scattered to its sorted rows while the next
    crosses the bus; the field must hold exactly what the one-shot device
    permutation gives: identical cubes (both layouts, a channel count that is
    not a multiple of 4, planes split across chunks)."""
    torch = pytest.importorskip("torch")
    job = synth.config2(n=1_100_000, nchan=4, nx=128, size_deg=4.0)
    prepare(ctx, job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    nchan = 150  # 1.1M x 150 x 4 B = 660 MB > 2 x 256 MB
    rng = np.random.default_rng(11)
    vals = rng.standard_normal((job.n, nchan), dtype=np.float32)
    host = vals if layout == api.SAMPLE_MAJOR else np.ascontiguousarray(vals.T)
    t = ctx.target_from_header(job.header)
    f_host = ctx.field(job.lon, job.lat)
    f_host.set_spectra(host, layout)
    f_dev = ctx.field(job.lon, job.lat)
    f_dev.set_spectra(torch.from_numpy(host).cuda(), layout)
    a, wa = ctx.grid(f_host, t, engine=api.ENGINE_FP32)
    b, wb = ctx.grid(f_dev, t, engine=api.ENGINE_FP32)
    np.testing.assert_array_equal(wa, wb)
    np.testing.assert_array_equal(a, b)
    for f in (f_host, f_dev):
        f.close()
    t.close()
