"""Grid kernels other than GAUSS1D (HCGrid/gridding.cu:237-257) on every
engine, through the C ABI: GAUSS2D with the great-circle bearing
(helpers.cu:133-137) and TAPERED_SINC in the reference's form (taper
exp(+(arg/a)^2)) and with HCG_TAPER_FIX, against the reference's golden
vectors (tests/golden/kernels.npz) and the FP64 oracle.

These kernels' weights can be negative (sinc lobes) and, in the reference's
taper, grow with distance, so a normalised pixel loses digits to
cancellation. Each pixel's error is bounded by tol * kappa * max|x| with
kappa = sum|w| / |sum w| (from the oracle) and max|x| the channel's largest
|value|:
  * FP32 single-channel engine (FP64 weights and sums): 1e-6;
  * FP32 multi-channel engine (FP32 weights and sums): 1e-5;
  * tensor cores, FP16 hi/lo: 1e-5; BF16 hi/lo: 5e-5.
Weight maps: within 1e-6 * sum|w| (FP32 weights summed in FP64)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from hcgrid_b200 import api, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SINGLE = "single"  # the FP32 engine on a one-channel field (FP64 weights)
TOL = {SINGLE: 1e-6, api.ENGINE_FP32: 1e-5, api.ENGINE_TC_F16: 1e-5, api.ENGINE_TC_BF16: 5e-5}
ENGINES = [SINGLE, api.ENGINE_FP32, api.ENGINE_TC_F16, api.ENGINE_TC_BF16]


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def golden():
    z = np.load(os.path.join(GOLDEN, "kernels.npz"))
    return {k: z[k] for k in z.files}


def oracle(lon, lat, vals, xw, yw, sigma, r, res, kt, params, weights=None):
    """FP64 oracle: unnormalised cube [npix, C], weight sums, sum |w|."""
    g = O.prepare_grid_kernel(sigma, r, res, kt, params)
    ps = O.presort(g.hpx, lon, lat)
    w = None if weights is None else np.asarray(weights, np.float64)[ps.perm]
    v = np.asarray(vals, np.float64).reshape(len(lon), -1)
    oc, ow, _, wabs = O.grid(g, ps, lon[ps.perm], lat[ps.perm], v[ps.perm], xw, yw, weights=w, want_abs=True)
    return oc, ow, wabs


def run(ctx, lon, lat, vals32, t, kt, params, r, res, engine, weights=None):
    """Field under kernel (kt, params) gridded on `engine`; returns the
    normalised cube [npix, C] and the weight map."""
    ctx.prepare_grid_kernel(kt, np.array(params, np.float64), r, res)
    f = ctx.field(lon, lat, weights)
    v = vals32[:, :1] if engine == SINGLE else vals32
    f.set_spectra(np.ascontiguousarray(v if v.shape[1] > 1 else v[:, 0]))
    if engine in (api.ENGINE_TC_F16, api.ENGINE_TC_BF16):
        f.split_spectra(engine)
    cube, w = ctx.grid(f, t, engine=api.ENGINE_FP32 if engine == SINGLE else engine)
    f.close()
    return cube.reshape(cube.shape[0], -1), w


def check(cube, wts, oc, ow, wabs, vals, tol):
    """Normalised cube against the oracle's sums, conditioning-scaled."""
    C = cube.shape[1]
    ref = oc[:, :C] / ow[:, None]
    nan = np.isnan(ref)
    assert np.array_equal(np.isnan(cube), nan)
    ok = ~nan
    with np.errstate(divide="ignore", invalid="ignore"):
        kappa = wabs / np.abs(ow)
    xmax = np.abs(np.asarray(vals, np.float64).reshape(len(vals), -1)[:, :C]).max(axis=0)
    err = np.abs(cube.astype(np.float64) - ref)
    bound = tol * kappa[:, None] * xmax[None, :]
    worst = np.max(np.where(ok, err / np.where(ok, bound, 1.0), 0.0))
    assert worst <= 1.0, worst
    assert np.all(np.abs(wts.astype(np.float64) - ow) <= 1e-6 * wabs + 1e-300)
    return worst


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("name", ["gauss2d_pa04", "gauss2d_pa_neg", "sinc"])
def test_kernels_match_reference_golden(ctx, golden, name, engine):
    """The reference's own kernel body (golden vectors) on each engine."""
    z = golden
    kt, params = int(z[name + "_type"]), z[name + "_params"]
    sigma, r, res = float(z["sigma"]), float(z["sphere_radius"]), float(z["hpx_max_res"])
    t = ctx.target(int(z["nx"]), int(z["ny"]), z["xwcs"], z["ywcs"])
    vals = z["values"]
    cube, w = run(ctx, z["lon"], z["lat"], vals.astype(np.float32), t, kt, params, r, res, engine)
    oc, ow, wabs = oracle(z["lon"], z["lat"], vals, z["xwcs"], z["ywcs"], sigma, r, res, kt, params)
    # the oracle is the reference here, bit for bit
    assert np.array_equal(ow, z[name + "_wts"]) and np.array_equal(oc, z[name + "_cube"])
    # float32 spectra: the inputs' rounding (2^-24 relative) is inside the bound
    check(cube, w, oc, ow, wabs, vals, TOL[engine])
    t.close()


@pytest.fixture(scope="module")
def multi(ctx):
    """70 channels (two 64-channel blocks on the tensor cores), 60k samples
    over 1 deg, 48x48 map."""
    job = synth.config2(n=60_000, nchan=70, nx=48, size_deg=1.0, build_values=True)
    t = ctx.target_from_header(job.header)
    xw, yw = t.coords()
    yield job, t, xw, yw
    t.close()


def kernel_params(job, kind):
    s = job.sigma_deg
    return {"gauss2d": (api.GAUSS2D, [1.4 * s, 0.7 * s, 0.9]),
            "sinc": (api.TAPERED_SINC, [s, 2.52, 1.55]),
            "sinc_fix": (api.TAPERED_SINC | api.TAPER_FIX, [s, 2.52, 1.55])}[kind]


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("kind", ["gauss2d", "sinc", "sinc_fix"])
def test_kernels_multichannel_match_oracle(ctx, multi, kind, engine):
    """The reference's taper here grows to exp((3 pi / 2.52)^2) ~ 1.2e6 at
    the radius: the FP16 weight scale drops to 2^-6."""
    job, t, xw, yw = multi
    kt, params = kernel_params(job, kind)
    cube, w = run(ctx, job.lon, job.lat, job.values, t, kt, params, job.sphere_radius, job.hpx_max_res, engine)
    v = job.values[:, :1] if engine == SINGLE else job.values
    oc, ow, wabs = oracle(job.lon, job.lat, v, xw, yw, job.sigma_deg, job.sphere_radius, job.hpx_max_res, kt,
                          params)
    check(cube, w, oc, ow, wabs, v, TOL[engine])


@pytest.mark.parametrize("engine,mode", [(e, api.TC_WEIGHTS_ENTRIES) for e in ENGINES] +
                         [(e, api.TC_WEIGHTS_DIRECT) for e in (api.ENGINE_TC_F16, api.ENGINE_TC_BF16)])
def test_sample_weights_of_either_sign_and_above_one(ctx, multi, engine, mode):
    """GAUSS1D with per-sample weights in [-3, 10]: the reference adds
    in_weights * w whatever its sign (gridding.cu:386-391), so negative
    weights count, and the FP16 tensor-core weights are scaled to the
    field's bound (10 -> 2^11). Both tensor-core weight operands."""
    job, t, xw, yw = multi
    win = np.random.default_rng(7).uniform(-3.0, 10.0, job.n)
    params = [job.sigma_deg, 0.0, 0.0]
    ctx.tc_set_weights(mode)
    try:
        cube, w = run(ctx, job.lon, job.lat, job.values, t, api.GAUSS1D, params, job.sphere_radius,
                      job.hpx_max_res, engine, weights=win)
    finally:
        ctx.tc_set_weights(api.TC_WEIGHTS_AUTO)
    v = job.values[:, :1] if engine == SINGLE else job.values
    oc, ow, wabs = oracle(job.lon, job.lat, v, xw, yw, job.sigma_deg, job.sphere_radius, job.hpx_max_res,
                          api.GAUSS1D, params, weights=win)
    check(cube, w, oc, ow, wabs, v, TOL[engine])


def test_batch_mixes_kernel_types(ctx, multi):
    """hcg_grid_batch with GAUSS1D, GAUSS2D and TAPERED_SINC jobs: each
    equals its single call (the batch kernels take the GAUSS1D jobs, the
    others run on their own)."""
    torch = pytest.importorskip("torch")
    job, t, xw, yw = multi
    fields = []
    for kt, params in [(api.GAUSS1D, [job.sigma_deg, 0.0, 0.0]), kernel_params(job, "gauss2d"),
                       kernel_params(job, "sinc_fix")]:
        ctx.prepare_grid_kernel(kt, np.array(params, np.float64), job.sphere_radius, job.hpx_max_res)
        f = ctx.field(job.lon, job.lat)
        f.set_spectra(job.values)
        fields.append(f)
    P = t.nx * t.ny
    outs, spec = [], []
    for f in fields:
        cube = torch.full((P * job.nchan,), float("inf"), dtype=torch.float32, device="cuda")
        wt = torch.full((P,), float("inf"), dtype=torch.float32, device="cuda")
        outs.append((cube, wt))
        spec.append((f, t, cube, wt, api.SAMPLE_MAJOR))
    ctx.grid_batch(spec)
    torch.cuda.synchronize()
    for k, (f, (cube, wt)) in enumerate(zip(fields, outs)):
        c1, w1 = ctx.grid(f, t)
        got = cube.cpu().numpy().reshape(P, -1)
        if k > 0:  # the same single-job path
            np.testing.assert_array_equal(got, c1)
            np.testing.assert_array_equal(wt.cpu().numpy(), w1)
            continue
        assert np.array_equal(np.isnan(got), np.isnan(c1))
        ok = ~np.isnan(c1)
        assert np.abs(got[ok] - c1[ok]).max() <= 1e-6 * np.abs(c1[ok]).max()
        np.testing.assert_allclose(wt.cpu().numpy(), w1, rtol=1e-6)
    for f in fields:
        f.close()


def test_direct_weight_mode_takes_entries_for_other_kernels(ctx, multi):
    """The in-kernel weight operand evaluates GAUSS1D only: a GAUSS2D field
    under HCG_TC_WEIGHTS_DIRECT grids exactly as with entries."""
    job, t, xw, yw = multi
    kt, params = kernel_params(job, "gauss2d")
    args = (ctx, job.lon, job.lat, job.values, t, kt, params, job.sphere_radius, job.hpx_max_res,
            api.ENGINE_TC_F16)
    ctx.tc_set_weights(api.TC_WEIGHTS_ENTRIES)
    try:
        ref = run(*args)
        ctx.tc_set_weights(api.TC_WEIGHTS_DIRECT)
        got = run(*args)
    finally:
        ctx.tc_set_weights(api.TC_WEIGHTS_AUTO)
    np.testing.assert_array_equal(got[0], ref[0])
    np.testing.assert_array_equal(got[1], ref[1])


def test_weight_range_limits(ctx, multi):
    """The reference's taper with a narrow width a grows to
    exp((pi r / (sigma a))^2) at the radius: a = 1.08 about 1e33, a = 0.5
    about 1e154, both above the multi-channel engines' 2^100 (the tensor
    cores and the FP32 engine refuse such a field, AUTO included). A single
    channel still grids in FP64; at a = 0.5 its FP32 weight map overflows to
    inf."""
    job, t, xw, yw = multi
    s, r, res = job.sigma_deg, job.sphere_radius, job.hpx_max_res
    for a in (1.08, 0.5):
        params = [s, a, 1.55]
        ctx.prepare_grid_kernel(api.TAPERED_SINC, np.array(params), r, res)
        f = ctx.field(job.lon, job.lat)
        f.set_spectra(job.values)
        for engine in (api.ENGINE_AUTO, api.ENGINE_FP32):
            with pytest.raises(api.HcgError) as e:
                ctx.grid(f, t, engine=engine)
            assert e.value.status == 1
        f.split_spectra(api.ENGINE_TC_F16)
        for engine in (api.ENGINE_AUTO, api.ENGINE_TC_F16):
            with pytest.raises(api.HcgError) as e:
                ctx.grid(f, t, engine=engine)
            assert e.value.status == 1
        f.close()
        f = ctx.field(job.lon, job.lat)
        f.set_spectra(np.ascontiguousarray(job.values[:, 0]))
        cube, w = ctx.grid(f, t)
        f.close()
        v = job.values[:, :1]
        oc, ow, wabs = oracle(job.lon, job.lat, v, xw, yw, s, r, res, api.TAPERED_SINC, params)
        ref = oc / ow[:, None]
        nan = np.isnan(ref)
        assert np.array_equal(np.isnan(cube), nan) and (~nan).sum() > 0
        with np.errstate(divide="ignore", invalid="ignore"):
            kappa = wabs / np.abs(ow)
        err = np.abs(cube.astype(np.float64) - ref)[~nan]
        assert np.all(err <= TOL[SINGLE] * kappa[:, None][~nan] * np.abs(v).max())
        with np.errstate(over="ignore"):
            big = np.isinf(ow.astype(np.float32))  # beyond FP32, either sign
        assert np.array_equal(np.isinf(w), big) and np.all(np.sign(w[big]) == np.sign(ow[big]))
        assert np.all(np.abs(w[~big].astype(np.float64) - ow[~big]) <= 1e-6 * wabs[~big] + 1e-300)


def test_noalloc_grids_other_kernels(ctx, golden):
    """hcg_grid_noalloc runs the same single-channel kernel for every kernel
    type: identical to hcg_grid."""
    torch = pytest.importorskip("torch")
    import ctypes as C
    z = golden
    name = "gauss2d_pa04"
    ctx.prepare_grid_kernel(int(z[name + "_type"]), z[name + "_params"].copy(), float(z["sphere_radius"]),
                            float(z["hpx_max_res"]))
    f = ctx.field(z["lon"], z["lat"])
    f.set_spectra(z["values"][:, 0].astype(np.float32))
    t = ctx.target(int(z["nx"]), int(z["ny"]), z["xwcs"], z["ywcs"])
    ref_c, ref_w = ctx.grid(f, t)
    P = t.nx * t.ny
    cube = torch.full((P,), float("inf"), dtype=torch.float32, device="cuda")
    w = torch.full((P,), float("inf"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    st = ctx.L.hcg_grid_noalloc(ctx.h, f.h, t.h, C.c_void_p(cube.data_ptr()), C.c_void_p(w.data_ptr()))
    assert st == 0, ctx.L.hcg_last_error(ctx.h)
    ctx.synchronize()
    np.testing.assert_array_equal(cube.cpu().numpy(), ref_c[:, 0])
    np.testing.assert_array_equal(w.cpu().numpy(), ref_w)
    f.close()
    t.close()
