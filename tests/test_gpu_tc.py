"""Tensor-core engines (tcgen05, compensated 16-bit hi/lo products) against
the FP64 oracle and the FP32 engine, through the C ABI.

Tolerances, relative to the largest |value| of each channel plane (the
measure of the FP32 parity tests), 1e-5 for both splits, the bound the
north-star workload states:
  * FP16 hi/lo: per-term error of the three-product split ~3 * 2^-22, plus
    FP32 accumulation (measured up to 7.3e-6 on the densest field);
  * BF16 hi/lo: per-term bound 3 * 2^-16 = 4.6e-5, but the errors of the
    many terms of a pixel are independent and partly cancel: measured up to
    5.9e-6 on every field here.
Weights are the FP64 sums of the same entries the FP32 engine uses, so the
weight map is bit-identical to the FP32 engine's, as is the NaN pattern of
empty pixels."""
import numpy as np
import pytest

from hcgrid_b200 import api, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = {api.ENGINE_TC_F16: 1e-5, api.ENGINE_TC_BF16: 1e-5}
ENGINES = [api.ENGINE_TC_F16, api.ENGINE_TC_BF16]


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def prepare(ctx, job):
    ctx.prepare_grid_kernel(api.GAUSS1D, np.array([job.sigma_deg, 0.0, 0.0]), job.sphere_radius, job.hpx_max_res)


def plane_errors(cube, ref):
    """max over channels of max|cube - ref| / max|ref| (NaN patterns equal)."""
    nan = np.isnan(ref)
    assert np.array_equal(np.isnan(cube), nan)
    worst = 0.0
    for c in range(ref.shape[1]):
        r = ref[~nan[:, c], c]
        if r.size == 0:
            continue
        g = cube[~nan[:, c], c].astype(np.float64)
        worst = max(worst, np.abs(g - r).max() / max(np.abs(r).max(), 1e-30))
    return worst


@pytest.fixture
def entries_mode(ctx):
    """Weight operands from the FP64 weight pass's entries: the weight sums
    are then bit-identical to the FP32 engine's."""
    ctx.tc_set_weights(api.TC_WEIGHTS_ENTRIES)
    yield
    ctx.tc_set_weights(api.TC_WEIGHTS_AUTO)


@pytest.fixture(scope="module")
def small(ctx):
    """Config-2 generator, 150k samples over 2 deg, 100 channels (not a
    multiple of 64), 120x120 map: several tiles, ring runs of all lengths."""
    job = synth.config2(n=150_000, nchan=100, nx=120, size_deg=2.0, build_values=True)
    prepare(ctx, job)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    t = ctx.target_from_header(job.header)
    xw, yw = t.coords()
    g = O.prepare_grid_kernel(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    ps = O.presort(g.hpx, job.lon, job.lat)
    oc, ow, _ = O.grid(g, ps, job.lon[ps.perm], job.lat[ps.perm], job.values[ps.perm].astype(np.float64), xw, yw)
    ref = oc / ow[:, None]
    c32, w32 = ctx.grid(f, t, engine=api.ENGINE_FP32)
    yield job, f, t, ref, c32, w32
    f.close()
    t.close()


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("layout", [api.SAMPLE_MAJOR, api.CHANNEL_MAJOR])
def test_tc_matches_oracle(ctx, small, entries_mode, engine, layout):
    job, f, t, ref, c32, w32 = small
    prepare(ctx, job)
    f.split_spectra(engine)
    cube, w = ctx.grid(f, t, layout=layout, engine=engine)
    if layout == api.CHANNEL_MAJOR:
        cube = cube.T
    np.testing.assert_array_equal(w, w32)
    err = plane_errors(cube, ref)
    print(f"engine {engine} layout {layout}: max plane-relative error vs FP64 oracle {err:.3e}")
    assert err <= TOL[engine]
    assert plane_errors(c32, ref) <= 1e-5


def test_auto_engine_uses_the_split(ctx, small):
    job, f, t, ref, c32, w32 = small
    prepare(ctx, job)
    f.split_spectra(api.ENGINE_TC_F16)
    a, _ = ctx.grid(f, t)
    b, _ = ctx.grid(f, t, engine=api.ENGINE_TC_F16)
    np.testing.assert_array_equal(a, b)
    # deterministic: the same launch twice gives the same bits
    c, _ = ctx.grid(f, t, engine=api.ENGINE_TC_F16)
    np.testing.assert_array_equal(b, c)


@pytest.mark.parametrize("nchan", [64, 98, 300])
def test_tc_channel_blocks(ctx, entries_mode, nchan):
    """64 channels (one 64-channel block), 98 (rows not a multiple of 16
    bytes: direct stores instead of the TMA store) and 300 (two CTAs per
    tile, the second partly past the last channel)."""
    job = synth.config2(n=60_000, nchan=nchan, nx=64, size_deg=1.2, build_values=True)
    prepare(ctx, job)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    t = ctx.target_from_header(job.header)
    c32, w32 = ctx.grid(f, t, engine=api.ENGINE_FP32)
    f.split_spectra(api.ENGINE_TC_F16)
    ct, wt = ctx.grid(f, t, engine=api.ENGINE_TC_F16)
    np.testing.assert_array_equal(wt, w32)
    # FP32 engine and FP16 hi/lo engine agree to the split's precision
    assert plane_errors(ct, c32.astype(np.float64)) <= 1e-5


@pytest.mark.parametrize("layout", [api.SAMPLE_MAJOR, api.CHANNEL_MAJOR])
def test_tc_empty_tiles_and_padding(ctx, entries_mode, layout):
    """A 97x97 map larger than the field: partial edge tiles (the TMA store
    clips them; channel-major rows of 97 floats take direct stores) and
    whole tiles without samples, which come out NaN with zero weight exactly
    where the FP32 engine puts them."""
    job = synth.config2(n=30_000, nchan=64, nx=97, size_deg=1.0, build_values=True)
    prepare(ctx, job)
    hdr = synth.sin_header(97, 97, 180.0, 30.0, 2.0 / 97)  # config2 is centred at (180, 30)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    t = ctx.target_from_header(hdr)
    c32, w32 = ctx.grid(f, t, layout=layout, engine=api.ENGINE_FP32)
    f.split_spectra(api.ENGINE_TC_BF16)
    ct, wt = ctx.grid(f, t, layout=layout, engine=api.ENGINE_TC_BF16)
    if layout == api.CHANNEL_MAJOR:
        ct, c32 = ct.T, c32.T
    assert np.isnan(ct).any() and (~np.isnan(ct)).any()
    np.testing.assert_array_equal(np.isnan(ct), np.isnan(c32))
    np.testing.assert_array_equal(wt, w32)
    assert plane_errors(ct, c32.astype(np.float64)) <= 5e-5


@pytest.fixture(scope="module")
def dense(ctx):
    """A beam 27 pixels wide over 2.8k samples per pixel disc (20k samples on
    0.3 deg, 64x64 map, FWHM 180"): tiles whose staged samples mostly lie within
    the radius of their pixels, where the kernel evaluates the weights itself.
    100 channels: two 64-channel blocks, the second partly past the last."""
    shape = dict(block=0, n=20_000, size_deg=0.3, ra=150.0, dec=20.0, grid=64, nchan=100, fwhm=180.0, seed=5)
    job = synth.block_job(shape)
    prepare(ctx, job)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    t = ctx.target_from_header(job.header)
    xw, yw = t.coords()
    g = O.prepare_grid_kernel(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    ps = O.presort(g.hpx, job.lon, job.lat)
    oc, ow, ost = O.grid(g, ps, job.lon[ps.perm], job.lat[ps.perm], job.values[ps.perm].astype(np.float64), xw, yw)
    yield job, f, t, oc / ow[:, None], ow, ost
    f.close()
    t.close()


@pytest.mark.parametrize("mode", [api.TC_WEIGHTS_DIRECT, api.TC_WEIGHTS_ENTRIES])
@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("layout", [api.SAMPLE_MAJOR, api.CHANNEL_MAJOR])
def test_tc_weight_modes_match_oracle(ctx, dense, mode, engine, layout):
    """Both weight-operand modes give the reference's pairs (accepted and
    candidate counts equal to the oracle's), its weight sums within 1e-6 and
    its cube within the split's tolerance."""
    job, f, t, ref, ow, ost = dense
    prepare(ctx, job)
    f.split_spectra(engine)
    ctx.tc_set_weights(mode)
    try:
        cube, w = ctx.grid(f, t, layout=layout, engine=engine)
        st = ctx.stats()
    finally:
        ctx.tc_set_weights(api.TC_WEIGHTS_AUTO)
    if layout == api.CHANNEL_MAJOR:
        cube = cube.T
    assert st.pairs_within == ost.pairs_within
    assert st.pairs_candidate == ost.pairs_visited
    ok = ow > 0
    assert np.abs(w[ok] - ow[ok]).max() / ow.max() <= 1e-6
    err = plane_errors(cube, ref)
    print(f"mode {mode} engine {engine} layout {layout}: max plane-relative error {err:.3e}")
    assert err <= TOL[engine]


@pytest.mark.parametrize("engine", ENGINES)
def test_tc_segments_in_both_cube_layouts(ctx, engine):
    """Tiles longer than one accumulation segment (the dense beam of the
    fixture above) with 256 channels, so pixel-major rows take the 32-byte
    stores and later segments are added to the stored partial sums: the
    pixel-major cube equals the channel-plane cube bit for bit and is within
    the split's tolerance of the FP32 engine."""
    shape = dict(block=0, n=20_000, size_deg=0.3, ra=150.0, dec=20.0, grid=64, nchan=256, fwhm=180.0, seed=5)
    job = synth.block_job(shape)
    prepare(ctx, job)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    t = ctx.target_from_header(job.header)
    try:
        c32, w32 = ctx.grid(f, t, engine=api.ENGINE_FP32)
        f.split_spectra(engine, keep_fp32=False)
        ctx.tc_set_weights(api.TC_WEIGHTS_ENTRIES)
        cs, ws = ctx.grid(f, t, layout=api.SAMPLE_MAJOR, engine=engine)
        cc, wc = ctx.grid(f, t, layout=api.CHANNEL_MAJOR, engine=engine)
        st = ctx.stats()
    finally:
        ctx.tc_set_weights(api.TC_WEIGHTS_AUTO)
        f.close()
        t.close()
    assert st.tc_macs > 0
    np.testing.assert_array_equal(cs, cc.T)
    np.testing.assert_array_equal(ws, wc)
    np.testing.assert_array_equal(ws, w32)
    np.testing.assert_array_equal(np.isnan(cs), np.isnan(c32))
    assert plane_errors(cs, c32.astype(np.float64)) <= TOL[engine]


def test_tc_weight_modes_deterministic_and_checked(ctx, dense):
    """Each mode gives the same bits on every call; the automatic mode is one
    of the two; unknown modes are refused."""
    job, f, t, ref, ow, ost = dense
    prepare(ctx, job)
    f.split_spectra(api.ENGINE_TC_F16)
    out = {}
    for mode in (api.TC_WEIGHTS_AUTO, api.TC_WEIGHTS_ENTRIES, api.TC_WEIGHTS_DIRECT):
        ctx.tc_set_weights(mode)
        try:
            a, wa = ctx.grid(f, t, engine=api.ENGINE_TC_F16)
            b, wb = ctx.grid(f, t, engine=api.ENGINE_TC_F16)
        finally:
            ctx.tc_set_weights(api.TC_WEIGHTS_AUTO)
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(wa, wb)
        out[mode] = (a, wa)
    auto = out[api.TC_WEIGHTS_AUTO][0]
    assert any(np.array_equal(auto, out[m][0], equal_nan=True)
               for m in (api.TC_WEIGHTS_ENTRIES, api.TC_WEIGHTS_DIRECT))
    with pytest.raises(RuntimeError, match="HCG_EINVAL"):
        ctx.tc_set_weights(3)


@pytest.mark.parametrize("nchan", [64, 300])
def test_tc_direct_weights_channel_blocks(ctx, nchan):
    """Direct weights with one 64-channel block (64-channel items) and with
    300 channels (256-channel items, the second partly past the last channel),
    against the FP64 oracle."""
    shape = dict(block=0, n=20_000, size_deg=0.3, ra=150.0, dec=20.0, grid=64, nchan=nchan, fwhm=180.0, seed=6)
    job = synth.block_job(shape)
    prepare(ctx, job)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    t = ctx.target_from_header(job.header)
    xw, yw = t.coords()
    f.split_spectra(api.ENGINE_TC_F16)
    ctx.tc_set_weights(api.TC_WEIGHTS_DIRECT)
    try:
        ct, wt = ctx.grid(f, t, engine=api.ENGINE_TC_F16)
    finally:
        ctx.tc_set_weights(api.TC_WEIGHTS_AUTO)
    g = O.prepare_grid_kernel(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    ps = O.presort(g.hpx, job.lon, job.lat)
    oc, ow, _ = O.grid(g, ps, job.lon[ps.perm], job.lat[ps.perm], job.values[ps.perm].astype(np.float64), xw, yw)
    ok = ow > 0
    assert np.abs(wt[ok] - ow[ok]).max() / ow.max() <= 1e-6
    assert plane_errors(ct, oc / ow[:, None]) <= TOL[api.ENGINE_TC_F16]
    f.close()
    t.close()


def test_tc_state_and_input_checks(ctx):
    job = synth.config2(n=20_000, nchan=64, nx=32, size_deg=0.6, build_values=True)
    prepare(ctx, job)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    t = ctx.target_from_header(job.header)
    with pytest.raises(RuntimeError, match="HCG_ESTATE"):  # no split yet
        ctx.grid(f, t, engine=api.ENGINE_TC_F16)
    f.split_spectra(api.ENGINE_TC_BF16)
    with pytest.raises(RuntimeError, match="HCG_ESTATE"):  # split of the other format
        ctx.grid(f, t, engine=api.ENGINE_TC_F16)
    with pytest.raises(RuntimeError, match="HCG_EINVAL"):
        ctx.grid(f, t, engine=7)
    with pytest.raises(RuntimeError, match="HCG_EINVAL"):
        f.split_spectra(api.ENGINE_FP32)
    ref, _ = ctx.grid(f, t, engine=api.ENGINE_TC_BF16)
    # dropping the FP32 copy keeps the tensor-core result and closes the FP32 engine
    f.split_spectra(api.ENGINE_TC_BF16, keep_fp32=False)
    again, _ = ctx.grid(f, t)
    np.testing.assert_array_equal(ref, again)
    with pytest.raises(RuntimeError, match="HCG_ESTATE"):
        ctx.grid(f, t, engine=api.ENGINE_FP32)
    # new spectra drop the split; non-finite values are refused by the tensor-core engines
    bad = job.values.copy()
    bad[::50, 3] = np.nan
    f.set_spectra(bad)
    with pytest.raises(RuntimeError, match="HCG_ESTATE"):
        ctx.grid(f, t, engine=api.ENGINE_TC_BF16)
    f.split_spectra(api.ENGINE_TC_BF16)
    with pytest.raises(RuntimeError, match="HCG_EINVAL"):
        ctx.grid(f, t, engine=api.ENGINE_TC_BF16)
    c32, _ = ctx.grid(f, t, engine=api.ENGINE_FP32)  # the FP32 engine grids them
    assert np.isnan(c32[:, 3]).any()


def test_pipeline_shapes_and_autotune(ctx, small):
    """Every tensor-core pipeline shape (256 channels x 64-sample chunks x 2
    stages, 128 x 64 x 3, 64 x 64 x 4, 256 x 32 x 4) gives the same weights
    and stays within tolerance of the oracle; the autotuner times them and
    keeps one."""
    job, f, t, ref, c32, w32 = small
    prepare(ctx, job)
    f.split_spectra(api.ENGINE_TC_F16)
    outs = []
    try:
        for cfg in range(6):
            ctx.tc_set_config(cfg)
            c, w = ctx.grid(f, t, engine=api.ENGINE_TC_F16)
            np.testing.assert_array_equal(w, w32)
            err = plane_errors(c, ref)
            print(f"pipeline shape {cfg}: max plane-relative error {err:.3e}")
            assert err <= TOL[api.ENGINE_TC_F16]
            outs.append(c)
        ctx.tc_set_config(-1)
        best, ms = ctx.autotune(f, t, reps=1)
        print("autotune", best, ms)
        assert best in range(6) and all(m > 0 for m in ms)
        # timed in channel-plane cubes: the choice is still a valid shape and grids within tolerance
        ctx.autotune_layout(api.CHANNEL_MAJOR)
        best, ms = ctx.autotune(f, t, reps=1)
        print("autotune (channel planes)", best, ms)
        assert best in range(6) and all(m > 0 for m in ms)
        c, w = ctx.grid(f, t, engine=api.ENGINE_TC_F16, layout=api.CHANNEL_MAJOR)
        np.testing.assert_array_equal(w, w32)
        assert plane_errors(np.ascontiguousarray(c.T), ref) <= TOL[api.ENGINE_TC_F16]
        with pytest.raises(RuntimeError, match="HCG_EINVAL"):
            ctx.tc_set_config(6)
        with pytest.raises(RuntimeError, match="HCG_EINVAL"):
            ctx.autotune_layout(7)
    finally:
        ctx.tc_set_config(-1)
        ctx.autotune_layout(api.SAMPLE_MAJOR)


def test_coarse_pixels_many_rings(ctx):
    """Pixels 12x the kernel (64x64 map over 13 deg, FWHM 60"): a tile's ring
    span exceeds a thousand HEALPix rings but few of them hold candidates;
    the compacted tile table keeps the tensor-core and FP32 tile engines on."""
    shape = dict(block=0, n=26_206, size_deg=13.016, ra=154.57, dec=7.25, grid=64, nchan=64, fwhm=60.0, seed=5)
    job = synth.block_job(shape)
    prepare(ctx, job)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(np.ascontiguousarray(job.values.reshape(job.n, -1)))
    f.nchan = job.nchan
    t = ctx.target_from_header(job.header)
    c32, w32 = ctx.grid(f, t, engine=api.ENGINE_FP32)
    f.split_spectra(api.ENGINE_TC_F16, keep_fp32=False)
    ct, wt = ctx.grid(f, t)
    np.testing.assert_array_equal(wt, w32)
    assert plane_errors(ct, c32.astype(np.float64)) <= 1e-5


def test_config3_precision_subcube(ctx):
    """The precision form (config 3) at reduced size: the config-2 generator
    (same sample density, 60" pixels) with 4,096 channels, BF16 hi/lo
    spectra with per-channel scales; the relative error of a 256 x 256 x 64
    sub-cube (central pixels, 64 channels across the band) against the FP64
    oracle stays within the BF16 tolerance, and the FP16 split within 1e-5."""
    torch = pytest.importorskip("torch")
    job = synth.config2(n=600_000, nchan=4096, nx=464, size_deg=7.75)
    prepare(ctx, job)
    G, L, noise = job.factors
    dev = torch.device("cuda", 0)
    gen = torch.Generator(device=dev)
    gen.manual_seed(job.seed)
    S = torch.empty((job.n, job.nchan), dtype=torch.float32, device=dev)
    Ld = torch.from_numpy(L).to(dev)
    for i in range(0, job.n, 1 << 17):
        Gd = torch.from_numpy(G[i:i + (1 << 17)]).to(dev)
        torch.matmul(Gd, Ld, out=S[i:i + (1 << 17)])
        S[i:i + (1 << 17)].add_(torch.randn((Gd.shape[0], job.nchan), generator=gen, device=dev), alpha=noise)
    chans = np.linspace(0, job.nchan - 1, 64).round().astype(np.int64)
    vals = S[:, torch.from_numpy(chans).to(dev)].double().cpu().numpy()
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(S)
    del S
    t = ctx.target_from_header(job.header)
    xw, yw = t.coords()
    y0 = x0 = (464 - 256) // 2
    sub = (np.arange(256)[:, None] + y0) * 464 + (np.arange(256)[None, :] + x0)
    sub = sub.reshape(-1)
    g = O.prepare_grid_kernel(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    ps = O.presort(g.hpx, job.lon, job.lat)
    oc, ow, _ = O.grid(g, ps, job.lon[ps.perm], job.lat[ps.perm], vals[ps.perm], xw[sub], yw[sub])
    ref = oc / ow[:, None]
    P = 464 * 464
    errs = {}
    for engine in (api.ENGINE_TC_BF16, api.ENGINE_TC_F16):
        f.split_spectra(engine)
        cube = torch.empty((P, job.nchan), dtype=torch.float32, device=dev)
        w = torch.empty(P, dtype=torch.float32, device=dev)
        ctx.grid(f, t, cube, w, engine=engine)
        got = cube[torch.from_numpy(sub).to(dev)][:, torch.from_numpy(chans).to(dev)].cpu().numpy()
        errs[engine] = plane_errors(got, ref)
        ok = ow > 0
        assert np.abs(w[torch.from_numpy(sub).to(dev)].cpu().numpy()[ok] - ow[ok]).max() / ow.max() <= 1e-6
        del cube
    print("config-3 sub-cube max plane-relative error: bf16 %.3e, f16 %.3e"
          % (errs[api.ENGINE_TC_BF16], errs[api.ENGINE_TC_F16]))
    assert errs[api.ENGINE_TC_BF16] <= TOL[api.ENGINE_TC_BF16]
    assert errs[api.ENGINE_TC_F16] <= TOL[api.ENGINE_TC_F16]
    f.close()
    t.close()


def test_config2_full_size_subcube(ctx):
    """The headline workload at its full size (config 2: 4,000,000 samples x
    1,024 channels onto 1200 x 1200 pixels): the tensor-core cube (FP16
    hi/lo, the pipeline shape the engine picks for this size, accumulation
    segments, entry runs) and the FP32 engine's cube on the central 64 x 64
    pixels x 16 channels spread over the band, against the FP64 oracle."""
    torch = pytest.importorskip("torch")
    job = synth.config2()
    assert (job.n, job.nchan, job.nx, job.ny) == (4_000_000, 1024, 1200, 1200)
    prepare(ctx, job)
    G, L, noise = job.factors
    dev = torch.device("cuda", 0)
    gen = torch.Generator(device=dev)
    gen.manual_seed(job.seed)
    S = torch.empty((job.n, job.nchan), dtype=torch.float32, device=dev)
    Ld = torch.from_numpy(L).to(dev)
    for i in range(0, job.n, 1 << 18):
        Gd = torch.from_numpy(G[i:i + (1 << 18)]).to(dev)
        torch.matmul(Gd, Ld, out=S[i:i + (1 << 18)])
        S[i:i + (1 << 18)].add_(torch.randn((Gd.shape[0], job.nchan), generator=gen, device=dev), alpha=noise)
    chans = np.linspace(0, job.nchan - 1, 16).round().astype(np.int64)
    vals = S[:, torch.from_numpy(chans).to(dev)].double().cpu().numpy()
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(S)
    del S
    t = ctx.target_from_header(job.header)
    xw, yw = t.coords()
    y0 = x0 = (1200 - 64) // 2
    sub = ((np.arange(64)[:, None] + y0) * 1200 + (np.arange(64)[None, :] + x0)).reshape(-1)
    g = O.prepare_grid_kernel(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    ps = O.presort(g.hpx, job.lon, job.lat)
    oc, ow, _ = O.grid(g, ps, job.lon[ps.perm], job.lat[ps.perm], vals[ps.perm], xw[sub], yw[sub])
    ref = oc / ow[:, None]
    P = 1200 * 1200
    sub_d, chans_d = torch.from_numpy(sub).to(dev), torch.from_numpy(chans).to(dev)
    errs = {}
    f.split_spectra(api.ENGINE_TC_F16)
    for engine in (api.ENGINE_TC_F16, api.ENGINE_FP32):
        cube = torch.empty((P, job.nchan), dtype=torch.float32, device=dev)
        w = torch.empty(P, dtype=torch.float32, device=dev)
        ctx.grid(f, t, cube, w, engine=engine)
        got = cube[sub_d][:, chans_d].cpu().numpy()
        errs[engine] = plane_errors(got, ref)
        ok = ow > 0
        assert np.abs(w[sub_d].cpu().numpy()[ok] - ow[ok]).max() / ow.max() <= 1e-6
        del cube
    print("config-2 full size, 64x64x16 sub-cube max plane-relative error: tc f16 %.3e, fp32 %.3e"
          % (errs[api.ENGINE_TC_F16], errs[api.ENGINE_FP32]))
    assert errs[api.ENGINE_TC_F16] <= TOL[api.ENGINE_TC_F16]
    assert errs[api.ENGINE_FP32] <= 1e-5
    f.close()
    t.close()
