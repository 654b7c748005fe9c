"""hcg_grid_noalloc: single-channel gridding whose scratch is a fixed array
inside the library, for callers that cannot allocate device memory when they
grid (a real-time pipeline that reserved its memory at start-up, or code
inside an open stream capture). Called through the C ABI and checked against
hcg_grid on two calls in a row, within the single-channel tolerance the
parity tests use (1e-6 relative, identical NaN pattern); both entry points
run the same arithmetic, so the results are expected to be identical.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from hcgrid_b200 import api, synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL = 1e-6
MAX_PIXELS = 131072


def close(a, b):
    assert np.array_equal(np.isnan(a), np.isnan(b))
    ok = ~np.isnan(b)
    assert np.abs(a[ok] - b[ok]).max() <= TOL * np.abs(b[ok]).max()


def test_noalloc_matches_hcg_grid_on_two_calls():
    ctx = api.Context(0)
    L = ctx.L
    results = []
    for nx, n, seed in ((96, 40_000, 5), (128, 60_000, 6)):
        job = synth.config1(n=n, nx=nx, seed=seed)
        kp = np.array([job.sigma_deg, 0.0, 0.0])
        ctx.prepare_grid_kernel(api.GAUSS1D, kp, job.sphere_radius, job.hpx_max_res)
        f = ctx.field(job.lon, job.lat)
        f.set_spectra(job.values)
        t = ctx.target_from_header(job.header)
        ref_cube, ref_w = ctx.grid(f, t)          # existing entry point
        P = t.nx * t.ny
        cube = torch.full((P,), float("inf"), dtype=torch.float32, device="cuda")
        w = torch.full((P,), float("inf"), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st = L.hcg_grid_noalloc(ctx.h, f.h, t.h, C.c_void_p(cube.data_ptr()), C.c_void_p(w.data_ptr()))
        assert st == 0, L.hcg_last_error(ctx.h)
        ctx.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        results.append((cube.cpu().numpy(), w.cpu().numpy(), ref_cube[:, 0], ref_w, free_before - free_after))
    for got_c, got_w, ref_c, ref_w, _ in results:
        close(got_c, ref_c)
        close(got_w, ref_w)
    # the second call found the scratch set up and took no device memory
    assert results[1][4] == 0
    ctx.close()


def test_noalloc_rejects_targets_beyond_its_scratch():
    ctx = api.Context(0)
    job = synth.config1(n=20_000, nx=32, seed=7)
    kp = np.array([job.sigma_deg, 0.0, 0.0])
    ctx.prepare_grid_kernel(api.GAUSS1D, kp, job.sphere_radius, job.hpx_max_res)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    big = 400  # 160000 pixels > 131072
    t = ctx.target(big, big, np.full(big * big, 30.0), np.full(big * big, 40.0))
    cube = torch.empty(big * big, dtype=torch.float32, device="cuda")
    st = ctx.L.hcg_grid_noalloc(ctx.h, f.h, t.h, C.c_void_p(cube.data_ptr()), None)
    assert st == 1 and b"at most 131072" in ctx.L.hcg_last_error(ctx.h)
    ctx.close()
