"""hcg_grid_noalloc: single-channel gridding whose scratch is a fixed array
inside the library. It is for callers that cannot allocate device memory at
the time they grid: a real-time pipeline that reserved all its device memory
when it started, or a host application whose own allocator holds the GPU's
memory and lends the library only inputs and outputs.

Called through the C ABI on a fresh context that has never run hcg_grid (so
the context's growable scratch pool is still empty), twice in a row on two
different jobs; device memory must not move across either call. The cubes and
weight maps are then checked against hcg_grid's, within the single-channel
tolerance the parity tests use (1e-6 relative, identical NaN pattern); both
entry points run the same arithmetic.

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


def _job(ctx, n, nx, seed):
    job = synth.config1(n=n, nx=nx, seed=seed)
    ctx.prepare_grid_kernel(api.GAUSS1D, np.array([job.sigma_deg, 0.0, 0.0]), job.sphere_radius, job.hpx_max_res)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    t = ctx.target_from_header(job.header)
    return f, t


def _noalloc(ctx, f, t, cube, w):
    return ctx.L.hcg_grid_noalloc(ctx.h, f.h, t.h, C.c_void_p(cube.data_ptr()),
                                  C.c_void_p(w.data_ptr()) if w is not None else None)


def test_noalloc_allocates_nothing_and_matches_hcg_grid_on_two_calls():
    # A first call on another context loads the library's module on this
    # device and looks up the scratch array's address (the once-per-device set-up).
    warm = api.Context(0)
    fw, tw = _job(warm, 20_000, 32, 7)
    cw = torch.empty(32 * 32, dtype=torch.float32, device="cuda")
    assert _noalloc(warm, fw, tw, cw, None) == 0, warm.L.hcg_last_error(warm.h)
    warm.synchronize()

    ctx = api.Context(0)  # never runs hcg_grid before the checks below
    jobs = [_job(ctx, 40_000, 96, 5), _job(ctx, 60_000, 128, 6)]
    outs = []
    for f, t in jobs:
        P = t.nx * t.ny
        outs.append((torch.full((P,), float("inf"), dtype=torch.float32, device="cuda"),
                     torch.full((P,), float("inf"), dtype=torch.float32, device="cuda")))
    ctx.synchronize()
    torch.cuda.synchronize()
    free = [torch.cuda.mem_get_info()[0]]
    for (f, t), (cube, w) in zip(jobs, outs):
        # the kernel setup of each field travels with the field
        st = _noalloc(ctx, f, t, cube, w)
        assert st == 0, ctx.L.hcg_last_error(ctx.h)
        ctx.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
    assert free[1] == free[0] and free[2] == free[0], "device memory moved across hcg_grid_noalloc: %s" % free
    for (f, t), (cube, w) in zip(jobs, outs):
        ref_cube, ref_w = ctx.grid(f, t)  # the existing entry point
        close(cube.cpu().numpy(), ref_cube[:, 0])
        close(w.cpu().numpy(), ref_w)
    for f, t in jobs + [(fw, tw)]:
        f.close()
        t.close()
    ctx.close()
    warm.close()


def test_noalloc_rejects_targets_beyond_its_scratch_and_host_outputs():
    ctx = api.Context(0)
    f, _ = _job(ctx, 20_000, 32, 7)
    big = 400  # 160000 pixels > 131072
    t = ctx.target(big, big, np.full(big * big, 30.0), np.full(big * big, 40.0))
    cube = torch.empty(big * big, dtype=torch.float32, device="cuda")
    st = _noalloc(ctx, f, t, cube, None)
    assert st == 1 and b"at most 131072" in ctx.L.hcg_last_error(ctx.h)
    small = ctx.target(8, 8, np.full(64, 30.0), np.full(64, 40.0))
    host = np.zeros(64, np.float32)  # pageable host memory: refused before any launch
    st = ctx.L.hcg_grid_noalloc(ctx.h, f.h, small.h, host.ctypes.data_as(C.c_void_p), None)
    assert st == 1 and b"device buffers" in ctx.L.hcg_last_error(ctx.h)
    f.close()
    t.close()
    small.close()
    ctx.close()
