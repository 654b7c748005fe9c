"""Dec-band sharding of one gridding job over ranks, one GPU each.

Output pixels are independent, so a job shards by bands of target rows with
no reduction: each rank grids its rows from the samples they need, a
contiguous range of the ring-sorted samples (hcg_field_band_samples), and
rank 0 assembles the band slabs. Band edges fall on multiples of 16 rows
(the tensor-core tiles are 8 rows high, the weight-pass groups 2), so every
band's tiles are tiles of the whole map.

    bands = plan(ny, world)
    geo = ctx.field(lon, lat)                       # positions only: the sort
    cube_rows, w_rows = grid_band(ctx, geo, target, lon, lat, values, *bands[rank])
    cube, w = assemble(dist, rank, world, bands, nx, cube_rows, w_rows)   # rank 0

No reference counterpart: HCGrid runs one job per GPU.
"""
from __future__ import annotations

import numpy as np

from . import api

ALIGN = 16


def plan(ny: int, parts: int, align: int = ALIGN):
    """[y0, y1) rows of `parts` contiguous bands covering [0, ny), edges on
    multiples of `align`, sizes as equal as the alignment allows (trailing
    bands may be empty when ny is small)."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    units = (ny + align - 1) // align
    out = []
    for r in range(parts):
        u0, u1 = units * r // parts, units * (r + 1) // parts
        out.append((min(ny, u0 * align), min(ny, u1 * align)))
    return out


def grid_band(ctx: api.Context, geometry: api.Field, target: api.Target, lon, lat, values, y0: int, y1: int,
              weights=None, engine: int = api.ENGINE_AUTO, perm=None):
    """Rows [y0, y1) of `target`, gridded from the samples they need.

    geometry: a field of all the job's samples made under the job's kernel
    setup (spectra not needed); values: [n] or [n, C] float32, sample-major.
    engine: ENGINE_TC_F16 / ENGINE_TC_BF16 split the band's spectra for the
    tensor cores. Returns (cube [(y1 - y0) * nx, C], weights [(y1 - y0) * nx]).
    """
    nx = target.nx
    values = np.asarray(values, np.float32)
    nchan = 1 if values.ndim == 1 else values.shape[1]
    npix = (y1 - y0) * nx
    s0, s1 = geometry.band_samples(target, y0, y1)
    if s1 == s0:  # no sample within reach: empty pixels, as the gridder leaves them (0/0)
        return np.full((npix, nchan), np.nan, np.float32), np.zeros(npix, np.float32)
    if perm is None:
        perm = geometry.sorted()[1]
    idx = perm[s0:s1]
    f = ctx.field(np.ascontiguousarray(lon[idx]), np.ascontiguousarray(lat[idx]),
                  None if weights is None else np.ascontiguousarray(np.asarray(weights)[idx]))
    try:
        f.set_spectra(np.ascontiguousarray(values[idx]))
        if engine in (api.ENGINE_TC_F16, api.ENGINE_TC_BF16) and nchan > 1:
            f.split_spectra(engine, keep_fp32=False)
        xw, yw = target.coords()
        p0, p1 = y0 * nx, y1 * nx
        bt = ctx.target(nx, y1 - y0, np.ascontiguousarray(xw[p0:p1]), np.ascontiguousarray(yw[p0:p1]))
        try:
            cube, w = ctx.grid(f, bt, engine=engine)
        finally:
            bt.close()
    finally:
        f.close()
    return cube.reshape(npix, nchan), w


def assemble(dist, rank: int, world: int, bands, nx: int, cube_rows, w_rows):
    """Rank 0 gathers every rank's band slab into the whole cube [ny * nx, C]
    and weight map; the other ranks return (None, None). `dist` is
    torch.distributed (any backend) or None for a single rank."""
    if dist is None or world == 1:
        return cube_rows, w_rows
    got = [None] * world if rank == 0 else None
    dist.gather_object((cube_rows, w_rows), got, dst=0)
    if rank != 0:
        return None, None
    ny = bands[-1][1]
    nchan = cube_rows.shape[1]
    cube = np.empty((ny * nx, nchan), np.float32)
    w = np.empty(ny * nx, np.float32)
    for (y0, y1), (c, ww) in zip(bands, got):
        cube[y0 * nx:y1 * nx] = c
        w[y0 * nx:y1 * nx] = ww
    return cube, w


def assemble_tensors(dist, rank: int, world: int, bands, nx: int, cube_rows, w_rows):
    """assemble() for torch tensors: rank 0 receives every band slab through
    one torch.distributed gather (NCCL keeps CUDA tensors on the device; any
    backend works for CPU tensors). Slabs are padded to the largest band so
    the gather moves equal sizes. Returns the whole cube [ny * nx, C] and
    weight map on rank 0, (None, None) elsewhere."""
    import torch
    if dist is None or world == 1:
        return cube_rows, w_rows
    nchan = cube_rows.shape[1]
    rows = max(y1 - y0 for y0, y1 in bands) * nx
    slab = torch.zeros((rows, nchan + 1), dtype=cube_rows.dtype, device=cube_rows.device)
    n = cube_rows.shape[0]
    slab[:n, :nchan] = cube_rows
    slab[:n, nchan] = w_rows
    got = [torch.empty_like(slab) for _ in range(world)] if rank == 0 else None
    dist.gather(slab, got, dst=0)
    if rank != 0:
        return None, None
    ny = bands[-1][1]
    cube = torch.empty((ny * nx, nchan), dtype=cube_rows.dtype, device=cube_rows.device)
    w = torch.empty(ny * nx, dtype=cube_rows.dtype, device=cube_rows.device)
    for (y0, y1), g in zip(bands, got):
        k = (y1 - y0) * nx
        cube[y0 * nx:y1 * nx] = g[:k, :nchan]
        w[y0 * nx:y1 * nx] = g[:k, nchan]
    return cube, w


def band_field(ctx: api.Context, geometry: api.Field, target: api.Target, lon, lat, y0: int, y1: int, perm=None):
    """The samples rows [y0, y1) of `target` need: (field of those samples in
    sorted order, their input indices, the band's target). The field is
    created from host coordinates of that range only; spectra are attached
    by the caller (values[idx])."""
    s0, s1 = geometry.band_samples(target, y0, y1)
    if perm is None:
        perm = geometry.sorted()[1]
    idx = perm[s0:s1]
    nx = target.nx
    xw, yw = target.coords()
    p0, p1 = y0 * nx, y1 * nx
    bt = ctx.target(nx, y1 - y0, np.ascontiguousarray(xw[p0:p1]), np.ascontiguousarray(yw[p0:p1]))
    if s1 == s0:
        return None, idx, bt
    f = ctx.field(np.ascontiguousarray(lon[idx]), np.ascontiguousarray(lat[idx]))
    return f, idx, bt
