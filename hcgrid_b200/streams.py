"""Request streams of the batched (config 4) and served (config 5) forms.

A stream is a list of requests ``{request, field, shape, spectra_seed}``: a
request grids a scan block of ``shape`` (the config-4 shape dictionary of
hcgrid_b200/synth.py) with spectra drawn from ``spectra_seed``, on the
samples of field ``field`` (several requests may share a field: new spectra
on known sample positions). On one GPU the stream is staged in windows that
fit a device-memory budget; each request's spectra are generated on the
device, attached to a share of its field (hcg_field_share, so the sort and
ring tables are reused), split for the tensor cores when asked, and given
device output buffers. The runner then grids a window one request at a time
(hcg_grid), as one batch (hcg_grid_batch), or through a server
(hcg_server); only the gridding is timed by the callers.

Fields and targets are built when a request first needs them and are closed
after the last request that uses them, so reuse never rebuilds a sort and
the resident set stays bounded."""
from __future__ import annotations

import numpy as np

from . import api, synth


def request_work(r: dict) -> int:
    """Sample-channels of one request (the metric's unit)."""
    return r["shape"]["n"] * r["shape"]["nchan"]


def fills_gpu(shape: dict, nsm: int = 148) -> bool:
    """The server's large jobs (run alone, as one hcg_grid each): 2^20 target
    pixels or more, or a multi-channel job with at least one channel-sum item
    (16 x 8-pixel tile, 256-channel block) per SM."""
    g = shape["grid"]
    if g * g >= 1 << 20:
        return True
    if shape["nchan"] <= 1:
        return False
    return ((g + 15) // 16) * ((g + 7) // 8) * ((shape["nchan"] + 255) // 256) >= nsm


def footprint(shape: dict) -> int:
    """Device bytes of one staged request: FP32 spectra while they are
    attached, the 16-bit hi/lo split, cube, weight map and the per-pixel
    scratch of the gridding engines (pixel setup, weight sums, tile tables,
    entries)."""
    P = shape["grid"] ** 2
    return 2 * shape["n"] * shape["nchan"] * 4 + P * (shape["nchan"] + 1) * 4 + P * 600


def plan_windows(reqs: list, budget: int) -> list:
    """Consecutive runs of requests whose footprints fit `budget` (a request
    larger than the budget gets a window of its own)."""
    windows, cur, used = [], [], 0
    for r in reqs:
        fp = footprint(r["shape"])
        if cur and used + fp > budget:
            windows.append(cur)
            cur, used = [], 0
        cur.append(r)
        used += fp
    if cur:
        windows.append(cur)
    return windows


def last_use(reqs: list) -> dict:
    """Index (in stream order) of the last request of each field."""
    out = {}
    for i, r in enumerate(reqs):
        out[r["field"]] = i
    return out


def block_spectra(lon_d, lat_d, shape: dict, seed: int, torch, dev):
    """[n][nchan] float32 spectra of one request on the device: 20 Gaussian
    sources of the block's field with seeded line profiles (a continuum
    value with a 1 K offset for single-channel blocks), plus N(0, 0.05)."""
    nchan = shape["nchan"]
    rng = np.random.default_rng(seed)
    src = synth.make_sources(20, shape["ra"], shape["dec"], shape["size_deg"], rng)
    ra = torch.tensor(src.ra, device=dev)
    dec = torch.tensor(src.dec, device=dev)
    amp = torch.tensor(src.amp, device=dev)
    sig = torch.tensor(src.sigma_deg, device=dev)
    if nchan == 1:
        L = torch.ones((len(src.amp), 1), device=dev, dtype=torch.float32)
    else:
        c0 = rng.uniform(0.1, 0.9, len(src.amp)) * nchan
        w = rng.uniform(0.01, 0.05, len(src.amp)) * nchan
        ch = np.arange(nchan)
        L = torch.tensor(np.exp(-((ch[None, :] - c0[:, None]) ** 2) / (2.0 * w[:, None] ** 2)), device=dev,
                         dtype=torch.float32)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    n = lon_d.shape[0]
    S = torch.empty((n, nchan), dtype=torch.float32, device=dev)
    step = max(1, (1 << 26) // max(nchan, 1))
    for i in range(0, n, step):
        lo, la = lon_d[i:i + step, None], lat_d[i:i + step, None]
        dx = torch.remainder(lo - ra[None, :] + 180.0, 360.0) - 180.0
        dx = dx * torch.cos(torch.deg2rad(dec))[None, :]
        dy = la - dec[None, :]
        G = (amp[None, :] * torch.exp(-(dx * dx + dy * dy) / (2.0 * sig[None, :] ** 2))).float()
        torch.matmul(G, L, out=S[i:i + step])
        if nchan == 1:
            S[i:i + step].add_(1.0)
        S[i:i + step].add_(torch.randn((G.shape[0], nchan), generator=gen, device=dev), alpha=0.05)
    return S


def check_channels(nchan: int, k: int = 3) -> np.ndarray:
    """Up to k channels spread over the band (the checked columns)."""
    return np.unique(np.linspace(0, nchan - 1, min(k, nchan)).round().astype(np.int64))


class Staged:
    """One staged request: its field share (with spectra), target, device
    cube [pixels][channels] and weight map; `cols` holds the spectra of the
    checked channels (host, input order) when the request is checked."""

    def __init__(self, r, field, target, cube, weights, cols=None):
        self.r, self.field, self.target, self.cube, self.weights, self.cols = r, field, target, cube, weights, cols


class Runner:
    """Resident fields and targets of a stream on one context, and the
    staging of its windows."""

    def __init__(self, ctx: api.Context, reqs: list, torch, dev):
        self.ctx, self.reqs, self.torch, self.dev = ctx, reqs, torch, dev
        self.last = last_use(reqs)
        self.pos = {r["request"]: i for i, r in enumerate(reqs)}
        self.fields = {}  # field id -> (Field, Target, lon_d, lat_d)
        self.built = 0

    def field(self, r: dict):
        fid = r["field"]
        if fid not in self.fields:
            sh = r["shape"]
            rng = np.random.default_rng(sh["seed"])
            lon, lat = synth.raster_scan(sh["n"], sh["ra"], sh["dec"], sh["size_deg"], 2.0, rng)
            sigma = sh["fwhm"] / 3600.0 * synth.FWHM_TO_SIGMA
            self.ctx.prepare_grid_kernel(api.GAUSS1D, np.array([sigma, 0.0, 0.0]), 3.0 * sigma, sigma / 2.0)
            f = self.ctx.field(lon, lat)
            hdr = synth.sin_header(sh["grid"], sh["grid"], sh["ra"], sh["dec"], sh["size_deg"] / sh["grid"])
            t = self.ctx.target_from_header(hdr)
            self.fields[fid] = (f, t, self.torch.from_numpy(lon).to(self.dev), self.torch.from_numpy(lat).to(self.dev))
            self.built += 1
        return self.fields[fid]

    def release_done(self, upto: int):
        """Close the fields whose last request is at or before stream index `upto`."""
        for fid in [k for k in self.fields if self.last[k] <= upto]:
            f, t, _, _ = self.fields.pop(fid)
            f.close()
            t.close()

    def stage(self, win: list, tc: bool, keep=()) -> list:
        """Stage the requests of `win`; for requests in `keep`, the spectra of
        the checked channels are copied to the host (Staged.cols)."""
        out = []
        for r in win:
            sh = r["shape"]
            f0, t, lon_d, lat_d = self.field(r)
            S = block_spectra(lon_d, lat_d, sh, r["spectra_seed"], self.torch, self.dev)
            self.torch.cuda.synchronize(self.dev)
            cols = None
            if r["request"] in keep:
                ch = self.torch.from_numpy(check_channels(sh["nchan"])).to(self.dev)
                cols = S.index_select(1, ch).double().cpu().numpy()
            f = f0.share()
            f.set_spectra(S)
            del S
            if tc and sh["nchan"] > 1:
                f.split_spectra(api.ENGINE_TC_F16, keep_fp32=False)
            P = t.nx * t.ny
            cube = self.torch.empty((P * sh["nchan"],), dtype=self.torch.float32, device=self.dev)
            wts = self.torch.empty((P,), dtype=self.torch.float32, device=self.dev)
            out.append(Staged(r, f, t, cube, wts, cols))
        self.ctx.synchronize()
        return out

    def unstage(self, staged: list):
        last = max(self.pos[s.r["request"]] for s in staged) if staged else -1
        for s in staged:
            s.field.close()
        staged.clear()
        self.ctx.synchronize()
        self.release_done(last)
        self.ctx.trim()
        self.torch.cuda.empty_cache()

    def close(self):
        self.release_done(len(self.reqs))
