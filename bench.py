#!/usr/bin/env python
"""Benchmark of the B200 gridder on the reference's headline workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload config2|config1|config3|config4|config5] [--served-jobs J]
                    [--shard bands|replicas]

A step is one gridding pass (hcg_grid: pixel setup, candidate selection,
FP64 weights, channel sums, normalisation) over the resident field of the
workload: config 2 = 4,000,000 raster-scan samples x 1,024 float32 channels
onto a 1200x1200 SIN grid, GAUSS1D FWHM 180" (seeded synthetic data, see
hcgrid_b200/synth.py). `value` is gridded sample-channels/s with inputs
resident in HBM; `e2e` repeats the metric through the C ABI from pinned
host buffers (field creation with the on-device sort, then hcg_grid_planes:
the spectra as channel planes uploaded, split and gridded block by block with
the cube downloaded as blocks finish). Inputs are larger than L2 (16 GB of
spectra), so no flush.

At N=1 the config-2 line also carries `served_config5`: the served form
(config 5, a stream of J gridding requests through hcg_server, timed against
the plain FP32 engine and the tensor-core engine per call on the same
requests; `--workload config5` prints its full record).

Multi-GPU (torchrun): with --shard bands (the default) the one job is split
into Dec bands of target rows, one per rank; each rank grids its band from
the contiguous range of ring-sorted samples the band needs (strong scaling,
no collective in the timed steps) and rank 0 then gathers the band slabs
(NCCL, timed apart as `assemble_ms`). With --shard replicas every rank grids
its own copy of the job (weak scaling). Timings are the max over ranks.

--impl reference times the reference's own CPU path (oracle/_ref: HCGrid's
host pre-sort plus its kernel body built for the host cores) on a bounded
sample of the same workload and extrapolates to the whole job.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC = os.path.join(ROOT, "profiles", "traffic.json")
METRIC = "gridded sample-channels/s"
UNIT = "sample-channels/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="config2", choices=["config2", "config1", "config3", "config4", "config5"])
    ap.add_argument("--jobs", type=int, default=2000, help="config5: requests in the stream (the full form's 2000)")
    ap.add_argument("--blocks", type=int, default=256, help="config4: scan blocks (the full form's 256)")
    ap.add_argument("--stage-gb", type=float, default=48.0,
                    help="config4/config5: device bytes of requests staged at once (a window)")
    ap.add_argument("--oracle-checks", type=int, default=1,
                    help="config5: check sampled requests against the FP64 oracle in the CPU leg (0: skip)")
    ap.add_argument("--hbm-budget-gb", type=float, default=120.0, help="config5: admission budget")
    ap.add_argument("--lanes", type=int, default=1, help="config5: server lanes")
    ap.add_argument("--layout", default="channel", choices=["channel", "sample"],
                    help="cube layout of the config-1/2/3 steps: channel = [channel][pixel], the reference's "
                         "h_datacube planes; sample = [pixel][channel]")
    ap.add_argument("--detail", default=None, help="config5: write per-window times of the served and per-call arms here")
    ap.add_argument("--tc-weights", default="auto", choices=["auto", "entries", "direct"],
                    help="tensor-core weight operands (hcg_tc_set_weights)")
    ap.add_argument("--served-jobs", type=int, default=200,
                    help="config2 at N=1: also run the served form (config5) on this many requests and report it "
                         "under 'served_config5' (0: skip)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--plane-block", type=int, default=0,
                    help="end to end: channels per block of hcg_grid_planes (a multiple of 64; 0: the "
                         "library's 64)")
    ap.add_argument("--shard", default="bands", choices=["bands", "replicas"],
                    help="N>1: split the one job into Dec bands of target rows, one per rank, gathered to rank 0 "
                         "over NCCL (strong scaling), or grid a replica of the whole job on every rank (weak)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-check", action="store_true",
                    help="skip the check of the timed cube against the FP64 oracle and the FP32 engine")
    ap.add_argument("--engine", default=None, choices=list(ENGINES),
                    help="channel-sum engine: tensor cores with a 16-bit hi/lo split, or FP32 CUDA cores "
                         "(default: tc-bf16 for config3, tc-f16 otherwise)")
    ap.add_argument("--plain-steps", type=int, default=2,
                    help="also time this many steps of the plain FP32 engine on the same field (0: skip)")
    ap.add_argument("--tc-prefetch", type=int, default=-1, help="with --tc-config: prefetch distance (chunks)")
    ap.add_argument("--tc-strip", type=int, default=-1, help="with --tc-config: persistent tile walk strip width")
    ap.add_argument("--tune-reps", type=int, default=3, help="timed runs per autotuner setting")
    ap.add_argument("--batch-shape", type=int, default=None, choices=[0, 1, 2, 3],
                    help="config4: the batch pass's tensor-core shape for every channel class (default: "
                         "hcg_autotune_batch on the first window)")
    ap.add_argument("--tc-config", type=int, default=None,
                    help="tensor-core pipeline shape (0: 256 ch x 64-sample chunks x 2 stages, 1: 128 x 64 x 3, "
                         "2: 64 x 64 x 4, 3: 256 x 32 x 4, 4/5: 0/3 persistent); "
                         "default: autotuned on the workload before the timed steps")
    # reduced cases (profiling, quick checks); the headline run uses none of these
    ap.add_argument("--samples", type=int, default=None)
    ap.add_argument("--channels", type=int, default=None)
    ap.add_argument("--pixels-x", type=int, default=None)
    ap.add_argument("--field-deg", type=float, default=None)
    args = ap.parse_args()
    if args.engine is None:
        args.engine = "tc-bf16" if args.workload == "config3" else "tc-f16"
    if args.workload == "config3" and "--e2e-steps" not in sys.argv:
        args.e2e_steps = 0  # 65 GB of host spectra: the e2e leg is the config-2 line's
    return args


ENGINES = {"fp32": 1, "tc-f16": 3, "tc-bf16": 2}
DTYPE_TEXT = {"fp32": "f32 (FP64 geometry)",
              "tc-f16": "f16 hi/lo x3, f32 accumulate (FP64 geometry)",
              "tc-bf16": "bf16 hi/lo x3, f32 accumulate (FP64 geometry)"}
ENGINE_TEXT = {"fp32": "FP32 CUDA-core channel sums, FP64 geometry",
               "tc-f16": "tcgen05 channel sums, compensated FP16 hi/lo (3 products, FP32 accumulate), FP64 geometry",
               "tc-bf16": "tcgen05 channel sums, compensated BF16 hi/lo (3 products, FP32 accumulate), FP64 geometry"}


def peaks():
    try:
        d = json.load(open(MEASURED))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def tensor_peak():
    """Dense bf16 TFLOP/s (f16 runs at the same rate): the burst figure, for
    a kernel timed on its own."""
    try:
        d = json.load(open(MEASURED))
        return float(d["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


# ---------------------------------------------------------------------------
# workload

def job_for(args):
    from hcgrid_b200 import synth
    kw = {}
    if args.samples:
        kw["n"] = args.samples
    if args.pixels_x:
        kw["nx"] = args.pixels_x
    if args.workload == "config1":
        return synth.config1(**kw)
    if args.workload == "config3":
        kw["nchan"] = 4096  # the precision form: config-2 geometry, 4,096 channels
    if args.channels:
        kw["nchan"] = args.channels
    if args.field_deg:
        kw["size_deg"] = args.field_deg
    job = synth.config2(**kw)
    if args.workload == "config3":
        job.name = "config3"
    return job


def workload_text(job):
    """The workload string both arms report (the same config, the same words)."""
    return ("%s: %d samples x %d channels -> %dx%d RA---SIN/DEC--SIN, GAUSS1D FWHM %g\", sphere_radius 3 sigma"
            % (job.name, job.n, job.nchan, job.nx, job.ny, job.fwhm_arcsec))


def algorithmic_bytes(n, c, p):
    """Per sample FP64 lon/lat + FP32 spectrum read once; per pixel FP32 cube
    row + FP32 weight written once."""
    return n * (16 + 4 * c) + p * (4 * c + 4)


def device_spectra(job, torch, dev):
    """[N][C] float32 spectra on the device: G @ L + N(0, noise), seeded."""
    if job.values is not None:
        v = torch.from_numpy(np.ascontiguousarray(job.values.reshape(job.n, -1))).to(dev)
        return v
    G, L, noise = job.factors
    gen = torch.Generator(device=dev)
    gen.manual_seed(job.seed)
    Ld = torch.from_numpy(L).to(dev)
    S = torch.empty((job.n, job.nchan), dtype=torch.float32, device=dev)
    step = 1 << 18
    for i in range(0, job.n, step):
        Gd = torch.from_numpy(G[i:i + step]).to(dev)
        torch.matmul(Gd, Ld, out=S[i:i + step])
        S[i:i + step].add_(torch.randn((Gd.shape[0], job.nchan), generator=gen, device=dev), alpha=noise)
    return S


# ---------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.uuid, "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 8:
                    continue
                try:
                    sm.append(float(f[0]))
                    mx.append(float(f[1]))
                except ValueError:
                    continue
                for nm, v in zip(names, f[4:8]):
                    if v.lower() == "active":
                        reasons.add(nm)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baselines (the reference's own host build, else the oracle port)

class CStdoutToStderr:
    """Send what C code prints to stdout (the reference's host pre-sort
    prints its timings) to stderr, so stdout carries only the JSON line."""

    def __enter__(self):
        import ctypes
        sys.stdout.flush()
        self.libc = ctypes.CDLL(None)
        self.libc.fflush(None)
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *a):
        self.libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)


def reference_coords(job):
    """Target pixel centres of the workload's header as the reference computes
    them (its own read_output_map + set_WCS through oracle/_ref), else, where
    that build is absent, the library's host SIN projection."""
    from oracle import oracle as O
    if O.have_ref():
        nx, ny, xw, yw = O.ref_header_coords(job.header)
        return nx, ny, xw, yw, "reference set_WCS (wcslib)"
    from hcgrid_b200 import api
    nx, ny, xw, yw = api.header_coords(job.header)
    return nx, ny, xw, yw, "hcg_header_coords (reference build absent)"


def cpu_baseline(job, budget_s=12.0):
    """Reference CPU path on a bounded sample: full pre-sort of all samples
    plus the kernel body for one channel on central squares of the target,
    100x100 and then doubling while the sample stays within about `budget_s`
    (up to the whole map); extrapolated to the whole job as HCGrid+ runs it
    (geometry repeated per channel): T = T_sort + C * T_kernel, with T_kernel
    the whole map's time for one channel, measured when the whole map was
    sampled, else from a + b * pixels fitted to the two largest squares (a:
    the per-call setup, b: the per-pixel body). Target pixel centres come
    from the reference's own set_WCS."""
    from oracle import oracle as O
    nx, ny, xw, yw, coords_from = reference_coords(job)
    P = nx * ny
    vals = job.values if job.values is not None else (job.factors[0] @ job.factors[1][:, :1])[:, 0]
    vals = np.asarray(vals, np.float64).reshape(job.n, -1)[:, 0].copy()
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    full = min(nx, ny)  # the reference grids square maps (HCGrid/gridding.cu:289)

    def square(side):
        x0, y0 = (nx - side) // 2, (ny - side) // 2
        sel = (np.arange(side)[:, None] + y0) * nx + (np.arange(side)[None, :] + x0)
        return np.ascontiguousarray(xw[sel.ravel()]), np.ascontiguousarray(yw[sel.ravel()])

    with CStdoutToStderr():
        if O.have_ref():
            kind = "reference"
            O.ref_prepare(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
            t0 = time.perf_counter()
            keys, slon, slat, sdat, fr, ur, lut = O.ref_presort(job.lon, job.lat, vals, 2)
            t_sort = time.perf_counter() - t0

            def body(side):
                sx, sy = square(side)
                t0 = time.perf_counter()
                O.ref_grid(keys, slon, slat, sdat, lut, fr, ur, side, side, sx, sy)
                return time.perf_counter() - t0
        else:
            kind = "port"
            g = O.prepare_grid_kernel(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
            t0 = time.perf_counter()
            ps = O.presort(g.hpx, job.lon, job.lat)
            t_sort = time.perf_counter() - t0
            sl, sb, sd = job.lon[ps.perm], job.lat[ps.perm], vals[ps.perm]

            def body(side):
                sx, sy = square(side)
                t0 = time.perf_counter()
                O.grid(g, ps, sl, sb, sd, sx, sy)
                return time.perf_counter() - t0
        pts = [(min(full, 100), None)]
        pts[0] = (pts[0][0], body(pts[0][0]))
        spent = t_sort + pts[0][1]
        while pts[-1][0] < full:
            s = min(full, 2 * pts[-1][0])
            if spent + pts[-1][1] * (s / pts[-1][0]) ** 2 > budget_s:
                break
            pts.append((s, body(s)))
            spent += pts[-1][1]
    side, t_sub = pts[-1]
    if side * side >= P:
        t_kernel, how = t_sub, "the whole map measured"
    else:
        b, a = t_sub / side ** 2, 0.0
        if len(pts) >= 2:
            (s1, t1), (s2, t2) = pts[-2], pts[-1]
            if t2 > t1:
                b = (t2 - t1) / (s2 ** 2 - s1 ** 2)
                a = max(0.0, t1 - b * s1 ** 2)
        t_kernel = a + b * P
        how = "extrapolated to %d pixels by a + b * pixels (a = %.3f s, b = %.3g s)" % (P, a, b)
    t_job = t_sort + job.nchan * t_kernel
    value = job.n * job.nchan / t_job
    sample = ("pre-sort of all %d samples (%.2f s) + kernel body for 1 channel on central squares of %s pixels "
              "(%s s); one channel %.2f s (%s), times %d channels (T = %.1f s); target pixels from %s"
              % (job.n, t_sort, ", ".join("%d^2" % s for s, _ in pts), ", ".join("%.2f" % t for _, t in pts),
                 t_kernel, how, job.nchan, t_job, coords_from))
    return {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample,
            "seconds_measured": round(spent, 2)}


def reference_subcube(job, sub, vals):
    """The checker of the timed cube (part of the CPU leg, outside every
    timed region): the FP64 oracle (the C restatement of the reference's
    gridding, pinned bit-exact to the reference's host build) on the target
    pixels `sub` for the spectra columns `vals` [n, k] (input order). Returns
    (cube [len(sub), k] normalised, weights, cond [len(sub), k]) with cond =
    sum(w |x|) / sum(w): the magnitude of the summed terms, the scale of the
    rounding errors of any summation order."""
    from oracle import oracle as O
    _, _, xw, yw, _ = reference_coords(job)
    g = O.prepare_grid_kernel(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
    ps = O.presort(g.hpx, job.lon, job.lat)
    v = np.asarray(vals, np.float64)
    both = np.concatenate([v, np.abs(v)], axis=1)[ps.perm]
    oc, ow, _ = O.grid(g, ps, job.lon[ps.perm], job.lat[ps.perm], both, xw[sub], yw[sub])
    with np.errstate(invalid="ignore", divide="ignore"):
        k = v.shape[1]
        return oc[:, :k] / ow[:, None], ow, oc[:, k:] / ow[:, None]


def error_measures(got, ref, cond=None):
    """Relative errors of a gridded (sub-)cube against a reference, per
    channel plane (columns), over the pixels where the reference is finite:
      plane: max |got - ref| / max |ref| of the plane (the measure of the
             parity tests);
      elem:  max |got - ref| / |ref| over elements with |ref| above 1e-3 of
             their plane's largest |value|;
      cond:  max |got - ref| / cond, cond = sum(w |x|) / sum(w) per element
             (relative to the magnitude of the summed terms).
    The NaN patterns (pixels without samples) must agree."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    nan = np.isnan(ref)
    out = {"nan_pattern_equal": bool(np.array_equal(np.isnan(got), nan))}
    err = np.where(nan, 0.0, np.abs(got - ref))
    mag = np.where(nan, 0.0, np.abs(ref))
    pmax = mag.max(axis=0)
    out["max_rel_err_plane"] = float((err.max(axis=0) / np.maximum(pmax, 1e-300)).max())
    big = mag > 1e-3 * pmax[None, :]
    out["max_rel_err_elem"] = float((err[big] / mag[big]).max()) if big.any() else 0.0
    if cond is not None:
        c = np.where(nan, 1.0, np.asarray(cond, np.float64))
        out["max_rel_err_cond"] = float((err / np.maximum(c, 1e-300)).max())
    return out


def device_cube_errors(torch, got, ref, rows=1 << 17):
    """error_measures' plane and elem figures of two whole device cubes
    [pixels][channels] (ref: the FP32 engine's), in row blocks."""
    P = ref.shape[0]
    pmax = torch.zeros(ref.shape[1], dtype=torch.float64, device=ref.device)
    emax = torch.zeros_like(pmax)
    same_nan = True
    for i in range(0, P, rows):
        r, g = ref[i:i + rows].double(), got[i:i + rows].double()
        nan = torch.isnan(r)
        same_nan &= bool(torch.equal(nan, torch.isnan(g)))
        pmax = torch.maximum(pmax, torch.where(nan, 0.0, r.abs()).amax(dim=0))
        emax = torch.maximum(emax, torch.where(nan, 0.0, (g - r).abs()).amax(dim=0))
    elem = torch.zeros((), dtype=torch.float64, device=ref.device)
    for i in range(0, P, rows):
        r, g = ref[i:i + rows].double(), got[i:i + rows].double()
        mag = torch.where(torch.isnan(r), 0.0, r.abs())
        big = mag > 1e-3 * pmax[None, :]
        rel = torch.where(big, (g - r).abs() / torch.where(big, mag, 1.0), 0.0)
        elem = torch.maximum(elem, rel.max())
    return {"nan_pattern_equal": same_nan,
            "max_rel_err_plane": float((emax / torch.clamp(pmax, min=1e-300)).max()),
            "max_rel_err_elem": float(elem)}


# ---------------------------------------------------------------------------

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_max(torch, dist, v):
    """The largest of the ranks' values (every rank calls it; the timing
    convention: a multi-GPU step takes as long as its slowest rank)."""
    if dist is None:
        return v
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# served form (config 5) and batched form (config 4): request streams staged
# in windows (hcgrid_b200/streams.py), only the gridding timed


def check_sample(s, chans_max=3, side=16):
    """Host copy of a staged request's cube at its central side x side pixels
    and up to 3 channels spread over the band (for the per-result errors)."""
    from hcgrid_b200 import streams
    sh = s.r["shape"]
    g, C = sh["grid"], sh["nchan"]
    side = min(side, g)
    x0 = (g - side) // 2
    pix = ((np.arange(side)[:, None] + x0) * g + (np.arange(side)[None, :] + x0)).reshape(-1)
    chans = streams.check_channels(C, chans_max)
    cube = s.cube.view(-1, C)
    import torch
    return pix, chans, cube[torch.from_numpy(pix).to(cube.device)][:, torch.from_numpy(chans).to(cube.device)].cpu().numpy()


def served_run(args):
    """Config 5: a stream of `args.jobs` gridding requests with config-4 shapes
    (seed 3, no caps), 30% of them re-gridding an earlier request's field
    with new spectra. Windows of requests are staged on the device within
    the staging budget (fields and targets built on first use, resident
    until their last request); on each window, every arm runs on the same
    staged requests:

      plain        one hcg_grid call at a time, FP32 CUDA-core engine;
      tc_per_call  one hcg_grid call at a time, tensor-core engine;
      served       the window's requests submitted to hcg_server at once
                   (continuous batching over --lanes lanes, persistent batch
                   kernels replayed from CUDA graphs, tensor cores,
                   footprint admission against the HBM budget); capacity =
                   work / time from a window's first submit to its last
                   completion (closed loop).

    A second pass stages the windows again and submits with Poisson arrivals
    at 80% of the closed-loop capacity: p50/p99 latency (submit -> cube
    written). Every 100th request and the 3 largest are checked: served
    against the single call (bit for bit), the tensor cores against the FP32
    engine and, in the CPU leg, both against the FP64 oracle."""
    import torch
    from hcgrid_b200 import api, streams, synth
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    api.load(build_if_missing=True)
    budget = int(args.hbm_budget_gb * (1 << 30))
    reqs = synth.config5_requests(njobs=args.jobs, seed=3, reuse=0.3, max_grid=2048)
    work = [streams.request_work(r) for r in reqs]
    tot_work = sum(work)
    big = set(np.argsort(work)[-3:].tolist())
    checks = {r["request"] for r in reqs if r["request"] % 100 == 0 or r["request"] in big}
    stage_budget = min(budget, int(args.stage_gb * (1 << 30)))
    windows = streams.plan_windows(reqs, stage_budget)
    ctx = api.Context(0)
    ctx.tc_set_weights(api.TC_WEIGHTS_AUTO)
    samples = {}  # request -> {arm: (pix, chans, values)}
    plain_lat, tc_lat, lats_cl, busy, grids = [], [], [], 0.0, []
    busy_part, work_part = {False: 0.0, True: 0.0}, {False: 0, True: 0}  # by "fills the GPU alone"
    large_ids = set()  # requests whose channel sums fill the GPU (the server runs them alone)
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    srv = api.Server(ctx, lanes=args.lanes, hbm_budget=budget, max_batch=64)
    fields_built = 0
    try:
        run = streams.Runner(ctx, reqs, torch, dev)
        detail = open(args.detail, "w") if args.detail else None
        for wi, win in enumerate(windows):
            staged = []
            lat0 = len(tc_lat)
            for r in win:  # FP32 spectra kept beside the split: every arm runs on this staging
                st1 = run.stage([r], tc=False, keep=checks)[0]
                if st1.cols is not None:
                    samples.setdefault(r["request"], {})["cols"] = st1.cols
                if r["shape"]["nchan"] > 1:
                    st1.field.split_spectra(api.ENGINE_TC_F16, keep_fp32=True)
                staged.append(st1)
            ctx.synchronize()
            for s in staged:  # plain FP32, one call at a time
                t0 = time.perf_counter()
                ctx.grid(s.field, s.target, s.cube, s.weights, engine=api.ENGINE_FP32)
                ctx.synchronize()
                plain_lat.append(time.perf_counter() - t0)
                if s.r["request"] in checks:
                    samples.setdefault(s.r["request"], {})["plain"] = check_sample(s)
            for s in staged:  # tensor cores, one call at a time
                eng = api.ENGINE_TC_F16 if s.r["shape"]["nchan"] > 1 else api.ENGINE_FP32
                t0 = time.perf_counter()
                ctx.grid(s.field, s.target, s.cube, s.weights, engine=eng)
                ctx.synchronize()
                tc_lat.append(time.perf_counter() - t0)
                grids.append(s.r["shape"]["grid"])
                if streams.fills_gpu(s.r["shape"], nsm):
                    large_ids.add(len(tc_lat) - 1)
                if s.r["request"] in checks:
                    samples[s.r["request"]]["tc"] = check_sample(s)
            # the window once through the server, untimed: lanes capture their
            # batch graphs and grow their scratch to the window's sizes, as the
            # per-call arms' context already has from the passes above
            for tk in [srv.submit(s.field, s.target, s.cube, s.weights, api.SAMPLE_MAJOR,
                                  footprint=streams.footprint(s.r["shape"])) for s in staged]:
                srv.wait(tk)
            # closed loop, timed in two parts: the window's small requests (the
            # server batches them), then the ones that fill the GPU alone (each
            # runs as one hcg_grid); capacity = all work / both parts' time
            for part in (False, True):
                sub = [s for s in staged if streams.fills_gpu(s.r["shape"], nsm) == part]
                if not sub:
                    continue
                t0 = time.perf_counter()
                tickets = [srv.submit(s.field, s.target, s.cube, s.weights, api.SAMPLE_MAJOR,
                                      footprint=streams.footprint(s.r["shape"])) for s in sub]
                for tk in tickets:
                    lats_cl.append(srv.wait(tk)[0])
                dt = time.perf_counter() - t0
                busy += dt
                busy_part[part] += dt
                work_part[part] += sum(streams.request_work(s.r) for s in sub)
                if detail:
                    tcs = sum(tc_lat[lat0 + i] for i, s in enumerate(staged)
                              if streams.fills_gpu(s.r["shape"], nsm) == part)
                    detail.write(json.dumps({"window": wi, "large": part, "requests": len(sub), "served_s": dt,
                                             "tc_per_call_s": tcs}) + "\n")
            for s in staged:
                if s.r["request"] in checks:
                    samples[s.r["request"]]["served"] = check_sample(s)
            run.unstage(staged)
        fields_built += run.built
        run.close()
        if detail:
            detail.close()
        capacity = tot_work / busy
        rate = 0.8 * len(reqs) / busy
        # second pass: Poisson arrivals at 80% of the closed-loop capacity
        rng = np.random.default_rng(3)
        run = streams.Runner(ctx, reqs, torch, dev)
        lats, queues, busy_p = [], [], 0.0
        for win in windows:
            staged = run.stage(win, tc=True)
            arr = np.cumsum(rng.exponential(1.0 / rate, len(staged)))
            arr -= arr[0]
            t0 = time.perf_counter()
            tickets = []
            for i, s in enumerate(staged):
                d = t0 + arr[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets.append(srv.submit(s.field, s.target, s.cube, s.weights, api.SAMPLE_MAJOR,
                                          footprint=streams.footprint(s.r["shape"])))
            for tk in tickets:
                lt, q = srv.wait(tk)
                lats.append(lt)
                queues.append(q)
            busy_p += time.perf_counter() - t0
            run.unstage(staged)
        fields_built += run.built
        run.close()
        st = srv.stats()
    finally:
        srv.close()
    pct = lambda v, q: float(np.percentile(np.asarray(v), q))
    plain = tot_work / sum(plain_lat)
    tcv = tot_work / sum(tc_lat)
    # served vs single call (bit for bit) and tensor cores vs FP32 engine, on the checked requests
    served_same, tc_vs_fp32 = True, 0.0
    for rid, d in samples.items():
        if "served" in d and "tc" in d:
            served_same &= bool(np.array_equal(d["served"][2], d["tc"][2], equal_nan=True))
        if "plain" in d and "tc" in d:
            tc_vs_fp32 = max(tc_vs_fp32, error_measures(d["tc"][2], d["plain"][2])["max_rel_err_plane"])
    out = {"metric": METRIC, "value": capacity, "unit": UNIT, "n_gpus": 1, "steps": len(reqs), "warmup": 1,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "fp16 hi/lo tensor-core channel sums (FP64 geometry)",
           "data": "synthetic (seeded config-5 request stream, hcgrid_b200/synth.py)",
           "config": {"workload": "config5: %d requests, config-4 shapes (seed 3, uncapped), 30%% field reuse, HBM "
                                  "budget %.0f GB" % (len(reqs), args.hbm_budget_gb),
                      "unique_fields": len({r["field"] for r in reqs}), "windows": len(windows),
                      "staging_budget_gb": args.stage_gb, "total_sample_channels": tot_work,
                      "fields_built": fields_built,
                      "engine": "served: hcg_server (%d lane%s, batch graphs, tensor cores FP16 hi/lo); "
                                % (args.lanes, "" if args.lanes == 1 else "s") +
                                "plain: hcg_grid FP32 engine per call"},
           "served": {"capacity": capacity, "busy_s": round(busy, 4), "batches": st["batches"],
                      "p50_s_closed_loop": pct(lats_cl, 50), "p99_s_closed_loop": pct(lats_cl, 99),
                      "poisson_rate_per_s": round(rate, 3), "throughput_at_80pct": tot_work / busy_p,
                      "p50_s": pct(lats, 50), "p99_s": pct(lats, 99), "queue_p99_s": pct(queues, 99)},
           "plain": {"value": plain, "p50_s": pct(plain_lat, 50), "p99_s": pct(plain_lat, 99),
                     "total_s": round(sum(plain_lat), 4)},
           "tc_per_call": {"value": tcv, "p50_s": pct(tc_lat, 50), "p99_s": pct(tc_lat, 99),
                           "total_s": round(sum(tc_lat), 4)},
           "served_over_plain": round(capacity / plain, 3), "served_over_tc_per_call": round(capacity / tcv, 3),
           "by_size": {
               "what": "closed-loop capacity of the server and per-call rates on the requests batched by the "
                       "server (small) and on those whose channel sums fill the GPU (large: run alone by both)",
               "small": {"served": work_part[False] / max(busy_part[False], 1e-9),
                         "tc_per_call": work_part[False] / max(sum(x for i, x in enumerate(tc_lat)
                                                                    if i not in large_ids), 1e-9),
                         "served_s": round(busy_part[False], 4)},
               "large": {"served": work_part[True] / max(busy_part[True], 1e-9),
                         "tc_per_call": work_part[True] / max(sum(tc_lat[i] for i in large_ids), 1e-9),
                         "served_s": round(busy_part[True], 4)}},
           "per_call_time_split": {
               "what": "seconds of the per-call arms in requests whose channel sums fill the GPU (2^20 pixels or "
                       "more, or one 16x8-pixel x 256-channel item per SM; the server runs those alone, as one "
                       "hcg_grid each) and in the others (batched by the server)",
               "large": {"requests": len(large_ids), "tc_s": round(sum(tc_lat[i] for i in large_ids), 3),
                         "plain_s": round(sum(plain_lat[i] for i in large_ids), 3)},
               "small": {"requests": len(tc_lat) - len(large_ids),
                         "tc_s": round(sum(x for i, x in enumerate(tc_lat) if i not in large_ids), 3),
                         "plain_s": round(sum(x for i, x in enumerate(plain_lat) if i not in large_ids), 3)},
               "by_grid": {str(g): {"requests": grids.count(g),
                                    "tc_s": round(sum(x for x, gg in zip(tc_lat, grids) if gg == g), 3),
                                    "plain_s": round(sum(x for x, gg in zip(plain_lat, grids) if gg == g), 3)}
                           for g in sorted(set(grids))}},
           "checks": {"requests": sorted(samples), "served_equals_single_call": served_same,
                      "tc_vs_fp32_engine_max_rel_err_plane": tc_vs_fp32},
           "gpu_launches": None, "e2e": None, "cpu_baseline": None}
    if args.oracle_checks:
        out["checks"]["vs_fp64_oracle"] = served_oracle_checks(reqs, samples)
    ctx.close()
    return out


def served_oracle_checks(reqs, samples):
    """The CPU leg's checker for the served stream: the FP64 oracle on each
    checked request's sampled pixels and channels (the request's samples
    regenerated on the host from their seed, its spectra columns as staged on
    the device), against the tensor-core and served cubes. Requests above 2e8
    candidate pair-channels are left to the comparison with the FP32 engine."""
    from oracle import oracle as O
    from hcgrid_b200 import api, synth
    by_id = {r["request"]: r for r in reqs}
    out = {}
    for rid, d in sorted(samples.items()):
        r = by_id[rid]
        sh = r["shape"]
        if synth.job_work(dict(sh, nchan=3)) > 2e8 or "tc" not in d or "cols" not in d:
            continue
        rng = np.random.default_rng(sh["seed"])
        lon, lat = synth.raster_scan(sh["n"], sh["ra"], sh["dec"], sh["size_deg"], 2.0, rng)
        pix, chans, got = d["tc"]
        vals = d["cols"]
        sigma = sh["fwhm"] / 3600.0 * synth.FWHM_TO_SIGMA
        hdr = synth.sin_header(sh["grid"], sh["grid"], sh["ra"], sh["dec"], sh["size_deg"] / sh["grid"])
        _, _, xw, yw = api.header_coords(hdr)
        g = O.prepare_grid_kernel(sigma, 3.0 * sigma, sigma / 2.0)
        ps = O.presort(g.hpx, lon, lat)
        both = np.concatenate([vals, np.abs(vals)], axis=1)[ps.perm]
        oc, ow, _ = O.grid(g, ps, lon[ps.perm], lat[ps.perm], both, xw[pix], yw[pix])
        k = len(chans)
        with np.errstate(invalid="ignore", divide="ignore"):
            ref, cond = oc[:, :k] / ow[:, None], oc[:, k:] / ow[:, None]
        e = error_measures(got, ref, cond)
        e["served"] = error_measures(d["served"][2], ref, cond)["max_rel_err_plane"] if "served" in d else None
        e["shape"] = {k2: sh[k2] for k2 in ("n", "nchan", "grid", "fwhm")}
        out[str(rid)] = e
    return out


def config4_run(args):
    """Config 4, the batched form: 256 independent scan blocks (seed 2, the
    config-4 shapes, each its own field), staged in windows that fit the
    staging budget (all 256 hold 340 GB of spectra and 608 GB of cubes);
    each window is gridded by one hcg_grid_batch call (persistent kernels fed
    by device work queues, replayed from the context's captured graphs).
    value = the blocks' sample-channels / the summed wall time of the batch
    calls; the same blocks one hcg_grid call at a time (tensor cores) beside
    it."""
    import torch
    from hcgrid_b200 import api, streams, synth
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    api.load(build_if_missing=True)
    shapes = synth.config4_shapes(nblocks=args.blocks, seed=2)
    reqs = [dict(request=i, field=i, shape=sh, spectra_seed=sh["seed"] + 1) for i, sh in enumerate(shapes)]
    windows = streams.plan_windows(reqs, int(args.stage_gb * (1 << 30)))
    ctx = api.Context(0)
    run = streams.Runner(ctx, reqs, torch, dev)
    t_batch, t_call, same = 0.0, 0.0, True
    tuning = None
    try:
        for win in windows:
            staged = run.stage(win, tc=True)
            jobs = [(s.field, s.target, s.cube, s.weights, api.SAMPLE_MAJOR) for s in staged]
            if tuning is None and args.batch_shape is not None:
                ctx.batch_set_shape(args.batch_shape)
                ctx.grid_batch(jobs)  # untimed: the batch graphs are captured
                tuning = [{"shape": args.batch_shape, "how": "fixed by --batch-shape for every class"}]
            if tuning is None:  # untimed: the batch graphs are captured and the batch autotuner picks
                # a tensor-core shape per channel class on the first window's blocks
                tuning = ctx.autotune_batch(jobs, reps=args.tune_reps)
            ctx.synchronize()
            t0 = time.perf_counter()
            ctx.grid_batch(jobs)
            t_batch += time.perf_counter() - t0
            keep = [s.cube[:4096].clone() for s in staged]
            for s, k in zip(staged, keep):
                t0 = time.perf_counter()
                ctx.grid(s.field, s.target, s.cube, s.weights)
                ctx.synchronize()
                t_call += time.perf_counter() - t0
                same &= bool(torch.equal(torch.nan_to_num(s.cube[:4096], 7.0), torch.nan_to_num(k, 7.0)))
            run.unstage(staged)
    finally:
        run.close()
    # where batching pays: the same blocks at the small end of each range
    # (10,000 samples, 64^2 pixels, 1 or 64 channels), launch-bound one by one
    tiny = [dict(request=i, field=i, shape=dict(r["shape"], n=10000, grid=64,
                                                nchan=1 if r["shape"]["nchan"] == 1 else 64),
                 spectra_seed=r["spectra_seed"]) for i, r in enumerate(reqs)]
    run = streams.Runner(ctx, tiny, torch, dev)
    try:
        staged = run.stage(tiny, tc=True)
        jobs = [(s.field, s.target, s.cube, s.weights, api.SAMPLE_MAJOR) for s in staged]
        tb, tc1 = [], []
        for rep in range(4):  # the first of each is a warm-up
            ctx.synchronize()
            t0 = time.perf_counter()
            ctx.grid_batch(jobs)
            tb.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
            for s in staged:
                ctx.grid(s.field, s.target, s.cube, s.weights)
            ctx.synchronize()
            tc1.append(time.perf_counter() - t0)
        run.unstage(staged)
    finally:
        run.close()
    tiny_work = sum(streams.request_work(r) for r in tiny)
    tiny_out = {"what": "the 256 blocks at 10,000 samples, 64^2 pixels and 1 or 64 channels: one hcg_grid_batch "
                        "against one hcg_grid call at a time (best of 3 after a warm-up)",
                "batch_s": round(min(tb[1:]), 5), "per_call_s": round(min(tc1[1:]), 5),
                "batch": tiny_work / min(tb[1:]), "per_call": tiny_work / min(tc1[1:]),
                "batch_over_per_call": round(min(tc1[1:]) / min(tb[1:]), 3)}
    work = sum(streams.request_work(r) for r in reqs)
    out = {"metric": METRIC, "value": work / t_batch, "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 1,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "fp16 hi/lo tensor-core channel sums (FP64 geometry); FP64 single-channel blocks",
           "data": "synthetic (seeded config-4 scan blocks, hcgrid_b200/synth.py)",
           "config": {"workload": "config4: %d scan blocks (seed 2), log-uniform 1e4-2e6 samples, 1-15 deg, "
                                  "64^2-2048^2 SIN, {1,64,256,1024,2048} channels, FWHM {60,180,300}\""
                                  % len(reqs), "windows": len(windows), "staging_budget_gb": args.stage_gb,
                      "total_sample_channels": work},
           "batch_s": round(t_batch, 4), "per_call_tc": {"value": work / t_call, "total_s": round(t_call, 4)},
           "batch_over_per_call": round(t_call / t_batch, 3), "batch_equals_single_call": same,
           "launch_bound_blocks": tiny_out,
           "batch_tuning": {"classes": tuning, "how": "hcg_autotune_batch on the first window: per channel class, "
                            "each of the 4 shapes (0: 256 ch x 32 slots x 4 stages, 1: 256 x 64 x 2, "
                            "2: 128 x 64 x 3, 3: 64 x 64 x 4) timed as one hcg_grid_batch of the class's "
                            "blocks, best of %d runs after a warm-up" % args.tune_reps},
           "gpu_launches": None, "e2e": None, "cpu_baseline": None}
    ctx.close()
    return out


def main():
    args = parse()
    if args.workload in ("config4", "config5"):
        if args.impl == "ours":
            print(json.dumps(served_run(args) if args.workload == "config5" else config4_run(args)))
            return
        print(json.dumps({"impl": "reference", "unavailable": "the batched and served forms run the B200 batch "
                          "engine and request loop; the reference's CPU path is timed on config2 and config1"}))
        return
    world, rank, local = dist_setup(args)
    job = job_for(args)
    P = job.nx * job.ny
    served = None
    if args.impl == "ours" and world == 1 and args.workload == "config2" and args.served_jobs > 0:
        # the served form (config 5) before the config-2 field takes its memory
        import torch
        sargs = argparse.Namespace(**vars(args))
        sargs.jobs, sargs.detail, sargs.oracle_checks = args.served_jobs, None, 0
        try:
            s = served_run(sargs)
            served = {"value": s["value"], "unit": UNIT, "requests": s["steps"],
                      "served_over_plain": s["served_over_plain"], "plain_per_call": s["plain"]["value"],
                      "tc_per_call": s["tc_per_call"]["value"], "p50_s": s["served"]["p50_s"],
                      "p99_s": s["served"]["p99_s"], "load": "Poisson arrivals at 80% of closed-loop capacity",
                      "workload": s["config"]["workload"]}
        except Exception as ex:  # reported, not fatal
            served = {"value": None, "error": repr(ex)}
        gc.collect()  # the served leg's server, fields and buffers are released here, not inside a later timed step
        torch.cuda.empty_cache()
    if args.impl == "reference":
        if rank == 0:
            vals = []
            info = None
            for i in range(args.warmup + args.steps):
                info = cpu_baseline(job)
                if i >= args.warmup:
                    vals.append(info["value"])
            v = statistics.median(vals)
            info["value"] = v
            out = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
                   "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                   "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, %s generator)" % job.name,
                   "config": {"workload": workload_text(job)},
                   "cpu_baseline": info, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                                                 "d2h_bytes_per_step": 0}}
            print(json.dumps(out))
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from hcgrid_b200 import api
    api.load(build_if_missing=True)
    stream = torch.cuda.Stream(device=dev)
    ctx = api.Context(local, stream=stream.cuda_stream)
    kp = np.array([job.sigma_deg, 0.0, 0.0])
    ctx.prepare_grid_kernel(api.GAUSS1D, kp, job.sphere_radius, job.hpx_max_res)
    with torch.cuda.stream(stream):
        lon_d = torch.from_numpy(job.lon).to(dev)
        lat_d = torch.from_numpy(job.lat).to(dev)
        S = device_spectra(job, torch, dev)
    stream.synchronize()
    engine = ENGINES[args.engine]
    bands = None
    if world > 1 and args.shard == "bands":
        # Dec-band sharding of the one job: this rank grids target rows
        # [y0, y1) from the contiguous range of ring-sorted samples they need
        # (hcg_field_band_samples); only that range's spectra are attached
        from hcgrid_b200 import shard
        bands = shard.plan(job.ny, world)
        y0, y1 = bands[rank]
        geometry = ctx.field(lon_d, lat_d)  # sample positions only: the sort that gives the ranges
        whole = ctx.target_from_header(job.header)
        field, band_idx, band_target = shard.band_field(ctx, geometry, whole, job.lon, job.lat, y0, y1)
        geometry.close()
        whole.close()
        if field is None:
            raise RuntimeError("band [%d, %d) holds no samples" % (y0, y1))
        S = S.index_select(0, torch.from_numpy(band_idx.astype(np.int64)).to(dev))
        P = (y1 - y0) * job.nx
    else:
        field = ctx.field(lon_d, lat_d)
    n_rank = S.shape[0]  # samples this rank grids from
    field.set_spectra(S)
    ctx.synchronize()
    # the checked sub-cube: central side x side pixels x k channels spread over
    # the band (config 3: 256 x 256 x 64, config 2: 64 x 64 x 16)
    check = None
    if rank == 0 and world == 1 and not args.no_check:
        side = min(256 if job.name == "config3" else 64, job.nx, job.ny)
        k = min(64 if job.name == "config3" else 16, job.nchan)
        chans = np.linspace(0, job.nchan - 1, k).round().astype(np.int64)
        x0, y0 = (job.nx - side) // 2, (job.ny - side) // 2
        subpix = ((np.arange(side)[:, None] + y0) * job.nx + (np.arange(side)[None, :] + x0)).reshape(-1)
        vals = S[:, torch.from_numpy(chans).to(dev)].double().cpu().numpy()
        check = {"side": side, "chans": chans, "sub": subpix, "vals": vals,
                 "sub_d": torch.from_numpy(subpix).to(dev), "chans_d": torch.from_numpy(chans).to(dev)}
    S_host = planes_host = None
    if args.e2e_steps > 0:
        # the host spectra of the end-to-end leg: channel planes [nchan][n] in
        # input sample order (the reference's h_data[channel][sample]) for
        # hcg_grid_planes, and sample rows [n][nchan] for the per-call path
        planes_host = torch.empty((S.shape[1], S.shape[0]), dtype=torch.float32, pin_memory=True)
        planes_host.copy_(S.t())
        S_host = torch.empty(tuple(S.shape), dtype=torch.float32, pin_memory=True)
        S_host.copy_(S)
    del S  # the field holds its own (sorted) copy
    torch.cuda.empty_cache()
    plain_steps = args.plain_steps if (engine != api.ENGINE_FP32 and job.nchan > 1) else 0
    if engine != api.ENGINE_FP32 and job.nchan > 1:
        field.split_spectra(engine, keep_fp32=plain_steps > 0)
    target = band_target if bands else ctx.target_from_header(job.header)
    ctx.synchronize()
    torch.cuda.empty_cache()
    LAY = api.CHANNEL_MAJOR if args.layout == "channel" else api.SAMPLE_MAJOR
    pm = (lambda c: c.t()) if LAY == api.CHANNEL_MAJOR else (lambda c: c)  # a [pixel][channel] view
    cube = torch.empty((job.nchan, P) if LAY == api.CHANNEL_MAJOR else (P, job.nchan), dtype=torch.float32,
                       device=dev)
    wts = torch.empty(P, dtype=torch.float32, device=dev)
    # prep, tile rings, count of overflowed tiles, 3-pass scan, row offsets, weights, sums
    launches_per_step = 2 if job.nchan == 1 else 9

    tune = None
    if engine != api.ENGINE_FP32 and job.nchan > 1:
        ctx.tc_set_weights({"auto": api.TC_WEIGHTS_AUTO, "entries": api.TC_WEIGHTS_ENTRIES,
                            "direct": api.TC_WEIGHTS_DIRECT}[args.tc_weights])
        if args.tc_config is not None:
            ctx.tc_set_config(args.tc_config)
            ctx.tc_set_pipeline(args.tc_prefetch, args.tc_strip)
            tune = {"config": args.tc_config, "prefetch": args.tc_prefetch, "strip": args.tc_strip,
                    "how": "fixed by --tc-config/--tc-prefetch/--tc-strip (-1: defaults)"}
        else:
            ctx.autotune_layout(LAY)
            tune = ctx.autotune_ex(field, target, reps=args.tune_reps)
            tune["how"] = ("hcg_autotune_ex: pipeline shape, then prefetch distance, then tile walk; each setting "
                           "the best of %d timed runs after a warm-up, gridding in the bench's cube layout; "
                           "spread = (slowest - fastest) / fastest of the chosen setting's runs" % args.tune_reps)
    for _ in range(args.warmup):
        ctx.grid(field, target, cube, wts, layout=LAY, engine=engine)
    ctx.synchronize()
    stats = ctx.stats()

    uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    phase_ms = [[] for _ in range(4)]
    step_ms = []
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(uuid) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            ctx.grid(field, target, cube, wts, layout=LAY, engine=engine)
            st = ctx.stats()  # phase times of this step (device events on the launching stream)
            for i in range(4):
                phase_ms[i].append(st.ms_phase[i])
            step_ms.append(st.ms_total)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    total_ms = ev0.elapsed_time(ev1)
    if dist is not None:
        dist.barrier()
    ms_per_step = reduce_max(torch, dist, total_ms / args.steps)
    clocks = clk.summary()
    assemble_ms = None
    if bands:
        # the band slabs to rank 0, device to device (NCCL gather), timed apart
        dist.barrier()
        torch.cuda.synchronize(dev)
        ta = time.perf_counter()
        whole_cube, whole_w = shard.assemble_tensors(dist, rank, world, bands, job.nx, pm(cube), wts)
        torch.cuda.synchronize(dev)
        assemble_ms = reduce_max(torch, dist, (time.perf_counter() - ta) * 1e3)
        del whole_cube, whole_w
        torch.cuda.empty_cache()
    st = ctx.stats()  # counters of the last timed step (before the plain engine runs)
    timed_sub = None
    cube_timed = None
    if check is not None:
        timed_sub = pm(cube)[check["sub_d"]][:, check["chans_d"]].double().cpu().numpy()
        if plain_steps > 0 and torch.cuda.mem_get_info(dev)[0] > cube.numel() * 4 + (8 << 30):
            cube_timed = cube.clone()  # the last timed step's cube, against the FP32 engine's below
    plain = None
    plain_sub = None
    vs_fp32 = None
    if plain_steps > 0:
        # the plain FP32 CUDA-core engine on the same resident field, same timing rules
        for _ in range(2):
            ctx.grid(field, target, cube, wts, layout=LAY, engine=api.ENGINE_FP32)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
        pe0 = torch.cuda.Event(enable_timing=True)
        pe1 = torch.cuda.Event(enable_timing=True)
        pe0.record(stream)
        for _ in range(plain_steps):
            ctx.grid(field, target, cube, wts, layout=LAY, engine=api.ENGINE_FP32)
        pe1.record(stream)
        torch.cuda.synchronize(dev)
        pms = reduce_max(torch, dist, pe0.elapsed_time(pe1) / plain_steps)
        if check is not None:
            plain_sub = pm(cube)[check["sub_d"]][:, check["chans_d"]].double().cpu().numpy()
            if cube_timed is not None:
                vs_fp32 = device_cube_errors(torch, pm(cube_timed), pm(cube))
                vs_fp32["what"] = "the whole timed cube against the FP32 engine's cube of the same field"
                del cube_timed
                torch.cuda.empty_cache()
        plain = {"engine": ENGINE_TEXT["fp32"], "value": job.n * job.nchan * (1 if bands else world) / (pms * 1e-3),
                 "ms_per_step": round(pms, 3), "steps": plain_steps, "warmup": 2}
    work = job.n * job.nchan
    copies = 1 if bands else world  # bands: one job over all ranks; replicas: a job per rank
    value = work * copies / (ms_per_step * 1e-3)

    # dominant kernel and its roofline
    tc = engine != api.ENGINE_FP32 and job.nchan > 1
    phase_names = ["pixel setup", "candidate count+scan", "FP64 weights (k_group)",
                   "channel sums (k_tile_tc)" if tc else "channel sums (k_tile_accum)"]
    kernels = ["k_pixel_prep", "k_group<true>+k_scan_offsets", "k_group<false>", "k_tile_tc" if tc else "k_tile_accum"]
    if job.nchan == 1:
        phase_names[3] = "single-channel gridding (k_grid_1chan)"
        kernels[3] = "k_grid_1chan"
    avg = [statistics.mean(x) for x in phase_ms]
    dom = int(np.argmax(avg))
    if dom == 3:
        alg = n_rank * 4 * job.nchan + P * (4 * job.nchan + 4)
        if job.nchan == 1:
            alg = algorithmic_bytes(n_rank, 1, P)
    else:
        alg = algorithmic_bytes(n_rank, 0, 0) if dom == 2 else P * 16
    peak, peak_kind = peaks()
    achieved = alg / (avg[dom] * 1e-3) / 1e9
    traffic = None
    try:
        tr = json.load(open(TRAFFIC))
        t = tr.get("%s:%dx%d:%d" % (job.name, job.n, job.nchan, job.nx), {}).get(kernels[dom])
        traffic = t if t is None else float(t)
    except Exception:
        pass
    roofline = {"bound": "hbm", "kernel": kernels[dom], "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6650 GB/s", "traffic": traffic,
                "algorithmic_bytes_per_launch": alg, "kernel_ms": round(avg[dom], 3),
                "phase_ms": {n: round(a, 3) for n, a in zip(phase_names, avg)},
                "whole_step_hbm_frac": round(algorithmic_bytes(n_rank, job.nchan, P) / (ms_per_step * 1e-3) / 1e9 / peak, 4),
                "pairs_within": int(st.pairs_within), "pairs_candidate": int(st.pairs_candidate)}
    if tc and dom == 3:
        tpk, tkind = tensor_peak()
        tflops = 2.0 * st.tc_macs / (avg[3] * 1e-3) / 1e12
        useful = int(st.pairs_within) * job.nchan
        tensor = {"achieved": round(tflops, 1), "peak": tpk, "unit": "TFLOP/s", "frac": round(tflops / tpk, 4),
                  "issued_macs": int(st.tc_macs), "useful_macs": useful,
                  "useful_tflops_x3": round(2.0 * 3 * useful / (avg[3] * 1e-3) / 1e12, 1),
                  "peak_source": tkind + " (MEASURED_PEAKS.json bf16_tflops, burst)",
                  "counts": "issued: the dense tile products the pipe executes (3 per MAC of the compensated "
                            "split); useful: accepted pairs x channels"}
        if tflops / tpk > roofline["frac"]:
            # the tensor pipe is the binding resource: its figures lead, HBM's are kept beside
            hbm = {k: roofline.pop(k) for k in ("achieved", "peak", "unit", "frac", "peak_source")}
            roofline.pop("bound")
            roofline = {"bound": "tensor", "kernel": roofline.pop("kernel"), **tensor, "hbm": hbm, **roofline}
        else:
            roofline["tensor"] = tensor

    # end to end through the C ABI from host buffers
    e2e = None
    if args.e2e_steps > 0:
        if bands:
            lon_h, lat_h = job.lon[band_idx], job.lat[band_idx]
            _, _, hx, hy = api.header_coords(job.header)
            bx = np.ascontiguousarray(hx[bands[rank][0] * job.nx:bands[rank][1] * job.nx])
            by = np.ascontiguousarray(hy[bands[rank][0] * job.nx:bands[rank][1] * job.nx])

            def make_target():
                return ctx.target(job.nx, bands[rank][1] - bands[rank][0], bx, by)
        else:
            lon_h, lat_h = job.lon, job.lat

            def make_target():
                return ctx.target_from_header(job.header)
        # sample positions in pinned host memory too
        lon_h = torch.from_numpy(np.ascontiguousarray(lon_h)).pin_memory()
        lat_h = torch.from_numpy(np.ascontiguousarray(lat_h)).pin_memory()
        cube_h = torch.empty((job.nchan, P) if LAY == api.CHANNEL_MAJOR else (P, job.nchan), dtype=torch.float32,
                             pin_memory=True)
        w_h = torch.empty(P, dtype=torch.float32, pin_memory=True)
        # garbage of the earlier legs is collected now, and the objects that
        # survive are left out of later collections, so that no collection
        # of the harness's own objects runs inside a timed step
        gc.collect()
        gc.freeze()
        times = []
        steps_calls = []  # host time of each call, every timed step
        free_gb = []  # device memory free after each step (the context's pool keeps what it maps)
        for i in range(args.e2e_steps + 1):
            if dist is not None:
                dist.barrier()
            t0 = time.perf_counter()
            f2 = ctx.field(lon_h, lat_h)
            ta = time.perf_counter()
            t2 = make_target()
            ctx.grid_planes(f2, t2, planes_host, cube_h, w_h, layout=LAY, engine=engine, block=args.plane_block)
            dt = time.perf_counter() - t0
            f2.close()
            t2.close()
            free_gb.append(round(torch.cuda.mem_get_info(dev)[0] / 1e9, 2))
            if i > 0:
                times.append(dt)
                steps_calls.append([round(ta - t0, 4), round(t0 + dt - ta, 4)])
        # the per-call path once, untimed, with a synchronize after each call
        calls = {}
        t0 = time.perf_counter()
        t_start = t0

        def mark(name):
            nonlocal t0
            ctx.synchronize()
            t = time.perf_counter()
            calls[name] = round(t - t0, 4)
            t0 = t

        f2 = ctx.field(lon_h, lat_h)
        mark("hcg_field_create")
        f2.set_spectra(S_host)
        mark("hcg_field_set_spectra")
        if tc:
            f2.split_spectra(engine, keep_fp32=False)
            mark("hcg_field_split_spectra")
        t2 = make_target()
        mark("hcg_target_from_header")
        ctx.grid(f2, t2, cube_h, w_h, layout=LAY, engine=engine)
        mark("hcg_grid")
        per_call_s = round(time.perf_counter() - t_start, 4)
        f2.close()
        t2.close()
        t_e2e = reduce_max(torch, dist, statistics.mean(times))
        h2d = 16 * n_rank + 4 * n_rank * job.nchan  # this rank's inputs
        d2h = 4 * P * job.nchan + 4 * P
        e2e = {"value": work * copies / t_e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "s_per_step": round(t_e2e, 4), "s_steps": [round(x, 4) for x in times],
               "calls_s_timed_steps": steps_calls, "device_free_gb_after_step": free_gb,
               "path": "hcg_field_create (sort) + hcg_target_from_header + hcg_grid_planes (channel planes in "
                       "pinned host memory, %d-channel blocks: upload, split, gridding and cube download "
                       "overlapped)" % (args.plane_block or 64),
               "calls_s_timed_steps_what": "[hcg_field_create, hcg_target_from_header + hcg_grid_planes]",
               "per_call_path": {"s": per_call_s, "calls_s": calls,
                                 "path": "hcg_field_create + hcg_field_set_spectra (sample rows)%s + "
                                         "hcg_target_from_header + hcg_grid, one untimed pass with a synchronize "
                                         "after each call" % (" + hcg_field_split_spectra" if tc else "")}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(job)
        except Exception as ex:  # reported, not fatal
            cpu = {"value": None, "error": repr(ex)}
    validation = None
    if check is not None:
        # the CPU leg's checker, after every timed region
        try:
            ref_sub, ref_w, cond = reference_subcube(job, check["sub"], check["vals"])
            validation = {"reference": "FP64 oracle (C restatement pinned bit-exact to the reference's host build) "
                                       "on the central %dx%d pixels x %d channels spread over the band"
                                       % (check["side"], check["side"], len(check["chans"])),
                          "channels": [int(c) for c in check["chans"]],
                          "elem_floor": "elements with |ref| > 1e-3 of their plane's max",
                          "timed_cube_vs_fp64": error_measures(timed_sub, ref_sub, cond)}
            if plain_sub is not None:
                validation["fp32_engine_vs_fp64"] = error_measures(plain_sub, ref_sub, cond)
            if vs_fp32 is not None:
                validation["timed_cube_vs_fp32_engine"] = vs_fp32
        except Exception as ex:  # reported, not fatal
            validation = {"error": repr(ex)}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True,
               "scaling": "strong" if bands else "weak", "vs_baseline": None,
               "dtype": DTYPE_TEXT[args.engine] if job.nchan > 1 else DTYPE_TEXT["fp32"],
               "data": "synthetic (seeded %s generator, hcgrid_b200/synth.py)" % job.name,
               "config": {"workload": workload_text(job),
                          "samples": job.n, "channels": job.nchan, "pixels": P, "nside": ctx.info(field).nside,
                          "parallelism": ("dec bands of target rows, one per rank, NCCL gather to rank 0"
                                          if bands else "replica per GPU" if world > 1 else "single GPU"),
                          "bands": bands, "assemble_ms": assemble_ms,
                          "l2": "inputs larger than L2 (spectra %.1f GB), no flush" % (4 * job.n * job.nchan / 1e9),
                          "cube_layout": ("[channel][pixel] (the reference's h_datacube planes)"
                                          if LAY == api.CHANNEL_MAJOR else "[pixel][channel]"),
                          "engine": ENGINE_TEXT[args.engine] if job.nchan > 1 else ENGINE_TEXT["fp32"],
                          "tc_pipeline": tune, "tc_weights": args.tc_weights},
               "gpu_launches": launches_per_step * args.steps, "clocks": clocks, "roofline": roofline,
               "e2e": e2e, "cpu_baseline": cpu, "plain_fp32": plain,
               "over_plain_fp32": round(value / plain["value"], 3) if plain else None,
               "served_config5": served, "validation": validation}
        print(json.dumps(out))
    field.close()
    target.close()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
