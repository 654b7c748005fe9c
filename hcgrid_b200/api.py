"""Python binding of the C ABI (include/hcgrid_c.h) through ctypes.

Host arrays are numpy; device arrays are any object exposing
``data_ptr()`` (torch CUDA tensors) and are passed as device pointers.
The library must have been built (``python -m hcgrid_b200.build``); there is
no fallback: loading fails loudly without it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

GAUSS1D, GAUSS2D, TAPERED_SINC = 1, 2, 3
TAPER_FIX = 0x100  # OR'd into TAPERED_SINC: taper exp(-(arg/a)^2) instead of the reference's exp(+(arg/a)^2)
MEM_HOST, MEM_DEVICE = 0, 1
SAMPLE_MAJOR, CHANNEL_MAJOR = 0, 1
ENGINE_AUTO, ENGINE_FP32, ENGINE_TC_BF16, ENGINE_TC_F16 = 0, 1, 2, 3
TC_WEIGHTS_AUTO, TC_WEIGHTS_ENTRIES, TC_WEIGHTS_DIRECT = 0, 1, 2

STATUS = {0: "HCG_OK", 1: "HCG_EINVAL", 2: "HCG_ENOMEM", 3: "HCG_ETIMEOUT", 4: "HCG_EDEVICE", 5: "HCG_EIO",
          6: "HCG_EUNSUPPORTED", 7: "HCG_ESTATE"}


class HcgError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__("%s: %s" % (STATUS.get(status, status), msg))
        self.status = status


class Job(C.Structure):
    _fields_ = [("field", C.c_void_p), ("target", C.c_void_p), ("cube", C.c_void_p), ("weights", C.c_void_p),
                ("layout", C.c_int)]


class Info(C.Structure):
    _fields_ = [("nside", C.c_uint64), ("npix", C.c_uint64), ("firstring", C.c_uint64), ("usedrings", C.c_uint64),
                ("resolution", C.c_double), ("disc_size", C.c_double), ("kernel_param0", C.c_double),
                ("sphere_radius", C.c_double)]


class Tuning(C.Structure):
    _fields_ = [("shape", C.c_int), ("prefetch", C.c_int), ("strip", C.c_int), ("ms_shape", C.c_float * 6),
                ("ms_prefetch", C.c_float * 5), ("ms_strip", C.c_float * 5), ("ms_best", C.c_float),
                ("spread", C.c_float)]


class BatchTuning(C.Structure):
    _fields_ = [("channel_class", C.c_int), ("shape", C.c_int), ("jobs", C.c_uint32), ("ms", C.c_float * 4),
                ("spread", C.c_float)]


BATCH_SHAPES = 4  # hcg_batch_set_shape: 0: 256 ch x 32 slots x 4 stages, 1: 256 x 64 x 2, 2: 128 x 64 x 3, 3: 64 x 64 x 4

TUNE_PREFETCH = (0, 2, 4, 6, 8)
TUNE_STRIP = (0, 4, 8, 16, 32)


class Stats(C.Structure):
    _fields_ = [("pairs_candidate", C.c_uint64), ("pairs_within", C.c_uint64), ("ring_skips", C.c_uint64),
                ("hard_roundings", C.c_uint64), ("ms_total", C.c_double), ("ms_phase", C.c_double * 4),
                ("tc_macs", C.c_uint64)]


EXPORTS = {
    "hcg_status_string": ([C.c_int], C.c_char_p),
    "hcg_context_create": ([C.c_int, C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
    "hcg_context_destroy": ([C.c_void_p], C.c_int),
    "hcg_last_error": ([C.c_void_p], C.c_char_p),
    "hcg_prepare_grid_kernel": ([C.c_void_p, C.c_uint32, C.c_void_p, C.c_double, C.c_double], C.c_int),
    "hcg_get_info": ([C.c_void_p, C.c_void_p, C.POINTER(Info)], C.c_int),
    "hcg_field_create": ([C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                          C.POINTER(C.c_void_p)], C.c_int),
    "hcg_field_set_spectra": ([C.c_void_p, C.c_uint32, C.c_void_p, C.c_int, C.c_int], C.c_int),
    "hcg_field_split_spectra": ([C.c_void_p, C.c_int, C.c_int], C.c_int),
    "hcg_tc_set_config": ([C.c_void_p, C.c_int, C.c_int], C.c_int),
    "hcg_tc_set_weights": ([C.c_void_p, C.c_int], C.c_int),
    "hcg_autotune": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
    "hcg_autotune_ex": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p], C.c_int),
    "hcg_tc_set_pipeline": ([C.c_void_p, C.c_int, C.c_int, C.c_int], C.c_int),
    "hcg_field_sorted": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "hcg_field_band_samples": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p],
                               C.c_int),
    "hcg_field_destroy": ([C.c_void_p], C.c_int),
    "hcg_field_share": ([C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
    "hcg_target_create": ([C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_int,
                           C.POINTER(C.c_void_p)], C.c_int),
    "hcg_target_from_header": ([C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_void_p)], C.c_int),
    "hcg_target_coords": ([C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p],
                          C.c_int),
    "hcg_target_destroy": ([C.c_void_p], C.c_int),
    "hcg_header_coords": ([C.c_char_p, C.c_size_t, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_void_p,
                           C.c_void_p], C.c_int),
    "hcg_grid": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int], C.c_int),
    "hcg_grid_planes": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_int,
                         C.c_void_p, C.c_int, C.c_uint32], C.c_int),
    "hcg_get_stats": ([C.c_void_p, C.POINTER(Stats)], C.c_int),
    "hcg_synchronize": ([C.c_void_p], C.c_int),
    "hcg_context_trim": ([C.c_void_p], C.c_int),
    "hcg_set_entry_budget": ([C.c_void_p, C.c_uint64], C.c_int),
    "hcg_set_coarsening_factor": ([C.c_void_p, C.c_uint32], C.c_int),
    "hcg_grid_batch": ([C.c_void_p, C.c_uint32, C.c_void_p], C.c_int),
    "hcg_batch_set_shape": ([C.c_void_p, C.c_int, C.c_int], C.c_int),
    "hcg_autotune_layout": ([C.c_void_p, C.c_int], C.c_int),
    "hcg_autotune_batch": ([C.c_void_p, C.c_uint32, C.c_void_p, C.c_int, C.c_uint32, C.c_void_p,
                            C.POINTER(C.c_uint32)], C.c_int),
    "hcg_grid_noalloc": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "hcg_server_create": ([C.c_void_p, C.c_int, C.c_uint32, C.c_uint64, C.c_uint32, C.POINTER(C.c_void_p)], C.c_int),
    "hcg_server_submit": ([C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)], C.c_int),
    "hcg_server_wait": ([C.c_void_p, C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
    "hcg_server_drain": ([C.c_void_p], C.c_int),
    "hcg_server_stats": ([C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_uint64),
                          C.POINTER(C.c_uint32)], C.c_int),
    "hcg_server_destroy": ([C.c_void_p], C.c_int),
    "hcg_fits_read_samples": ([C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p,
                               C.c_void_p], C.c_int),
    "hcg_fits_read_header": ([C.c_char_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
    "hcg_fits_write_cube": ([C.c_char_p, C.c_char_p, C.c_size_t, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                             C.c_void_p, C.c_int], C.c_int),
    "hcg_fits_write_samples": ([C.c_char_p, C.c_uint64, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
}

_lib = None


def lib_path() -> str:
    """The library this process loads: HCGRID_B200_LIB when set (another
    build of the same library), else the in-tree build."""
    return os.environ.get("HCGRID_B200_LIB") or _build.LIB


def load(build_if_missing: bool = False):
    """Load libhcgrid_b200.so (optionally compiling it first)."""
    global _lib
    if _lib is None:
        path = lib_path()
        if not os.path.exists(path):
            if not build_if_missing:
                raise RuntimeError("hcgrid_b200 native library not built: %s (run python -m hcgrid_b200.build)" % path)
            _build.build()
        L = C.CDLL(path)
        for name, (args, res) in EXPORTS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _ptr(a):
    """(pointer, mem) of a numpy array or a CUDA tensor."""
    if a is None:
        return None, MEM_HOST
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return C.c_void_p(a.data_ptr()), (MEM_DEVICE if a.is_cuda else MEM_HOST)
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return C.c_void_p(a.ctypes.data), MEM_HOST


def header_coords(header: str):
    """SIN target pixel centres (degrees) of a FITS header, on the host."""
    L = load()
    hb = header.encode("ascii")
    nx, ny = C.c_uint32(), C.c_uint32()
    st = L.hcg_header_coords(hb, len(hb), C.byref(nx), C.byref(ny), None, None)
    if st != 0:
        raise HcgError(st, "header")
    x = np.empty(nx.value * ny.value)
    y = np.empty(nx.value * ny.value)
    st = L.hcg_header_coords(hb, len(hb), C.byref(nx), C.byref(ny), x.ctypes.data, y.ctypes.data)
    if st != 0:
        raise HcgError(st, "header")
    return nx.value, ny.value, x, y


def fits_read_samples(path: str):
    """(lon, lat, values[nchan, n]) of an input map in the reference's layout."""
    L = load()
    n, c = C.c_uint64(), C.c_uint32()
    st = L.hcg_fits_read_samples(path.encode(), C.byref(n), C.byref(c), None, None, None)
    if st != 0:
        raise HcgError(st, path)
    lon, lat = np.empty(n.value), np.empty(n.value)
    vals = np.empty((c.value, n.value), np.float32)
    st = L.hcg_fits_read_samples(path.encode(), C.byref(n), C.byref(c), lon.ctypes.data, lat.ctypes.data,
                                 vals.ctypes.data)
    if st != 0:
        raise HcgError(st, path)
    return lon, lat, vals


def fits_read_header(path: str) -> str:
    L = load()
    ln = C.c_size_t()
    st = L.hcg_fits_read_header(path.encode(), None, 0, C.byref(ln))
    if st != 0:
        raise HcgError(st, path)
    buf = C.create_string_buffer(ln.value + 1)
    st = L.hcg_fits_read_header(path.encode(), buf, ln.value + 1, C.byref(ln))
    if st != 0:
        raise HcgError(st, path)
    return buf.value.decode("ascii")


def fits_write_cube(path: str, header: str, nx: int, ny: int, cube, weights=None, bitpix: int = -32):
    """cube: float32 [nchan, ny*nx] (channel-major)."""
    L = load()
    cube = np.ascontiguousarray(cube, np.float32)
    nchan = cube.shape[0] if cube.ndim == 2 else 1
    hb = header.encode("ascii")
    w = None if weights is None else np.ascontiguousarray(weights, np.float32)
    st = L.hcg_fits_write_cube(path.encode(), hb, len(hb), nx, ny, nchan, cube.ctypes.data,
                               None if w is None else w.ctypes.data, bitpix)
    if st != 0:
        raise HcgError(st, path)


class Context:
    """hcg_context: one CUDA device and stream plus the kernel setup."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self.L = load()
        h = C.c_void_p()
        self._check(self.L.hcg_context_create(device, C.c_void_p(stream) if stream else None, C.byref(h)), None)
        self.h = h

    def _check(self, st, h=None):
        if st != 0:
            msg = self.L.hcg_last_error(h if h is not None else getattr(self, "h", None))
            raise HcgError(st, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "h", None):
            self.L.hcg_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def prepare_grid_kernel(self, kernel_type: int, kernel_params, sphere_radius: float, hpx_max_res: float):
        """_prepare_grid_kernel; kernel_params (float64, len 3) is updated in place."""
        kp = kernel_params if isinstance(kernel_params, np.ndarray) else np.array(kernel_params, np.float64)
        assert kp.dtype == np.float64 and kp.size >= 3
        self._check(self.L.hcg_prepare_grid_kernel(self.h, kernel_type, kp.ctypes.data, sphere_radius, hpx_max_res))
        return kp

    def info(self, field=None) -> Info:
        inf = Info()
        self._check(self.L.hcg_get_info(self.h, field.h if field else None, C.byref(inf)))
        return inf

    def field(self, lon, lat, weights=None) -> "Field":
        return Field(self, lon, lat, weights)

    def target(self, nx, ny, xwcs, ywcs) -> "Target":
        return Target(self, nx, ny, xwcs, ywcs)

    def target_from_header(self, header: str) -> "Target":
        t = Target.__new__(Target)
        t.ctx = self
        h = C.c_void_p()
        hb = header.encode("ascii")
        self._check(self.L.hcg_target_from_header(self.h, hb, len(hb), C.byref(h)))
        t.h = h
        nx, ny = C.c_uint32(), C.c_uint32()
        self._check(self.L.hcg_target_coords(h, C.byref(nx), C.byref(ny), None, None))
        t.nx, t.ny = nx.value, ny.value
        return t

    def grid(self, field: "Field", target: "Target", cube=None, weights=None, layout: int = SAMPLE_MAJOR,
             engine: int = ENGINE_AUTO):
        """Grid and normalise. Without `cube`, returns host numpy arrays
        (cube [npix, nchan] or [nchan, npix], weights [npix])."""
        npix = target.nx * target.ny
        shape = (npix, field.nchan) if layout == SAMPLE_MAJOR else (field.nchan, npix)
        if cube is None:
            cube = np.empty(shape, np.float32)
            weights = np.empty(npix, np.float32)
        cp, mem = _ptr(cube)
        wp, _ = _ptr(weights)
        self._check(self.L.hcg_grid(self.h, field.h, target.h, cp, layout, wp, mem, engine))
        return cube, weights

    def grid_planes(self, geometry: "Field", target: "Target", planes, cube=None, weights=None,
                    layout: int = CHANNEL_MAJOR, engine: int = ENGINE_AUTO, block: int = 0):
        """Host channel planes [nchan, n] in, host cube out, pipelined in
        blocks of channels (hcg_grid_planes). Without `cube`, returns numpy
        arrays (cube [nchan, npix] or [npix, nchan], weights [npix])."""
        if hasattr(planes, "is_cuda") and planes.is_cuda:
            raise ValueError("planes must be host memory")
        nchan = planes.shape[0]
        npix = target.nx * target.ny
        shape = (npix, nchan) if layout == SAMPLE_MAJOR else (nchan, npix)
        if cube is None:
            cube = np.empty(shape, np.float32)
            weights = np.empty(npix, np.float32)
        pp, _ = _ptr(planes)
        cp, cmem = _ptr(cube)
        wp, wmem = _ptr(weights)
        if cmem != MEM_HOST or (weights is not None and wmem != MEM_HOST):
            raise ValueError("cube and weights must be host memory")
        self._check(self.L.hcg_grid_planes(self.h, geometry.h, target.h, pp, nchan, cp, layout, wp, engine, block))
        return cube, weights

    def stats(self) -> Stats:
        s = Stats()
        self._check(self.L.hcg_get_stats(self.h, C.byref(s)))
        return s

    def synchronize(self):
        self._check(self.L.hcg_synchronize(self.h))

    def trim(self):
        """Return the device memory the context's pool keeps for reuse."""
        self._check(self.L.hcg_context_trim(self.h))

    def tc_set_config(self, config: int, channel_class: int = -1):
        self._check(self.L.hcg_tc_set_config(self.h, channel_class, config))

    def tc_set_weights(self, mode: int):
        """How the tensor-core engines build weight operands: TC_WEIGHTS_AUTO,
        TC_WEIGHTS_ENTRIES (FP64 weight pass) or TC_WEIGHTS_DIRECT (evaluated in
        the kernel)."""
        self._check(self.L.hcg_tc_set_weights(self.h, mode))

    def tc_set_pipeline(self, prefetch: int = -1, strip: int = -1, channel_class: int = -1):
        """Prefetch distance (chunks) and persistent tile walk (strip width in
        tiles, 0: rows) of the tensor-core engine; -1 restores the default."""
        self._check(self.L.hcg_tc_set_pipeline(self.h, channel_class, prefetch, strip))

    def autotune_layout(self, layout: int):
        """Cube layout the single-job autotuners time (SAMPLE_MAJOR by default)."""
        self._check(self.L.hcg_autotune_layout(self.h, layout))

    def autotune_ex(self, field: "Field", target: "Target", reps: int = 3) -> dict:
        """The full search: shape, then prefetch distance, then tile walk."""
        t = Tuning()
        self._check(self.L.hcg_autotune_ex(self.h, field.h, target.h, reps, C.byref(t)))
        return {"shape": t.shape, "prefetch": t.prefetch, "strip": t.strip,
                "ms_shape": [round(x, 3) for x in t.ms_shape],
                "ms_prefetch": dict(zip(TUNE_PREFETCH, [round(x, 3) for x in t.ms_prefetch])),
                "ms_strip": dict(zip(TUNE_STRIP, [round(x, 3) for x in t.ms_strip])),
                "ms_best": round(t.ms_best, 3), "spread": round(t.spread, 4), "reps": reps}

    def autotune(self, field: "Field", target: "Target", reps: int = 2):
        """Time each tensor-core pipeline shape on (field, target); keeps and
        returns the fastest with the per-shape best times (ms)."""
        best = C.c_int()
        ms = (C.c_float * 6)()
        self._check(self.L.hcg_autotune(self.h, field.h, target.h, reps, C.byref(best), ms))
        return best.value, list(ms)

    def grid_batch(self, jobs):
        """jobs: list of (field, target, cube_tensor, weights_tensor_or_None, layout) with CUDA tensors."""
        arr = (Job * len(jobs))()
        for i, (f, t, cube, w, layout) in enumerate(jobs):
            if not (hasattr(cube, "is_cuda") and cube.is_cuda):
                raise ValueError("batch outputs must be CUDA tensors")
            arr[i] = Job(f.h.value, t.h.value, cube.data_ptr(), w.data_ptr() if w is not None else None, layout)
        self._check(self.L.hcg_grid_batch(self.h, len(jobs), arr))

    def batch_set_shape(self, shape: int, channel_class: int = -1):
        """Pipeline shape of the batch pass's tensor-core kernel (0-3) for a
        channel class (-1: every class); shape -1 restores the default."""
        self._check(self.L.hcg_batch_set_shape(self.h, channel_class, shape))

    def autotune_batch(self, jobs, reps: int = 3) -> list:
        """hcg_autotune_batch over `jobs` (as for grid_batch): per channel class
        present, the shape chosen, its ms per shape and spread."""
        arr = (Job * len(jobs))()
        for i, (f, t, cube, w, layout) in enumerate(jobs):
            arr[i] = Job(f.h.value, t.h.value, cube.data_ptr(), w.data_ptr() if w is not None else None, layout)
        out = (BatchTuning * 8)()
        n = C.c_uint32()
        self._check(self.L.hcg_autotune_batch(self.h, len(jobs), arr, reps, 8, out, C.byref(n)))
        return [{"channel_class": out[i].channel_class, "shape": out[i].shape, "jobs": out[i].jobs,
                 "ms": [round(x, 4) for x in out[i].ms], "spread": round(out[i].spread, 4)} for i in range(n.value)]

    def set_entry_budget(self, nbytes: int):
        self._check(self.L.hcg_set_entry_budget(self.h, nbytes))

    def set_coarsening_factor(self, factor: int):
        """HCGrid's coarsening factor (1-3): runs of `factor` pixels along a
        row take the candidate windows of the run's first pixel."""
        self._check(self.L.hcg_set_coarsening_factor(self.h, factor))


class Server:
    """hcg_server: continuous-batching request loop over `lanes` contexts."""

    def __init__(self, ctx: Context, lanes: int = 2, hbm_budget: int = 120 << 30, max_batch: int = 64,
                 device: int = 0):
        self.ctx = ctx
        h = C.c_void_p()
        ctx._check(ctx.L.hcg_server_create(ctx.h, device, lanes, hbm_budget, max_batch, C.byref(h)))
        self.h = h
        self._keep = {}

    def submit(self, field, target, cube, weights=None, layout: int = SAMPLE_MAJOR, footprint: int = 0) -> int:
        job = Job(field.h.value, target.h.value, cube.data_ptr(), weights.data_ptr() if weights is not None else None,
                  layout)
        t = C.c_uint64()
        st = self.ctx.L.hcg_server_submit(self.h, C.byref(job), footprint, C.byref(t))
        if st != 0:
            raise HcgError(st, "submit")
        self._keep[t.value] = (cube, weights)
        return t.value

    def wait(self, ticket: int):
        lat, q = C.c_double(), C.c_double()
        st = self.ctx.L.hcg_server_wait(self.h, ticket, C.byref(lat), C.byref(q))
        self._keep.pop(ticket, None)
        if st != 0:
            raise HcgError(st, "job %d" % ticket)
        return lat.value, q.value

    def drain(self):
        st = self.ctx.L.hcg_server_drain(self.h)
        if st != 0:
            raise HcgError(st, "drain")

    def stats(self):
        p50, p99, n, b = C.c_double(), C.c_double(), C.c_uint64(), C.c_uint32()
        self.ctx.L.hcg_server_stats(self.h, C.byref(p50), C.byref(p99), C.byref(n), C.byref(b))
        return {"p50_s": p50.value, "p99_s": p99.value, "jobs": n.value, "batches": b.value}

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.hcg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Field:
    """hcg_field: sorted samples, ring LUT and resident spectra."""

    def __init__(self, ctx: Context, lon, lat, weights=None):
        self.ctx = ctx
        self.n = len(lon)
        lp, mem = _ptr(lon)
        bp, _ = _ptr(lat)
        wp, _ = _ptr(weights)
        h = C.c_void_p()
        ctx._check(ctx.L.hcg_field_create(ctx.h, self.n, lp, bp, wp, mem, C.byref(h)))
        self.h = h
        self.nchan = 0

    def set_spectra(self, values, layout: int = SAMPLE_MAJOR):
        vp, mem = _ptr(values)
        if layout == SAMPLE_MAJOR:
            nchan = 1 if len(values.shape) == 1 else values.shape[1]
        else:
            nchan = values.shape[0]
        self.ctx._check(self.ctx.L.hcg_field_set_spectra(self.h, nchan, vp, layout, mem))
        self.nchan = nchan

    def split_spectra(self, engine: int = ENGINE_TC_F16, keep_fp32: bool = True):
        """16-bit hi/lo copy of the spectra for a tensor-core engine."""
        self.ctx._check(self.ctx.L.hcg_field_split_spectra(self.h, engine, 1 if keep_fp32 else 0))

    def share(self) -> "Field":
        """Another handle on this field's resident geometry, without spectra."""
        f = Field.__new__(Field)
        f.ctx, f.n, f.nchan = self.ctx, self.n, 0
        h = C.c_void_p()
        self.ctx._check(self.ctx.L.hcg_field_share(self.h, C.byref(h)))
        f.h = h
        return f

    def sorted(self):
        inf = self.ctx.info(self)
        keys = np.empty(self.n + 1, np.uint64)
        perm = np.empty(self.n, np.uint32)
        lut = np.empty(inf.usedrings + 1, np.uint32)
        self.ctx._check(self.ctx.L.hcg_field_sorted(self.h, keys.ctypes.data, perm.ctypes.data, lut.ctypes.data))
        return keys, perm, lut, inf.firstring, inf.usedrings

    def band_samples(self, target: "Target", y0: int, y1: int):
        """Sorted positions [s0, s1) whose samples alone grid target rows
        [y0, y1) as this field does (hcg_field_band_samples)."""
        s0, s1 = C.c_uint64(), C.c_uint64()
        self.ctx._check(self.ctx.L.hcg_field_band_samples(self.ctx.h, self.h, target.h, y0, y1, C.byref(s0),
                                                          C.byref(s1)))
        return s0.value, s1.value

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.hcg_field_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Target:
    """hcg_target: target pixel centres (degrees), yy*nx + xx order."""

    def __init__(self, ctx: Context, nx: int, ny: int, xwcs, ywcs):
        self.ctx = ctx
        self.nx, self.ny = nx, ny
        xp, mem = _ptr(xwcs)
        yp, _ = _ptr(ywcs)
        h = C.c_void_p()
        ctx._check(ctx.L.hcg_target_create(ctx.h, nx, ny, xp, yp, mem, C.byref(h)))
        self.h = h

    def coords(self):
        x = np.empty(self.nx * self.ny)
        y = np.empty(self.nx * self.ny)
        self.ctx._check(self.ctx.L.hcg_target_coords(self.h, None, None, x.ctypes.data, y.ctypes.data))
        return x, y

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.hcg_target_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
