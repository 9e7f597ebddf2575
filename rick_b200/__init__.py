"""rick_b200 -- B200-native imaging hot path of RICK (Radio Imaging Code Kernels).

Python mirror of the reference's operator interface for this path, over the C ABI
of ``librick_b200.so`` (include/rick_b200.h):

* :func:`wstack` and :func:`phase_correction` keep the argument contracts of
  w-stacking.h:39-57 and :70-83 (host arrays, accumulate semantics);
* :func:`fft_planes` is the arithmetic of fftw_data (fourier_transform.c:13-93);
* :class:`Plan` is the device-resident pipeline (binning -> tiled gridding ->
  batched inverse FFT -> fused w-correction), taking device pointers (torch
  CUDA tensors or raw addresses) and a CUDA stream.

There is no CPU fallback: every call runs the sm_100a kernels of the library,
and importing the module raises if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librick_b200.so")

OK = 0
ERR_NOT_ENOUGH_MEM = 3
ERR_INVALID_ARG = 16
ERR_CUDA = 17
ERR_CUFFT = 18
ERR_IO = 19
ERR_UNSUPPORTED = 20
ERR_BUDGET = 21
ERR_CANCELLED = 22
ERR_NO_ACCELERATORS_FOUND = 255

KERNELS = {"gauss": 0, "gauss_hi": 1, "kaiser_bessel": 2}
PRECISIONS = {"fp64": 0, "mixed": 1}
ROWS_ALL, ROWS_SECTOR0 = 0, 1


class RickError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: status {status} ({status_string(status)}) {detail}".strip())


class PlanDesc(C.Structure):
    _fields_ = [("grid_size_x", C.c_int), ("grid_size_y", C.c_int), ("num_w_planes", C.c_int),
                ("w_support", C.c_int), ("kernel", C.c_int), ("precision", C.c_int),
                ("phase_on", C.c_int), ("device", C.c_int), ("max_rows", C.c_uint64),
                ("freq_per_chan", C.c_uint32), ("polarizations", C.c_uint32),
                ("w_first", C.c_int), ("w_count", C.c_int), ("normalize_uvw", C.c_int)]


class PlanStats(C.Structure):
    _fields_ = [("rows_in", C.c_uint64), ("rows_gridded", C.c_uint64),
                ("rows_dropped", C.c_uint64), ("records", C.c_uint64),
                ("work_items", C.c_uint64), ("device_bytes", C.c_uint64),
                ("fft_rows", C.c_uint64), ("rows_other_shard", C.c_uint64)]


class JobDesc(C.Structure):
    _fields_ = [("grid_size_x", C.c_int), ("grid_size_y", C.c_int), ("num_w_planes", C.c_int),
                ("w_support", C.c_int), ("kernel", C.c_int), ("num_rows", C.c_uint64),
                ("freq_per_chan", C.c_uint32), ("polarizations", C.c_uint32),
                ("row_selection", C.c_int), ("phase_on", C.c_int), ("resolution", C.c_double),
                ("wmin", C.c_double), ("wmax", C.c_double), ("uu", C.c_void_p),
                ("vv", C.c_void_p), ("ww", C.c_void_p), ("weight", C.c_void_p),
                ("vis_real", C.c_void_p), ("vis_img", C.c_void_p), ("image_real", C.c_void_p),
                ("image_imag", C.c_void_p)]


class BatchTuning(C.Structure):
    _fields_ = [("max_chunk", C.c_uint32), ("grid_blocks_per_sm", C.c_int),
                ("planes_in_flight", C.c_int)]


class ServerDesc(C.Structure):
    _fields_ = [("device", C.c_int), ("precision", C.c_int), ("hbm_budget", C.c_uint64),
                ("max_batch_jobs", C.c_int), ("streams", C.c_int), ("solo_vis", C.c_uint64)]


class JobResult(C.Structure):
    _fields_ = [("status", C.c_int), ("queue_ms", C.c_double), ("latency_ms", C.c_double),
                ("batch_id", C.c_uint64), ("batch_jobs", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("jobs_submitted", C.c_uint64), ("jobs_done", C.c_uint64),
                ("vis_done", C.c_uint64), ("batches", C.c_uint64), ("bytes_in_use", C.c_uint64),
                ("peak_bytes", C.c_uint64), ("jobs_waiting", C.c_uint64)]


_lib = None
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_vp = C.c_void_p


def lib():
    """The loaded ``librick_b200.so`` with prototypes set (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"rick_b200: {LIB_PATH} is missing; build it with "
                          f"`make -C rick_b200/csrc` (there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    L.wstack.argtypes = [C.c_int, C.c_uint, C.c_uint, C.c_uint, _dp, _dp, _dp, _fp, _fp, _fp,
                         C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _dp, C.c_int, C.c_int]
    L.wstack.restype = None
    L.phase_correction.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_double, C.c_double, C.c_double, C.c_int, C.c_int]
    L.phase_correction.restype = None
    L.rick_fft_planes.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_int]
    for name, args in [("rick_set_kernel", [C.c_int]), ("rick_set_phase_on", [C.c_int]),
                       ("rick_set_device", [C.c_int]), ("rick_last_status", [])]:
        getattr(L, name).argtypes = args
        getattr(L, name).restype = C.c_int
    L.rick_status_string.argtypes = [C.c_int]
    L.rick_status_string.restype = C.c_char_p
    L.rick_last_error_message.argtypes = []
    L.rick_last_error_message.restype = C.c_char_p
    L.rick_plan_create.argtypes = [C.POINTER(_vp), C.POINTER(PlanDesc)]
    L.rick_plan_destroy.argtypes = [_vp]
    L.rick_plan_footprint.argtypes = [C.POINTER(PlanDesc), C.POINTER(C.c_uint64)]
    rows7 = [_vp, _vp, _vp, _vp, _vp, _vp]
    L.rick_plan_grid.argtypes = [_vp, C.c_uint64] + rows7 + [C.c_int, _vp]
    L.rick_plan_fft.argtypes = [_vp, _vp]
    L.rick_plan_phase.argtypes = [_vp, C.c_double, C.c_double, C.c_double, _vp, _vp, C.c_int, _vp]
    L.rick_plan_image.argtypes = ([_vp, C.c_uint64] + rows7 +
                                  [C.c_int, C.c_double, C.c_double, C.c_double, _vp, _vp, _vp])
    L.rick_plan_image_host.argtypes = ([_vp, C.c_uint64] + rows7 +
                                       [C.c_int, C.c_double, C.c_double, C.c_double, _vp, _vp])
    L.rick_plan_ingest_begin.argtypes = [_vp, C.c_uint64, _vp, _vp, _vp, _vp, C.c_int]
    L.rick_plan_ingest_samples.argtypes = [_vp, C.c_uint64, C.c_uint64, _vp, _vp]
    L.rick_plan_ingest_end.argtypes = [_vp, C.c_double, C.c_double, C.c_double, _vp, _vp]
    L.rick_host_alloc.argtypes = [C.POINTER(_vp), C.c_uint64]
    L.rick_host_free.argtypes = [_vp]
    L.rick_plan_export_cube.argtypes = [_vp, _vp, C.c_int, _vp]
    L.rick_plan_import_cube.argtypes = [_vp, _vp, C.c_int, _vp]
    L.rick_plan_get_stats.argtypes = [_vp, C.POINTER(PlanStats)]
    L.rick_plan_set_timing.argtypes = [_vp, C.c_int]
    L.rick_plan_stage_ms.argtypes = [_vp, C.POINTER(C.c_float), C.c_int]
    L.rick_batch_footprint.argtypes = [C.POINTER(JobDesc), C.c_int, C.c_int,
                                       C.POINTER(C.c_uint64)]
    L.rick_batch_create.argtypes = [C.POINTER(_vp), C.POINTER(JobDesc), C.c_int, C.c_int, C.c_int,
                                    C.POINTER(BatchTuning)]
    L.rick_batch_run.argtypes = [_vp, _vp]
    L.rick_batch_get_tuning.argtypes = [_vp, C.POINTER(BatchTuning)]
    L.rick_batch_get_stats.argtypes = [_vp, C.POINTER(PlanStats)]
    L.rick_batch_destroy.argtypes = [_vp]
    L.rick_batch_kernels_per_run.argtypes = [_vp, C.POINTER(C.c_uint32)]
    L.rick_server_create.argtypes = [C.POINTER(_vp), C.POINTER(ServerDesc)]
    L.rick_server_submit.argtypes = [_vp, C.POINTER(JobDesc), C.POINTER(C.c_uint64)]
    L.rick_server_wait.argtypes = [_vp, C.c_uint64, C.c_double, C.POINTER(JobResult)]
    L.rick_server_get_stats.argtypes = [_vp, C.POINTER(ServerStats)]
    L.rick_server_destroy.argtypes = [_vp]
    L.rick_server_cancel.argtypes = [_vp, C.c_uint64]
    L.rick_dropin_counters.argtypes = [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.rick_dropin_release.argtypes = []
    L.rick_server_shutdown.argtypes = [_vp, C.c_int]
    L.rick_normalize_uvw.argtypes = [C.c_uint64, _vp, _vp, _vp, _vp, _vp]
    L.rick_kernel_names.argtypes = [C.POINTER(C.c_char_p), C.c_int]
    L.rick_launch_count.argtypes = []
    L.rick_launch_count.restype = C.c_ulonglong
    for fn in ["rick_plan_create", "rick_plan_destroy", "rick_plan_footprint", "rick_plan_grid",
               "rick_plan_fft", "rick_plan_phase", "rick_plan_image", "rick_plan_image_host",
               "rick_plan_export_cube", "rick_plan_import_cube", "rick_plan_get_stats",
               "rick_kernel_names", "rick_fft_planes", "rick_plan_set_timing",
               "rick_plan_stage_ms", "rick_batch_footprint", "rick_batch_create",
               "rick_batch_run", "rick_batch_get_tuning", "rick_batch_get_stats",
               "rick_batch_destroy", "rick_batch_kernels_per_run", "rick_server_create",
               "rick_server_submit", "rick_server_wait", "rick_server_get_stats",
               "rick_server_destroy", "rick_server_cancel", "rick_server_shutdown",
               "rick_dropin_counters", "rick_dropin_release",
               "rick_normalize_uvw", "rick_plan_ingest_begin",
               "rick_plan_ingest_samples", "rick_plan_ingest_end", "rick_host_alloc",
               "rick_host_free"]:
        getattr(L, fn).restype = C.c_int
    _lib = L
    return L


def status_string(status: int) -> str:
    return lib().rick_status_string(status).decode()


def last_error() -> str:
    return lib().rick_last_error_message().decode(errors="replace")


def check(status: int, where: str) -> None:
    if status != OK:
        raise RickError(status, where, last_error())


def kernel_names() -> list[str]:
    arr = (C.c_char_p * 64)()
    n = lib().rick_kernel_names(arr, 64)
    return [arr[i].decode() for i in range(n)]


def launch_count() -> int:
    return int(lib().rick_launch_count())


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ---- drop-in operators (host arrays) --------------------------------------

def set_kernel(kernel: str) -> None:
    check(lib().rick_set_kernel(KERNELS[kernel]), "rick_set_kernel")


def set_phase_on(on: bool) -> None:
    check(lib().rick_set_phase_on(int(bool(on))), "rick_set_phase_on")


def wstack(num_w_planes, num_points, freq_per_chan, polarizations, uu, vv, ww, vis_real,
           vis_img, weight, dx, dw, w_support, grid_size_x, grid_size_y, grid, num_threads=1,
           rank=0):
    """w-stacking.h:39-57: adds the gridded rows into ``grid`` (float64, in place)."""
    if grid.dtype != np.float64 or not grid.flags.c_contiguous:
        raise ValueError("grid must be a C-contiguous float64 array")
    lib().wstack(num_w_planes, num_points, freq_per_chan, polarizations, _c(uu, np.float64),
                 _c(vv, np.float64), _c(ww, np.float64), _c(vis_real, np.float32),
                 _c(vis_img, np.float32), _c(weight, np.float32), dx, dw, w_support,
                 grid_size_x, grid_size_y, grid, num_threads, rank)
    check(lib().rick_last_status(), "wstack")
    return grid


def phase_correction(gridss, image_real, image_imag, xaxis, yaxis, num_w_planes, xaxistot,
                     yaxistot, resolution, wmin, wmax, num_threads=1, rank=0):
    """w-stacking.h:70-83: adds the w-corrected plane sum into the images (in place)."""
    for a in (image_real, image_imag):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError("images must be C-contiguous float64 arrays")
    lib().phase_correction(_c(gridss, np.float64), image_real, image_imag, xaxis, yaxis,
                           num_w_planes, xaxistot, yaxistot, resolution, wmin, wmax, num_threads,
                           rank)
    check(lib().rick_last_status(), "phase_correction")
    return image_real, image_imag


def dropin_counters() -> dict:
    """Plans the drop-ins created and their row-buffer allocations so far."""
    a, b = C.c_uint64(), C.c_uint64()
    check(lib().rick_dropin_counters(C.byref(a), C.byref(b)), "rick_dropin_counters")
    return {"plans_created": int(a.value), "row_allocations": int(b.value)}


def dropin_release() -> None:
    """Frees the drop-ins' cached plans and buffers on every device."""
    check(lib().rick_dropin_release(), "rick_dropin_release")


def fft_planes(grid, num_w_planes, grid_size_x, grid_size_y, out=None):
    """fourier_transform.c:13-93: per plane FFTW_BACKWARD / (Nx*Ny)."""
    grid = _c(grid, np.float64)
    if out is None:
        out = np.empty_like(grid)
    check(lib().rick_fft_planes(grid, out, num_w_planes, grid_size_x, grid_size_y),
          "rick_fft_planes")
    return out


# ---- plan (device-resident pipeline) -------------------------------------

def _ptr(x) -> Optional[int]:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    raise TypeError(f"cannot take the address of {type(x)}")


def _stream(stream) -> Optional[int]:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


@dataclass
class Geometry:
    grid_size_x: int
    grid_size_y: int
    num_w_planes: int
    w_support: int = 7
    kernel: str = "kaiser_bessel"
    precision: str = "fp64"
    phase_on: bool = True


class Plan:
    """Device-resident imaging plan (rick_plan_* in include/rick_b200.h)."""

    def __init__(self, geom: Geometry, max_rows: int, freq_per_chan: int, polarizations: int,
                 device: int = -1, planes: Optional[tuple] = None, normalize_uvw: bool = False):
        """``planes=(w_first, w_count)`` makes the plan one w-plane shard of the cube;
        ``normalize_uvw`` normalises the rows in place first (gridding.c:21-83)."""
        self.geom = geom
        w_first, w_count = planes if planes is not None else (0, 0)
        self.desc = PlanDesc(geom.grid_size_x, geom.grid_size_y, geom.num_w_planes,
                             geom.w_support, KERNELS[geom.kernel], PRECISIONS[geom.precision],
                             int(geom.phase_on), device, max_rows, freq_per_chan, polarizations,
                             w_first, w_count, int(bool(normalize_uvw)))
        h = _vp()
        check(lib().rick_plan_create(C.byref(h), C.byref(self.desc)), "rick_plan_create")
        self._h = h

    @staticmethod
    def footprint(geom: Geometry, max_rows: int, freq_per_chan: int, polarizations: int) -> int:
        d = PlanDesc(geom.grid_size_x, geom.grid_size_y, geom.num_w_planes, geom.w_support,
                     KERNELS[geom.kernel], PRECISIONS[geom.precision], int(geom.phase_on), -1,
                     max_rows, freq_per_chan, polarizations)
        b = C.c_uint64(0)
        check(lib().rick_plan_footprint(C.byref(d), C.byref(b)), "rick_plan_footprint")
        return int(b.value)

    def close(self):
        if getattr(self, "_h", None):
            lib().rick_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _rows(self, rows):
        uu, vv, ww, weight, vis_re, vis_im = rows
        return [_ptr(uu), _ptr(vv), _ptr(ww), _ptr(weight), _ptr(vis_re), _ptr(vis_im)]

    def grid(self, nrows, rows, selection=ROWS_ALL, stream=None):
        check(lib().rick_plan_grid(self._h, nrows, *self._rows(rows), selection, _stream(stream)),
              "rick_plan_grid")

    def fft(self, stream=None):
        check(lib().rick_plan_fft(self._h, _stream(stream)), "rick_plan_fft")

    def phase(self, resolution, wmin, wmax, image_re, image_im, accumulate=False, stream=None):
        check(lib().rick_plan_phase(self._h, resolution, wmin, wmax, _ptr(image_re),
                                    _ptr(image_im), int(accumulate), _stream(stream)),
              "rick_plan_phase")

    def image(self, nrows, rows, resolution, wmin, wmax, image_re, image_im,
              selection=ROWS_SECTOR0, stream=None):
        check(lib().rick_plan_image(self._h, nrows, *self._rows(rows), selection, resolution,
                                    wmin, wmax, _ptr(image_re), _ptr(image_im), _stream(stream)),
              "rick_plan_image")

    def image_host(self, nrows, rows, resolution, wmin, wmax, image_re, image_im,
                   selection=ROWS_SECTOR0):
        check(lib().rick_plan_image_host(self._h, nrows, *self._rows(rows), selection,
                                         resolution, wmin, wmax, _ptr(image_re), _ptr(image_im)),
              "rick_plan_image_host")

    def ingest(self, nrows, rows, resolution, wmin, wmax, image_re, image_im,
               selection=ROWS_ALL, slice_rows=65536):
        """Streaming ingest (rick_plan_ingest_*) of host rows: u, v, w and weights
        first, then the samples in slices of ``slice_rows`` rows."""
        uu, vv, ww, wt, vr, vi = rows
        nv = self.desc.freq_per_chan * self.desc.polarizations
        check(lib().rick_plan_ingest_begin(self._h, nrows, _ptr(uu), _ptr(vv), _ptr(ww),
                                           _ptr(wt), selection), "rick_plan_ingest_begin")
        for r0 in range(0, nrows, slice_rows):
            n = min(slice_rows, nrows - r0)
            check(lib().rick_plan_ingest_samples(self._h, r0, n, _ptr(vr) + 4 * r0 * nv,
                                                 _ptr(vi) + 4 * r0 * nv),
                  "rick_plan_ingest_samples")
        check(lib().rick_plan_ingest_end(self._h, resolution, wmin, wmax, _ptr(image_re),
                                         _ptr(image_im)), "rick_plan_ingest_end")

    def export_cube(self, dst, dst_is_host, stream=None):
        check(lib().rick_plan_export_cube(self._h, _ptr(dst), int(dst_is_host), _stream(stream)),
              "rick_plan_export_cube")

    def import_cube(self, src, src_is_host, stream=None):
        check(lib().rick_plan_import_cube(self._h, _ptr(src), int(src_is_host), _stream(stream)),
              "rick_plan_import_cube")

    STAGES = ("bin_count", "bin_scatter", "cube_zero", "grid", "fft", "phase")

    def set_timing(self, on: bool = True):
        check(lib().rick_plan_set_timing(self._h, int(on)), "rick_plan_set_timing")

    def stage_ms(self) -> dict:
        arr = (C.c_float * len(self.STAGES))()
        check(lib().rick_plan_stage_ms(self._h, arr, len(self.STAGES)), "rick_plan_stage_ms")
        return {k: float(arr[i]) for i, k in enumerate(self.STAGES) if arr[i] >= 0}

    def stats(self) -> dict:
        s = PlanStats()
        check(lib().rick_plan_get_stats(self._h, C.byref(s)), "rick_plan_get_stats")
        return {k: int(getattr(s, k)) for k, _ in PlanStats._fields_}


# ---- batched imaging --------------------------------------------------------

@dataclass
class Job:
    """One imaging job of a batch: geometry, device rows (uu, vv, ww, weights,
    vis_re, vis_im as torch CUDA tensors or addresses) and device image planes."""
    geom: Geometry
    nrows: int
    freq_per_chan: int
    polarizations: int
    rows: tuple
    resolution: float
    wmin: float
    wmax: float
    image_re: object
    image_im: object
    selection: int = ROWS_ALL

    def desc(self) -> JobDesc:
        g = self.geom
        r = [_ptr(x) for x in self.rows]
        return JobDesc(g.grid_size_x, g.grid_size_y, g.num_w_planes, g.w_support,
                       KERNELS[g.kernel], self.nrows,
                       self.freq_per_chan, self.polarizations, self.selection,
                       int(bool(g.phase_on)), self.resolution, self.wmin, self.wmax, *r,
                       _ptr(self.image_re), _ptr(self.image_im))


def _descs(jobs):
    arr = (JobDesc * len(jobs))()
    for i, j in enumerate(jobs):
        arr[i] = j.desc()
    return arr


class Batch:
    """Many imaging jobs run as one launch per stage, captured in a CUDA graph
    (include/rick_b200.h, section 4).  ``tuning=None`` autotunes."""

    def __init__(self, jobs, precision="mixed", device=0, tuning: Optional[dict] = None):
        self._keep = list(jobs)  # the descriptors hold raw device addresses
        descs = _descs(self._keep)
        t = None
        if tuning is not None:
            t = BatchTuning(tuning["max_chunk"], tuning["grid_blocks_per_sm"],
                            tuning["planes_in_flight"])
        h = _vp()
        check(lib().rick_batch_create(C.byref(h), descs, len(descs), PRECISIONS[precision],
                                      device, C.byref(t) if t is not None else None),
              "rick_batch_create")
        self._h = h

    @staticmethod
    def footprint(jobs, precision="mixed") -> int:
        descs = _descs(list(jobs))
        b = C.c_uint64()
        check(lib().rick_batch_footprint(descs, len(descs), PRECISIONS[precision], C.byref(b)),
              "rick_batch_footprint")
        return int(b.value)

    def run(self, stream=None):
        check(lib().rick_batch_run(self._h, _stream(stream)), "rick_batch_run")

    def tuning(self) -> dict:
        t = BatchTuning()
        check(lib().rick_batch_get_tuning(self._h, C.byref(t)), "rick_batch_get_tuning")
        return {k: int(getattr(t, k)) for k, _ in BatchTuning._fields_}

    def kernels_per_run(self) -> int:
        k = C.c_uint32()
        check(lib().rick_batch_kernels_per_run(self._h, C.byref(k)), "rick_batch_kernels_per_run")
        return int(k.value)

    def stats(self) -> dict:
        s = PlanStats()
        check(lib().rick_batch_get_stats(self._h, C.byref(s)), "rick_batch_get_stats")
        return {k: int(getattr(s, k)) for k, _ in PlanStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().rick_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---- served imaging (continuous batching) ------------------------------------

class Server:
    """Request loop with continuous batching (include/rick_b200.h, section 5):
    ``submit`` queues a job and returns a ticket at once; ``wait`` blocks until
    that job's image is complete and returns its latencies."""

    def __init__(self, precision="mixed", device=0, hbm_budget=150 * 10**9, max_batch_jobs=64,
                 streams=2, solo_vis=0):
        d = ServerDesc(device, PRECISIONS[precision], int(hbm_budget), max_batch_jobs, streams,
                       int(solo_vis))
        h = _vp()
        check(lib().rick_server_create(C.byref(h), C.byref(d)), "rick_server_create")
        self._h = h
        self._keep = {}

    def submit(self, job: Job) -> int:
        t = C.c_uint64()
        d = job.desc()
        check(lib().rick_server_submit(self._h, C.byref(d), C.byref(t)), "rick_server_submit")
        self._keep[int(t.value)] = job  # the job's buffers stay alive until waited for
        return int(t.value)

    def wait(self, ticket: int, timeout_ms: float = -1.0) -> dict:
        r = JobResult()
        st = lib().rick_server_wait(self._h, ticket, timeout_ms, C.byref(r))
        self._keep.pop(ticket, None)
        check(st, "rick_server_wait")
        return {k: (float(getattr(r, k)) if k.endswith("_ms") else int(getattr(r, k)))
                for k, _ in JobResult._fields_}

    def cancel(self, ticket: int) -> bool:
        """Cancels a job still waiting for admission (its wait then raises
        RickError with ERR_CANCELLED); False when it was already launched."""
        st = lib().rick_server_cancel(self._h, ticket)
        if st == ERR_INVALID_ARG:
            return False
        check(st, "rick_server_cancel")
        return True

    def shutdown(self, drain: bool = True):
        """Stops admitting jobs; with drain=False the waiting ones are cancelled
        while launched batches finish (include/rick_b200.h)."""
        check(lib().rick_server_shutdown(self._h, int(bool(drain))), "rick_server_shutdown")

    def stats(self) -> dict:
        s = ServerStats()
        check(lib().rick_server_get_stats(self._h, C.byref(s)), "rick_server_get_stats")
        return {k: int(getattr(s, k)) for k, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().rick_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def normalize_uvw(nrows, uu, vv, ww, scratch, stream=None):
    """gridding.c:21-83 in place on device rows (include/rick_b200.h);
    ``scratch``: a CUDA tensor of >= 128 bytes, its first 7 float64 values are
    then min u, v, w, max u, v, w and maxg."""
    check(lib().rick_normalize_uvw(nrows, _ptr(uu), _ptr(vv), _ptr(ww), _ptr(scratch),
                                   _stream(stream)), "rick_normalize_uvw")


def resolution_of(meta: dict) -> float:
    """gridding_cpu.c:78: resolution = 1 / max(|uvmin|, |uvmax|)."""
    return 1.0 / max(abs(meta["uvmin"]), abs(meta["uvmax"]))


def rows_read(meta: dict) -> int:
    """init.c:337-339: the last 1000 rows of a dataset are not read."""
    return max(int(meta["Nmeasures"]) - 1000, 0)
