"""deconwolf_b200 -- B200-native Richardson-Lucy / Scaled-Heavy-Ball deconvolution.

Python host side over the C ABI in include/dwcu.h (libdwcu.so, built in this
directory).  Two levels, mirroring deconwolf:

* :func:`run_method` is the ``dw_function`` call (src/dw.h:89-91): image and
  PSF go to the method as they are, exactly like ``s->fun(im, ..., psf, ...,
  s)`` in dw_run (src/dw.c:2841).
* :func:`deconvolve` mirrors the Python binding ``pydeconwolf.deconvolve``
  (src/pywrapper/src/pydeconwolf.c:284-394), i.e. dw_run around the method:
  the PSF is normalised to sum 1 (dw.c:2799, 2826), the offset (default 5) is
  added to the image before the method (dw.c:2835-2838).

There is no CPU path: without the built library or without a CUDA device the
calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = [
    "DwcuError", "Opts", "lib", "run_method", "deconvolve", "plan_size", "Job",
    "METHOD_RL", "METHOD_SHB", "ITER_ABS", "ITER_REL", "ITER_FIXED",
    "START_FLAT", "START_LP", "START_IDENTITY", "METRIC_MSE", "METRIC_IDIV",
]

HERE = os.path.dirname(os.path.abspath(__file__))
# the engine library (DWCU_LIBRARY names another build of it, e.g. one
# compiled for a subset of transform lengths)
LIB_PATH = os.environ.get("DWCU_LIBRARY") or os.path.join(HERE, "libdwcu.so")

METHOD_RL, METHOD_SHB = 0, 2
ITER_ABS, ITER_REL, ITER_FIXED = 0, 1, 2
START_FLAT, START_LP, START_IDENTITY = 0, 1, 2
METRIC_MSE, METRIC_IDIV = 0, 1

STATUS = {
    0: "SUCCESS", 1: "INVALID_VALUE", 2: "UNSUPPORTED", 3: "OUT_OF_MEMORY", 4: "CUDA",
    5: "INPUT", 6: "NOT_READY", 7: "CANCELLED", 8: "TIMEOUT", 9: "INTERNAL",
}


class DwcuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dwcu {STATUS.get(code, code)}: {msg}")
        self.code = code


class Opts(ctypes.Structure):
    """Mirror of ``dwcu_opts`` (include/dwcu.h)."""

    _fields_ = [
        ("method", ctypes.c_int32),
        ("n_iter", ctypes.c_int32),
        ("iter_type", ctypes.c_int32),
        ("maxiter", ctypes.c_int32),
        ("err_rel", ctypes.c_float),
        ("err_abs", ctypes.c_float),
        ("bg", ctypes.c_float),
        ("bg_auto", ctypes.c_int32),
        ("positivity", ctypes.c_int32),
        ("border_quality", ctypes.c_int32),
        ("start_condition", ctypes.c_int32),
        ("metric", ctypes.c_int32),
        ("alphamax", ctypes.c_float),
        ("device", ctypes.c_int32),
        ("verbosity", ctypes.c_int32),
        ("use_graph", ctypes.c_int32),
        ("iterations_done", ctypes.c_int32),
        ("error_trace", ctypes.POINTER(ctypes.c_float)),
        ("trace_capacity", ctypes.c_int32),
        ("work", ctypes.c_int64 * 3),
        ("seconds_setup", ctypes.c_double),
        ("seconds_iterate", ctypes.c_double),
        ("seconds_enqueue", ctypes.c_double),
    ]


class KernelStat(ctypes.Structure):
    """Mirror of ``dwcu_kernel_stat``."""

    _fields_ = [("name", ctypes.c_char * 40), ("launches", ctypes.c_int64),
                ("milliseconds", ctypes.c_double), ("bytes_per_launch", ctypes.c_double)]


def profile_enable(on: bool = True) -> None:
    _check(lib().dwcu_profile_enable(1 if on else 0))


def profile_collect() -> list[dict]:
    """Per-kernel-class launches, summed event milliseconds and algorithmic
    bytes per launch since the last collect (waits for the recorded work)."""
    cap = 256
    arr = (KernelStat * cap)()
    n = ctypes.c_int32()
    _check(lib().dwcu_profile_collect(arr, cap, ctypes.byref(n)))
    return [dict(name=arr[i].name.decode(), launches=int(arr[i].launches), ms=float(arr[i].milliseconds),
                 bytes_per_launch=float(arr[i].bytes_per_launch)) for i in range(min(n.value, cap))]


class Tile(ctypes.Structure):
    """dwcu_tile: struct tile of src/tiling.h:29-34 (x, y, z order)."""
    _fields_ = [("size", ctypes.c_int64 * 3), ("pos", ctypes.c_int64 * 6),
                ("xpos", ctypes.c_int64 * 6), ("xsize", ctypes.c_int64 * 3)]


class ServerStats(ctypes.Structure):
    """dwcu_server_stats."""
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("cancelled", ctypes.c_int64), ("active", ctypes.c_int64), ("queued", ctypes.c_int64),
                ("device_bytes_in_use", ctypes.c_double), ("latency_p50_s", ctypes.c_double),
                ("latency_p99_s", ctypes.c_double), ("latency_mean_s", ctypes.c_double),
                ("voxel_iterations", ctypes.c_double), ("wall_s", ctypes.c_double)]


class JobState(ctypes.Structure):
    """dwcu_job_state: a job's iteration state between iterations."""
    _fields_ = [("volume_elems", ctypes.c_int64), ("next_iter", ctypes.c_int32), ("done_iters", ctypes.c_int32),
                ("iter", ctypes.c_int32), ("error", ctypes.c_float), ("lasterror", ctypes.c_float),
                ("bg", ctypes.c_float)]


# every symbol include/dwcu.h declares
EXPORTS = [
    "dwcu_opts_init", "dwcu_deconvolve", "dwcu_deconvolve_device", "dwcu_plan_size",
    "dwcu_job_create", "dwcu_job_setup", "dwcu_job_step", "dwcu_job_done", "dwcu_job_result",
    "dwcu_job_destroy", "dwcu_job_set_stream", "dwcu_job_bytes", "dwcu_last_error",
    "dwcu_abi_version", "dwcu_device_count", "dwcu_launch_count", "dwcu_fft_r2c", "dwcu_fft_c2r",
    "dwcu_profile_enable", "dwcu_profile_collect", "dwcu_batch_run", "dwcu_psf_prepare",
    "dwcu_tiling_create", "dwcu_deconvolve_tiled", "dwcu_fft_r2c_noalloc", "dwcu_server_create",
    "dwcu_server_submit", "dwcu_server_wait", "dwcu_server_cancel", "dwcu_server_get_stats",
    "dwcu_server_destroy", "dwcu_tile_blend", "dwcu_release_cache",
    "dwcu_tune_set_mode", "dwcu_tune_get_mode", "dwcu_tune_select", "dwcu_tune_plan_count",
    "dwcu_tune_plan_info", "dwcu_tune_force", "dwcu_tune_run", "dwcu_tune_query", "dwcu_tune_clear",
    "dwcu_tune_export", "dwcu_tune_import", "dwcu_psf_prepare_device", "dwcu_selftest_bounded_wait",
    "dwcu_debug_guards", "dwcu_debug_guard_violations", "dwcu_deconvolve_slabs", "dwcu_slab_layout",
    "dwcu_job_snapshot", "dwcu_job_restore", "dwcu_slab_part_create", "dwcu_slab_part_export",
    "dwcu_slab_part_import", "dwcu_slab_part_run", "dwcu_slab_destroy",
]

# the collectives a process-per-part split calls back (dwcu_slab_sync)
SLAB_BARRIER = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p)
SLAB_ALLREDUCE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32)


class SlabSync(ctypes.Structure):
    """dwcu_slab_sync."""
    _fields_ = [("barrier", SLAB_BARRIER), ("allreduce", SLAB_ALLREDUCE), ("ctx", ctypes.c_void_p)]

# pass kinds of the autotuner (dwcu.h)
PLAN_LINES, PLAN_Y, PLAN_X = 0, 1, 2
TUNE_OFF, TUNE_MEASURE = 0, 1

_lib = None


def lib() -> ctypes.CDLL:
    """Load libdwcu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {HERE}/csrc -j8` "
                          "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    i64, i32, vp = ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p
    P_opts = ctypes.POINTER(Opts)
    L.dwcu_opts_init.argtypes = [P_opts]
    L.dwcu_opts_init.restype = None
    L.dwcu_deconvolve.argtypes = [vp, i64, i64, i64, vp, i64, i64, i64, P_opts, vp]
    L.dwcu_deconvolve.restype = ctypes.c_int
    L.dwcu_deconvolve_device.argtypes = [vp, i64, i64, i64, vp, i64, i64, i64, P_opts, vp, vp]
    L.dwcu_deconvolve_device.restype = ctypes.c_int
    L.dwcu_plan_size.argtypes = [i64, i64, i64, i64, i64, i64, i32, i32, ctypes.POINTER(i64), ctypes.POINTER(i64)]
    L.dwcu_plan_size.restype = ctypes.c_int
    L.dwcu_deconvolve_slabs.argtypes = [vp, i64, i64, i64, vp, i64, i64, i64, P_opts, i32, vp, vp]
    L.dwcu_deconvolve_slabs.restype = ctypes.c_int
    L.dwcu_slab_layout.argtypes = [i64, i64, i64, i64, i64, i64, i32, i32, i32, ctypes.POINTER(i64)]
    L.dwcu_slab_layout.restype = ctypes.c_int
    L.dwcu_slab_part_create.argtypes = [i64, i64, i64, i64, i64, i64, P_opts, i32, i32, vp, ctypes.POINTER(SlabSync),
                                        ctypes.POINTER(vp)]
    L.dwcu_slab_part_create.restype = ctypes.c_int
    L.dwcu_slab_part_export.argtypes = [vp, vp, ctypes.POINTER(i64)]
    L.dwcu_slab_part_export.restype = ctypes.c_int
    L.dwcu_slab_part_import.argtypes = [vp, i32, vp, i64]
    L.dwcu_slab_part_import.restype = ctypes.c_int
    L.dwcu_slab_part_run.argtypes = [vp, vp, vp, vp, P_opts]
    L.dwcu_slab_part_run.restype = ctypes.c_int
    L.dwcu_slab_destroy.argtypes = [vp]
    L.dwcu_slab_destroy.restype = None
    L.dwcu_release_cache.argtypes = [i32]
    L.dwcu_release_cache.restype = ctypes.c_int
    L.dwcu_job_create.argtypes = [i64, i64, i64, i64, i64, i64, P_opts, ctypes.POINTER(vp)]
    L.dwcu_job_create.restype = ctypes.c_int
    L.dwcu_job_setup.argtypes = [vp, vp, vp, i32]
    L.dwcu_job_setup.restype = ctypes.c_int
    L.dwcu_job_step.argtypes = [vp, i32, ctypes.POINTER(i32)]
    L.dwcu_job_step.restype = ctypes.c_int
    L.dwcu_job_done.argtypes = [vp]
    L.dwcu_job_done.restype = ctypes.c_int
    L.dwcu_job_result.argtypes = [vp, vp, i32, P_opts]
    L.dwcu_job_result.restype = ctypes.c_int
    L.dwcu_job_destroy.argtypes = [vp]
    L.dwcu_job_destroy.restype = None
    L.dwcu_job_set_stream.argtypes = [vp, vp]
    L.dwcu_job_set_stream.restype = ctypes.c_int
    L.dwcu_job_bytes.argtypes = [vp]
    L.dwcu_job_bytes.restype = i64
    L.dwcu_job_snapshot.argtypes = [vp, vp, vp, vp, i32, ctypes.POINTER(JobState)]
    L.dwcu_job_snapshot.restype = ctypes.c_int
    L.dwcu_job_restore.argtypes = [vp, vp, vp, vp, ctypes.POINTER(JobState)]
    L.dwcu_job_restore.restype = ctypes.c_int
    L.dwcu_last_error.argtypes = []
    L.dwcu_last_error.restype = ctypes.c_char_p
    L.dwcu_abi_version.restype = ctypes.c_int
    L.dwcu_device_count.restype = ctypes.c_int
    L.dwcu_launch_count.restype = i64
    L.dwcu_profile_enable.argtypes = [i32]
    L.dwcu_profile_enable.restype = ctypes.c_int
    L.dwcu_profile_collect.argtypes = [ctypes.POINTER(KernelStat), i32, ctypes.POINTER(i32)]
    L.dwcu_profile_collect.restype = ctypes.c_int
    for fn in (L.dwcu_fft_r2c, L.dwcu_fft_c2r, L.dwcu_fft_r2c_noalloc):
        fn.argtypes = [vp, i64, i64, i64, vp, i32, vp]
        fn.restype = ctypes.c_int
    L.dwcu_server_create.argtypes = [i32, ctypes.c_double, i32, i32, ctypes.POINTER(vp)]
    L.dwcu_server_create.restype = ctypes.c_int
    L.dwcu_server_submit.argtypes = [vp, vp, i64, i64, i64, vp, i64, i64, i64, P_opts, vp, ctypes.POINTER(i64)]
    L.dwcu_server_submit.restype = ctypes.c_int
    L.dwcu_server_wait.argtypes = [vp, i64, ctypes.c_double, P_opts]
    L.dwcu_server_wait.restype = ctypes.c_int
    L.dwcu_server_cancel.argtypes = [vp, i64]
    L.dwcu_server_cancel.restype = ctypes.c_int
    L.dwcu_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
    L.dwcu_server_get_stats.restype = ctypes.c_int
    L.dwcu_server_destroy.argtypes = [vp]
    L.dwcu_server_destroy.restype = None
    L.dwcu_tile_blend.argtypes = [vp, i64, i64, i64, ctypes.POINTER(Tile), i32, i32, vp, ctypes.c_float, i32, vp]
    L.dwcu_tile_blend.restype = ctypes.c_int
    f32p = ctypes.POINTER(ctypes.c_float)
    i32p = ctypes.POINTER(i32)
    L.dwcu_tune_set_mode.argtypes = [i32]
    L.dwcu_tune_get_mode.argtypes = [i32p]
    L.dwcu_tune_select.argtypes = [f32p, i32, ctypes.c_float, i32p]
    L.dwcu_tune_plan_count.argtypes = [i32, i32, i32p]
    L.dwcu_tune_plan_info.argtypes = [i32, i32, i32, i32p, i32p]
    L.dwcu_tune_force.argtypes = [i32, i32, i32]
    L.dwcu_tune_run.argtypes = [i32, i32, i32]
    L.dwcu_tune_query.argtypes = [i32, i32, i32, i32p, f32p, i32, i32p]
    L.dwcu_tune_clear.argtypes = []
    L.dwcu_tune_export.argtypes = [ctypes.c_char_p]
    L.dwcu_tune_import.argtypes = [ctypes.c_char_p]
    for fn in (L.dwcu_tune_set_mode, L.dwcu_tune_get_mode, L.dwcu_tune_select, L.dwcu_tune_plan_count,
               L.dwcu_tune_plan_info, L.dwcu_tune_force, L.dwcu_tune_run, L.dwcu_tune_query, L.dwcu_tune_clear,
               L.dwcu_tune_export, L.dwcu_tune_import):
        fn.restype = ctypes.c_int
    L.dwcu_debug_guards.argtypes = [i32]
    L.dwcu_debug_guards.restype = ctypes.c_int
    L.dwcu_debug_guard_violations.argtypes = []
    L.dwcu_debug_guard_violations.restype = i64
    L.dwcu_selftest_bounded_wait.argtypes = [i32, i32, ctypes.c_uint32]
    L.dwcu_selftest_bounded_wait.restype = ctypes.c_int
    L.dwcu_psf_prepare_device.argtypes = [vp, i64, i64, i64, i64, i64, i64, i32, ctypes.c_float, vp,
                                          ctypes.POINTER(i64), i32, vp]
    L.dwcu_psf_prepare_device.restype = ctypes.c_int
    L.dwcu_batch_run.argtypes = [ctypes.POINTER(vp), i32, vp]
    L.dwcu_batch_run.restype = ctypes.c_int
    L.dwcu_psf_prepare.argtypes = [vp, i64, i64, i64, i64, i64, i64, i32, ctypes.c_float, vp,
                                   ctypes.POINTER(i64)]
    L.dwcu_psf_prepare.restype = ctypes.c_int
    L.dwcu_tiling_create.argtypes = [i64, i64, i64, i64, i64, ctypes.POINTER(Tile), i32, ctypes.POINTER(i32)]
    L.dwcu_tiling_create.restype = ctypes.c_int
    L.dwcu_deconvolve_tiled.argtypes = [vp, i64, i64, i64, vp, i64, i64, i64, i64, i64, ctypes.c_float,
                                        ctypes.c_float, ctypes.c_double, P_opts, vp]
    L.dwcu_deconvolve_tiled.restype = ctypes.c_int
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != 0:
        raise DwcuError(rc, lib().dwcu_last_error().decode(errors="replace"))


def make_opts(*, method: str | int = "shb", n_iter: int = 50, iter_type: int = ITER_FIXED,
              maxiter: int = 250, err_rel: float = 0.02, err_abs: float = 1.0,
              bg: float | None = None, positivity: bool = True, border_quality: int = 2,
              start: int = START_FLAT, metric: int = METRIC_IDIV, alphamax: float = 1.0,
              device: int = 0, verbosity: int = 0, use_graph: bool = True) -> Opts:
    o = Opts()
    lib().dwcu_opts_init(ctypes.byref(o))
    if isinstance(method, str):
        method = {"shb": METHOD_SHB, "rl": METHOD_RL}[method.lower()]
    o.method = method
    o.n_iter = n_iter
    o.iter_type = iter_type
    o.maxiter = maxiter
    o.err_rel = err_rel
    o.err_abs = err_abs
    o.bg_auto = 1 if bg is None else 0
    o.bg = 0.01 if bg is None else bg
    o.positivity = 1 if positivity else 0
    o.border_quality = border_quality
    o.start_condition = start
    o.metric = metric
    o.alphamax = alphamax
    o.device = device
    o.verbosity = verbosity
    o.use_graph = 1 if use_graph else 0
    return o


class Result:
    def __init__(self, out, trace, o: Opts):
        self.out = out
        self.trace = trace
        self.iterations = o.iterations_done
        self.bg = o.bg
        self.work = tuple(o.work)
        self.seconds_setup = o.seconds_setup
        self.seconds_iterate = o.seconds_iterate
        self.seconds_enqueue = o.seconds_enqueue


def run_method(im: np.ndarray, psf: np.ndarray, out: np.ndarray | None = None, **kw) -> Result:
    """The dw_function call on host arrays: ``im`` (P, N, M) and ``psf``
    (pP, pN, pM), float32, x fastest.  Keyword options as :func:`make_opts`.
    ``out``: an optional C-contiguous float32 array of the image's shape for
    the result (for example in page-locked memory)."""
    im = np.ascontiguousarray(im, dtype=np.float32)
    psf = np.ascontiguousarray(psf, dtype=np.float32)
    if im.ndim != 3 or psf.ndim != 3:
        raise ValueError("image and PSF must be 3-D (P, N, M) arrays")
    o = make_opts(**kw)
    cap = max(o.n_iter, o.maxiter, 1)
    trace = np.zeros(cap, dtype=np.float32)
    o.error_trace = trace.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    o.trace_capacity = cap
    out = _out_array(out, im.shape)
    P, N, M = im.shape
    pP, pN, pM = psf.shape
    _check(lib().dwcu_deconvolve(im.ctypes.data, M, N, P, psf.ctypes.data, pM, pN, pP,
                                 ctypes.byref(o), out.ctypes.data))
    return Result(out, trace[: o.iterations_done].copy(), o)


def run_slabs(im: np.ndarray, psf: np.ndarray, parts: int = 2, devices=None, out: np.ndarray | None = None,
              **kw) -> Result:
    """:func:`run_method` with the job split over ``parts`` slabs of z planes
    (dwcu_deconvolve_slabs): one image over several GPUs.  ``devices``: the
    GPU of each part (default: every part on the ``device`` option)."""
    im = np.ascontiguousarray(im, dtype=np.float32)
    psf = np.ascontiguousarray(psf, dtype=np.float32)
    if im.ndim != 3 or psf.ndim != 3:
        raise ValueError("image and PSF must be 3-D (P, N, M) arrays")
    o = make_opts(**kw)
    cap = max(o.n_iter, o.maxiter, 1)
    trace = np.zeros(cap, dtype=np.float32)
    o.error_trace = trace.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    o.trace_capacity = cap
    out = _out_array(out, im.shape)
    dev = None
    if devices is not None:
        if len(devices) != parts:
            raise ValueError("one device per part")
        dev = (ctypes.c_int32 * parts)(*devices)
    P, N, M = im.shape
    pP, pN, pM = psf.shape
    _check(lib().dwcu_deconvolve_slabs(im.ctypes.data, M, N, P, psf.ctypes.data, pM, pN, pP, ctypes.byref(o),
                                       parts, dev, out.ctypes.data))
    return Result(out, trace[: o.iterations_done].copy(), o)


class SlabPart:
    """This process's part of an image split over processes (dwcu_slab_part_*).
    ``barrier(stream)`` and ``allreduce(stream, n, op)`` are the caller's
    collectives (see dwcu.h); ``sync_buf`` a device buffer of at least 4
    doubles that ``allreduce`` reduces in place."""

    def __init__(self, shape, psf_shape, parts: int, part: int, sync_buf: int, barrier, allreduce, **kw):
        self.shape = tuple(shape)
        self.opts = make_opts(**kw)

        def _barrier(ctx, stream):
            try:
                barrier(stream or 0)
                return 0
            except Exception:
                return 1

        def _allreduce(ctx, stream, n, op):
            try:
                allreduce(stream or 0, int(n), int(op))
                return 0
            except Exception:
                return 1

        self._cb = (SLAB_BARRIER(_barrier), SLAB_ALLREDUCE(_allreduce))  # kept alive while the part lives
        self._sync = SlabSync(self._cb[0], self._cb[1], None)
        P, N, M = self.shape
        pP, pN, pM = psf_shape
        h = ctypes.c_void_p()
        _check(lib().dwcu_slab_part_create(M, N, P, pM, pN, pP, ctypes.byref(self.opts), parts, part,
                                           ctypes.c_void_p(sync_buf), ctypes.byref(self._sync), ctypes.byref(h)))
        self.h = h

    def export(self):
        """(IPC handle bytes, spectrum offset) for the other processes."""
        buf = ctypes.create_string_buffer(64)
        off = ctypes.c_int64()
        _check(lib().dwcu_slab_part_export(self.h, buf, ctypes.byref(off)))
        return buf.raw, off.value

    def import_part(self, part: int, handle: bytes, offset: int) -> None:
        buf = ctypes.create_string_buffer(bytes(handle), 64)
        _check(lib().dwcu_slab_part_import(self.h, part, buf, offset))

    def run(self, im: np.ndarray, psf: np.ndarray, out: np.ndarray) -> Result:
        """Set-up, iterations and this part's image planes into ``out``."""
        im = np.ascontiguousarray(im, dtype=np.float32)
        psf = np.ascontiguousarray(psf, dtype=np.float32)
        o = self.opts
        cap = max(o.n_iter, o.maxiter, 1)
        trace = np.zeros(cap, dtype=np.float32)
        o.error_trace = trace.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        o.trace_capacity = cap
        _check(lib().dwcu_slab_part_run(self.h, im.ctypes.data, psf.ctypes.data, out.ctypes.data, ctypes.byref(o)))
        return Result(out, trace[: o.iterations_done].copy(), o)

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().dwcu_slab_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def slab_layout(shape, psf_shape, parts: int, part: int, border_quality: int = 2) -> dict:
    """The planes and z-pass columns of one part of a split job (dwcu_slab_layout)."""
    P, N, M = shape
    pP, pN, pM = psf_shape
    info = (ctypes.c_int64 * 6)()
    _check(lib().dwcu_slab_layout(M, N, P, pM, pN, pP, border_quality, parts, part, info))
    keys = ("planes", "image_planes", "col0", "cols", "plane_cols", "Z")
    return dict(zip(keys, list(info)))


def release_cache(device: int = -1) -> None:
    """Free the device blocks kept for reuse by later jobs
    (dwcu_release_cache); ``device`` < 0: every device."""
    _check(lib().dwcu_release_cache(device))


def _out_array(out, shape):
    if out is None:
        return np.empty(shape, dtype=np.float32)
    if out.shape != tuple(shape) or out.dtype != np.float32 or not out.flags["C_CONTIGUOUS"]:
        raise ValueError(f"out must be a C-contiguous float32 array of shape {tuple(shape)}")
    return out


def run_method_device(d_im, d_psf, d_out, shape, psf_shape, stream: int = 0, **kw) -> Result:
    """The dw_function call on device buffers (raw device pointers, e.g.
    ``tensor.data_ptr()``); ``stream`` is a cudaStream_t handle or 0."""
    o = make_opts(**kw)
    cap = max(o.n_iter, o.maxiter, 1)
    trace = np.zeros(cap, dtype=np.float32)
    o.error_trace = trace.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    o.trace_capacity = cap
    P, N, M = shape
    pP, pN, pM = psf_shape
    _check(lib().dwcu_deconvolve_device(ctypes.c_void_p(d_im), M, N, P, ctypes.c_void_p(d_psf), pM, pN, pP,
                                        ctypes.byref(o), ctypes.c_void_p(d_out), ctypes.c_void_p(stream or None)))
    return Result(None, trace[: o.iterations_done].copy(), o)


def fft_r2c_device(d_in: int, shape, d_out: int, device: int = 0, stream: int = 0) -> None:
    """3-D R2C (fft() of src/fft.c:401-415) on device buffers; shape (P, N, M)."""
    P, N, M = shape
    _check(lib().dwcu_fft_r2c(ctypes.c_void_p(d_in), M, N, P, ctypes.c_void_p(d_out), device,
                              ctypes.c_void_p(stream or None)))


def fft_r2c_noalloc_device(d_in: int, shape, d_out: int, device: int = 0, stream: int = 0) -> None:
    """:func:`fft_r2c_device` with the library's fixed work space (no device
    allocation; sizes up to the work space only)."""
    P, N, M = shape
    _check(lib().dwcu_fft_r2c_noalloc(ctypes.c_void_p(d_in), M, N, P, ctypes.c_void_p(d_out), device,
                                      ctypes.c_void_p(stream or None)))


def fft_c2r_device(d_in: int, shape, d_out: int, device: int = 0, stream: int = 0) -> None:
    """Unnormalised 3-D C2R on device buffers; shape (P, N, M) of the real output."""
    P, N, M = shape
    _check(lib().dwcu_fft_c2r(ctypes.c_void_p(d_in), M, N, P, ctypes.c_void_p(d_out), device,
                              ctypes.c_void_p(stream or None)))


def plan_size(shape, psf_shape, border_quality: int = 2, method: str = "shb"):
    """Padded job size (X, Y, Z) and device bytes for a job."""
    P, N, M = shape
    pP, pN, pM = psf_shape
    work = (ctypes.c_int64 * 3)()
    nbytes = ctypes.c_int64()
    _check(lib().dwcu_plan_size(M, N, P, pM, pN, pP, border_quality,
                                METHOD_SHB if method == "shb" else METHOD_RL, work, ctypes.byref(nbytes)))
    return tuple(work), nbytes.value


def psf_prepare(psf: np.ndarray, shape, border_quality: int = 2, xycropfactor: float = 0.001) -> np.ndarray:
    """dw_run's PSF preparation for an image of ``shape`` (P, N, M): normalise,
    psf_autocrop (dw.c:1973-1997), normalise (dwcu_psf_prepare)."""
    p = np.ascontiguousarray(psf, dtype=np.float32)
    P, N, M = shape
    pP, pN, pM = p.shape
    out = np.empty(p.size, dtype=np.float32)
    dims = (ctypes.c_int64 * 3)()
    _check(lib().dwcu_psf_prepare(p.ctypes.data, pM, pN, pP, M, N, P, border_quality, xycropfactor,
                                  out.ctypes.data, dims))
    return out[: dims[0] * dims[1] * dims[2]].reshape(dims[2], dims[1], dims[0]).copy()


def psf_prepare_device(d_psf: int, psf_shape, shape, d_out: int, border_quality: int = 2,
                       xycropfactor: float = 0.001, device: int = 0, stream: int = 0):
    """:func:`psf_prepare` on device buffers (d_psf, d_out: device pointers,
    d_out with room for the whole PSF); returns the prepared (P, N, M) size."""
    P, N, M = shape
    pP, pN, pM = psf_shape
    dims = (ctypes.c_int64 * 3)()
    _check(lib().dwcu_psf_prepare_device(ctypes.c_void_p(d_psf), pM, pN, pP, M, N, P, border_quality, xycropfactor,
                                         ctypes.c_void_p(d_out), dims, device, ctypes.c_void_p(stream or None)))
    return (int(dims[2]), int(dims[1]), int(dims[0]))


def tiling_create(shape, max_size: int, overlap: int = 20) -> list[dict]:
    """tiling_create (tiling.c:70-130) for an image of ``shape`` (P, N, M);
    each tile as a dict of x, y, z ordered ``size``, ``pos``, ``xpos``, ``xsize``."""
    P, N, M = shape
    n = ctypes.c_int32()
    _check(lib().dwcu_tiling_create(M, N, P, max_size, overlap, None, 0, ctypes.byref(n)))
    arr = (Tile * n.value)()
    _check(lib().dwcu_tiling_create(M, N, P, max_size, overlap, arr, n.value, ctypes.byref(n)))
    return [{k: tuple(getattr(t, k)) for k in ("size", "pos", "xpos", "xsize")} for t in arr]


def deconvolve_tiled(im: np.ndarray, psf: np.ndarray, tile_size: int, overlap: int = 20,
                     offset: float = 5.0, xycropfactor: float = 0.001, hbm_budget: float = 0.0,
                     out: np.ndarray | None = None, **kw) -> Result:
    """deconvolve_tiles (dw.c:2001-2229) on host arrays; ``psf`` as dw_run
    hands it over (already prepared for the whole image).  ``out`` as for
    :func:`run_method`."""
    im = np.ascontiguousarray(im, dtype=np.float32)
    psf = np.ascontiguousarray(psf, dtype=np.float32)
    o = make_opts(**kw)
    out = _out_array(out, im.shape)
    P, N, M = im.shape
    pP, pN, pM = psf.shape
    _check(lib().dwcu_deconvolve_tiled(im.ctypes.data, M, N, P, psf.ctypes.data, pM, pN, pP, tile_size,
                                       overlap, offset, xycropfactor, hbm_budget, ctypes.byref(o),
                                       out.ctypes.data))
    return Result(out, np.zeros(0, np.float32), o)


def tiles_array(tiles: list[dict]):
    """The ctypes array of dwcu_tile for tiles as tiling_create returns them."""
    arr = (Tile * len(tiles))()
    for a, t in zip(arr, tiles):
        for k in ("size", "pos", "xpos", "xsize"):
            getattr(a, k)[:] = list(t[k])
    return arr


def tile_blend_device(d_out: int, shape, tiles, tid: int, d_tile: int, offset: float = 5.0, device: int = 0,
                      stream: int = 0) -> None:
    """dwcu_tile_blend on device buffers; ``tiles`` from :func:`tiling_create`
    (or a :func:`tiles_array`)."""
    P, N, M = shape
    arr = tiles if not isinstance(tiles, list) else tiles_array(tiles)
    _check(lib().dwcu_tile_blend(ctypes.c_void_p(d_out), M, N, P, arr, len(arr), tid, ctypes.c_void_p(d_tile),
                                 offset, device, ctypes.c_void_p(stream or None)))


def batch_run(jobs: list["Job"], stream: int = 0) -> None:
    """Run set-up jobs to completion together (dwcu_batch_run)."""
    arr = (ctypes.c_void_p * len(jobs))(*[j.h.value for j in jobs])
    _check(lib().dwcu_batch_run(arr, len(jobs), ctypes.c_void_p(stream or None)))


class Server:
    """dwcu_server: continuous batching of deconvolution requests on one GPU.

    ``submit`` queues a dw_function call (host arrays) and returns its id;
    ``wait`` returns its :class:`Result`.  The arrays are kept referenced
    until the request is waited for."""

    def __init__(self, device: int = 0, hbm_budget: float = 0.0, max_active: int = 8, iters_per_turn: int = 5):
        h = ctypes.c_void_p()
        _check(lib().dwcu_server_create(device, hbm_budget, max_active, iters_per_turn, ctypes.byref(h)))
        self.h = h
        self.device = device
        self._req = {}

    def submit(self, im: np.ndarray, psf: np.ndarray, **kw) -> int:
        im = np.ascontiguousarray(im, dtype=np.float32)
        psf = np.ascontiguousarray(psf, dtype=np.float32)
        kw.setdefault("device", self.device)
        o = make_opts(**kw)
        cap = max(o.n_iter, o.maxiter, 1)
        trace = np.zeros(cap, dtype=np.float32)
        o.error_trace = trace.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        o.trace_capacity = cap
        out = np.empty_like(im)
        P, N, M = im.shape
        pP, pN, pM = psf.shape
        rid = ctypes.c_int64()
        _check(lib().dwcu_server_submit(self.h, im.ctypes.data, M, N, P, psf.ctypes.data, pM, pN, pP,
                                        ctypes.byref(o), out.ctypes.data, ctypes.byref(rid)))
        self._req[rid.value] = (im, psf, out, trace, o)
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0) -> Result:
        im, psf, out, trace, o = self._req[rid]
        so = Opts()
        so.error_trace = trace.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        so.trace_capacity = len(trace)
        _check(lib().dwcu_server_wait(self.h, rid, timeout, ctypes.byref(so)))
        del self._req[rid]
        return Result(out, trace[: so.iterations_done].copy(), so)

    def cancel(self, rid: int) -> None:
        _check(lib().dwcu_server_cancel(self.h, rid))

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().dwcu_server_get_stats(self.h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self) -> None:
        if self.h:
            lib().dwcu_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dw_run(image: np.ndarray, psf: np.ndarray, *, tilesize: int = 0, tilepad: int = 20,
           offset: float = 5.0, xycropfactor: float = 0.001, **kw) -> np.ndarray:
    """The method part of dw_run (dw.c:2797-2850) on in-memory arrays: PSF
    normalised and cropped against the image, then the method on the whole
    image (+offset; the returned buffer keeps the offset, as dw_run's result
    buffer does, dw.c:2835-2848 and 2907-2913) or, with ``tilesize`` > 0,
    deconvolve_tiles (offset removed per tile).  Options as :func:`make_opts`."""
    im = np.array(image, dtype=np.float32, copy=True)
    bq = kw.get("border_quality", 2)
    p = psf_prepare(psf, im.shape, bq, xycropfactor)
    if tilesize > 0:
        return deconvolve_tiled(im, p, tilesize, tilepad, offset, xycropfactor, **kw).out
    if offset > 0:
        im += np.float32(offset)
    return run_method(im, p, **kw).out


class Job:
    """A resident deconvolution job (dwcu_job_*): setup once, step, read."""

    def __init__(self, shape, psf_shape, **kw):
        self.shape = tuple(shape)
        self.psf_shape = tuple(psf_shape)
        self.opts = make_opts(**kw)
        P, N, M = self.shape
        pP, pN, pM = self.psf_shape
        h = ctypes.c_void_p()
        _check(lib().dwcu_job_create(M, N, P, pM, pN, pP, ctypes.byref(self.opts), ctypes.byref(h)))
        self.h = h

    def setup(self, im, psf, on_device: bool = False):
        if on_device:
            _check(lib().dwcu_job_setup(self.h, ctypes.c_void_p(im), ctypes.c_void_p(psf), 1))
        else:
            self._im = np.ascontiguousarray(im, dtype=np.float32)
            self._psf = np.ascontiguousarray(psf, dtype=np.float32)
            _check(lib().dwcu_job_setup(self.h, self._im.ctypes.data, self._psf.ctypes.data, 0))

    def step(self, n: int) -> int:
        rem = ctypes.c_int32()
        _check(lib().dwcu_job_step(self.h, n, ctypes.byref(rem)))
        return rem.value

    def done(self) -> bool:
        return bool(lib().dwcu_job_done(self.h))

    def set_stream(self, stream: int) -> None:
        _check(lib().dwcu_job_set_stream(self.h, ctypes.c_void_p(stream or None)))

    def nbytes(self) -> int:
        return int(lib().dwcu_job_bytes(self.h))

    def snapshot(self) -> dict:
        """The job's state between iterations (dwcu_job_snapshot): x_k, x_{k-1}
        (SHB), the error trace and the stopping rule's counters."""
        st = JobState()
        _check(lib().dwcu_job_snapshot(self.h, None, None, None, 0, ctypes.byref(st)))
        x = np.empty(st.volume_elems, dtype=np.float32)
        xp = np.empty(st.volume_elems, dtype=np.float32) if self.opts.method == METHOD_SHB else None
        cap = max(self.opts.n_iter, self.opts.maxiter, 1)
        trace = np.zeros(cap, dtype=np.float32)
        _check(lib().dwcu_job_snapshot(self.h, x.ctypes.data, None if xp is None else xp.ctypes.data,
                                       trace.ctypes.data, cap, ctypes.byref(st)))
        return dict(x=x, x_prev=xp, trace=trace[: st.done_iters].copy(), next_iter=st.next_iter,
                    done_iters=st.done_iters, iter=st.iter, error=st.error, lasterror=st.lasterror, bg=st.bg)

    def restore(self, snap: dict) -> None:
        """Continue from :meth:`snapshot` of a job with the same image, PSF and
        options (this job set up already): dwcu_job_restore."""
        st = JobState()
        st.volume_elems = snap["x"].size
        for k in ("next_iter", "done_iters", "iter", "error", "lasterror", "bg"):
            setattr(st, k, snap[k])
        x = np.ascontiguousarray(snap["x"], dtype=np.float32)
        xp = None if snap["x_prev"] is None else np.ascontiguousarray(snap["x_prev"], dtype=np.float32)
        tr = np.ascontiguousarray(snap["trace"], dtype=np.float32)
        _check(lib().dwcu_job_restore(self.h, x.ctypes.data, None if xp is None else xp.ctypes.data,
                                      tr.ctypes.data if tr.size else None, ctypes.byref(st)))

    def result(self, out=None, on_device: bool = False) -> Result:
        o = Opts()
        lib().dwcu_opts_init(ctypes.byref(o))
        cap = max(self.opts.n_iter, self.opts.maxiter, 1)
        trace = np.zeros(cap, dtype=np.float32)
        o.error_trace = trace.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        o.trace_capacity = cap
        if on_device:
            _check(lib().dwcu_job_result(self.h, ctypes.c_void_p(out), 1, ctypes.byref(o)))
            return Result(None, trace[: o.iterations_done].copy(), o)
        arr = np.empty(self.shape, dtype=np.float32) if out is None else out
        _check(lib().dwcu_job_result(self.h, arr.ctypes.data, 0, ctypes.byref(o)))
        return Result(arr, trace[: o.iterations_done].copy(), o)

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().dwcu_job_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def deconvolve(image: np.ndarray, psf: np.ndarray, iterations: int, bq: int = 2, verbose: int = 0,
               threads: int | None = None, gpu: bool = True, *, method: str = "shb",
               offset: float = 5.0, device: int = 0) -> np.ndarray:
    """pydeconwolf.deconvolve(image, psf, iterations, bq, verbose, threads,
    gpu) (pydeconwolf.c:284-394), which runs dw_run: fixed iteration count,
    PSF prepared as in :func:`dw_run`, offset added before the method and
    kept in the result (dw.c:2835-2848).
    ``threads`` is accepted for signature compatibility (the work runs on
    the GPU); ``gpu=False`` is rejected: this package has no CPU path."""
    if not gpu:
        raise ValueError("deconwolf_b200 runs on the GPU only (gpu=False is not available)")
    im = np.array(image, dtype=np.float32, copy=True)
    if np.min(im) < 0:
        raise ValueError("The image contains negative values, can not continue!")  # dw.c:2703-2710
    if np.max(im) < 1.0:
        raise ValueError("The image has too low intensity, can not continue!")  # dw.c:2711-2721
    return dw_run(im, psf, offset=offset, method=method, n_iter=iterations, iter_type=ITER_FIXED,
                  border_quality=bq, verbosity=verbose, device=device)


# ---------------------------------------------------------------- autotuning

def tune_select(times_ms, margin: float = 0.02) -> int:
    """The autotuner's selection rule on candidate times (host logic)."""
    arr = (ctypes.c_float * len(times_ms))(*times_ms)
    out = ctypes.c_int32()
    _check(lib().dwcu_tune_select(arr, len(times_ms), margin, ctypes.byref(out)))
    return out.value


def tune_plans(kind: int, n: int):
    """[(radices, tile), ...] of the candidate plans of a length (candidate 0 first)."""
    cnt = ctypes.c_int32()
    _check(lib().dwcu_tune_plan_count(kind, n, ctypes.byref(cnt)))
    out = []
    for c in range(cnt.value):
        rad = (ctypes.c_int32 * 3)()
        tile = ctypes.c_int32()
        _check(lib().dwcu_tune_plan_info(kind, n, c, rad, ctypes.byref(tile)))
        out.append((tuple(int(r) for r in rad if r > 1) or (1,), int(tile.value)))
    return out


def tune_force(kind: int, n: int, cand: int) -> None:
    """Use candidate ``cand`` for this length from now on (-1: measure again)."""
    _check(lib().dwcu_tune_force(kind, n, cand))


def tune_run(kind: int, n: int, device: int = 0) -> None:
    """Time the candidates of one length now (if not recorded yet)."""
    _check(lib().dwcu_tune_run(device, kind, n))


def tune_query(kind: int, n: int, device: int = 0):
    """(chosen candidate or -1, [ms per candidate])."""
    cand = ctypes.c_int32()
    ms = (ctypes.c_float * 16)()
    k = ctypes.c_int32()
    _check(lib().dwcu_tune_query(device, kind, n, ctypes.byref(cand), ms, 16, ctypes.byref(k)))
    return cand.value, [float(ms[i]) for i in range(k.value)]


def tune_set_mode(mode: int) -> None:
    _check(lib().dwcu_tune_set_mode(mode))


def tune_clear() -> None:
    _check(lib().dwcu_tune_clear())


def tune_export(path: str) -> None:
    _check(lib().dwcu_tune_export(os.fsencode(path)))


def tune_import(path: str) -> None:
    _check(lib().dwcu_tune_import(os.fsencode(path)))
