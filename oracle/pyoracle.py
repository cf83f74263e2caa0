"""Python access to the oracle (TEST INFRASTRUCTURE ONLY).

Two checkers, both CPU:

* ``port``      -- oracle/liboracle.so, the C restatement of deconwolf's
                   SHB / RL path (oracle/dwo.c);
* ``reference`` -- oracle/_ref/libdwref.so, deconwolf's own method_shb.c,
                   method_rl.c, fft.c and fim.c compiled unmodified against
                   the FFTW-API shim (oracle/Makefile, oracle/ref_glue.c).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only to check or time the CPU path.  The product
(deconwolf_b200/) never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdwref.so")

METHOD_RL = 0
METHOD_SHB = 2
ITER_ABS, ITER_REL, ITER_FIXED = 0, 1, 2
START_FLAT, START_LP, START_IDENTITY = 0, 1, 2
METRIC_MSE, METRIC_IDIV = 0, 1


class DwoOpts(ctypes.Structure):
    """Mirror of ``dwo_opts`` in oracle/dwo.h."""

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
        ("threads", ctypes.c_int32),
        ("work", ctypes.c_int64 * 3),
        ("iterations_done", ctypes.c_int32),
        ("error_trace", ctypes.POINTER(ctypes.c_float)),
        ("trace_capacity", ctypes.c_int32),
        ("loop_seconds", ctypes.c_double),
        ("setup_seconds", ctypes.c_double),
    ]


def build() -> None:
    """Compile the checkers (liboracle.so always; _ref when the reference
    sources are present on this machine)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_libs: dict[str, ctypes.CDLL] = {}


def _lib(kind: str) -> ctypes.CDLL:
    if kind in _libs:
        return _libs[kind]
    path = PORT_SO if kind == "port" else REF_SO
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library {path} is not built (make -C oracle)")
    lib = ctypes.CDLL(path)
    fn = lib.dwo_deconvolve if kind == "port" else lib.dwref_deconvolve
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                   ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                   ctypes.POINTER(DwoOpts), ctypes.c_void_p]
    if kind == "port":
        lib.dwo_idiv.restype = ctypes.c_float
        lib.dwo_idiv.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int64] * 6
        lib.dwo_fft_r2c.argtypes = [ctypes.c_void_p] + [ctypes.c_int64] * 3 + [ctypes.c_void_p, ctypes.c_int]
        lib.dwo_fft_c2r.argtypes = [ctypes.c_void_p] + [ctypes.c_int64] * 3 + [ctypes.c_void_p, ctypes.c_int]
        lib.dwo_argmax.argtypes = [ctypes.c_void_p] + [ctypes.c_int64] * 3 + [ctypes.POINTER(ctypes.c_int64)] * 3
        lib.dwo_circshift.argtypes = [ctypes.c_void_p] + [ctypes.c_int64] * 6
    _libs[kind] = lib
    return lib


def available(kind: str) -> bool:
    return os.path.exists(PORT_SO if kind == "port" else REF_SO)


class Result:
    def __init__(self, out, trace, opts: DwoOpts):
        self.out = out
        self.trace = trace
        self.iterations = opts.iterations_done
        self.bg = opts.bg
        self.loop_seconds = opts.loop_seconds
        self.setup_seconds = opts.setup_seconds


def deconvolve(im: np.ndarray, psf: np.ndarray, *, method: str = "shb", n_iter: int = 50,
               iter_type: int = ITER_FIXED, maxiter: int = 250, err_rel: float = 0.02,
               err_abs: float = 1.0, bg: float | None = None, positivity: bool = True,
               border_quality: int = 2, start: int = START_FLAT, metric: int = METRIC_IDIV,
               alphamax: float = 1.0, threads: int = 0, work=None,
               impl: str = "port") -> Result:
    """Run the CPU checker on ``im`` (P, N, M) float32 with ``psf`` (pP, pN, pM).

    ``bg=None`` means automatic background (bg_auto).  ``work`` optionally
    gives a padded job size (Wx, Wy, Wz) for the port (bq=2 only)."""
    im = np.ascontiguousarray(im, dtype=np.float32)
    psf = np.ascontiguousarray(psf, dtype=np.float32)
    P, N, M = im.shape
    pP, pN, pM = psf.shape
    o = DwoOpts()
    o.method = METHOD_SHB if method == "shb" else METHOD_RL
    o.n_iter = n_iter
    o.iter_type = iter_type
    o.maxiter = maxiter
    o.err_rel = err_rel
    o.err_abs = err_abs
    o.bg = 0.01 if bg is None else bg
    o.bg_auto = 1 if bg is None else 0
    o.positivity = 1 if positivity else 0
    o.border_quality = border_quality
    o.start_condition = start
    o.metric = metric
    o.alphamax = alphamax
    o.threads = threads if threads > 0 else (os.cpu_count() or 1)
    if work is not None:
        o.work[0], o.work[1], o.work[2] = (int(w) for w in work)
    cap = max(maxiter, n_iter, 1)
    trace = np.zeros(cap, dtype=np.float32)
    o.error_trace = trace.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    o.trace_capacity = cap
    out = np.empty_like(im)
    lib = _lib(impl)
    fn = lib.dwo_deconvolve if impl == "port" else lib.dwref_deconvolve
    rc = fn(im.ctypes.data, M, N, P, psf.ctypes.data, pM, pN, pP, ctypes.byref(o), out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle ({impl}) rejected the input: code {rc}")
    return Result(out, trace[: o.iterations_done].copy(), o)


def idiv(y: np.ndarray, g: np.ndarray) -> float:
    """get_fIdiv (dw.c:1492-1524) on same-shaped (P, N, M) arrays."""
    y = np.ascontiguousarray(y, dtype=np.float32)
    g = np.ascontiguousarray(g, dtype=np.float32)
    P, N, M = g.shape
    return float(_lib("port").dwo_idiv(y.ctypes.data, g.ctypes.data, M, N, P, M, N, P))


def rfftn(x: np.ndarray, threads: int = 0) -> np.ndarray:
    """FFTW-layout 3-D r2c of a (P, N, M) float32 array -> (P, N, M//2+1) complex64."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    P, N, M = x.shape
    out = np.empty((P, N, M // 2 + 1), dtype=np.complex64)
    _lib("port").dwo_fft_r2c(x.ctypes.data, M, N, P, out.ctypes.data, threads)
    return out


def irfftn(X: np.ndarray, M: int, threads: int = 0) -> np.ndarray:
    """Unnormalised 3-D c2r (input copied, FFTW destroys it)."""
    X = np.array(X, dtype=np.complex64, copy=True, order="C")
    P, N, _ = X.shape
    out = np.empty((P, N, M), dtype=np.float32)
    _lib("port").dwo_fft_c2r(X.ctypes.data, M, N, P, out.ctypes.data, threads)
    return out
