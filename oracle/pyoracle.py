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
    i64, vp, f32 = ctypes.c_int64, ctypes.c_void_p, ctypes.c_float
    tiling = lib.dwo_tiling_create if kind == "port" else lib.dwref_tiling_create
    tiling.restype = ctypes.c_int
    tiling.argtypes = [i64] * 5 + [vp, ctypes.c_int]
    tiled = lib.dwo_deconvolve_tiled if kind == "port" else lib.dwref_deconvolve_tiled
    tiled.restype = ctypes.c_int
    tiled.argtypes = [vp, i64, i64, i64, vp, i64, i64, i64, i64, i64, f32, f32, ctypes.POINTER(DwoOpts), vp]
    if kind == "reference":
        lib.dwref_iteration_seconds.restype = ctypes.c_int
        lib.dwref_iteration_seconds.argtypes = [vp, ctypes.c_int]
        lib.dwref_tiling_weights.argtypes = [i64] * 5 + [ctypes.c_int, vp, vp]
    if kind == "port":
        lib.dwo_psf_prepare.restype = ctypes.c_int
        lib.dwo_psf_prepare.argtypes = [vp] + [i64] * 6 + [ctypes.c_int, f32, vp, ctypes.POINTER(i64)]
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


PSF_SO = os.path.join(HERE, "_ref", "libdwpsf.so")


def psf_prepare_reference(psf: np.ndarray, shape, border_quality: int = 2, xycropfactor: float = 0.001):
    """deconwolf's own PSF preparation (dw_run, src/dw.c:2799-2826: normalise,
    psf_autocrop, normalise), from _ref/libdwpsf.so (dw.c compiled
    unmodified); None when that build is absent."""
    if not os.path.exists(PSF_SO):
        return None
    lib = _libs.get("psf")
    if lib is None:
        lib = ctypes.CDLL(PSF_SO)
        lib.dwpsf_prepare.restype = ctypes.c_int
        lib.dwpsf_prepare.argtypes = [ctypes.c_void_p] + [ctypes.c_int64] * 6 + [ctypes.c_int, ctypes.c_float,
                                                                                  ctypes.c_void_p, ctypes.c_void_p]
        _libs["psf"] = lib
    p = np.ascontiguousarray(psf, dtype=np.float32)
    P, N, M = shape
    pP, pN, pM = p.shape
    out = np.empty(p.size, dtype=np.float32)
    dims = (ctypes.c_int64 * 3)()
    rc = lib.dwpsf_prepare(p.ctypes.data, pM, pN, pP, M, N, P, border_quality, xycropfactor, out.ctypes.data, dims)
    if rc != 0:
        raise RuntimeError("dwpsf_prepare failed")
    return out[: dims[0] * dims[1] * dims[2]].reshape(dims[2], dims[1], dims[0]).copy()


class Result:
    def __init__(self, out, trace, opts: DwoOpts):
        self.out = out
        self.trace = trace
        self.iterations = opts.iterations_done
        self.bg = opts.bg
        self.loop_seconds = opts.loop_seconds
        self.setup_seconds = opts.setup_seconds


def make_opts(*, method: str = "shb", n_iter: int = 50, iter_type: int = ITER_FIXED, maxiter: int = 250,
              err_rel: float = 0.02, err_abs: float = 1.0, bg: float | None = None, positivity: bool = True,
              border_quality: int = 2, start: int = START_FLAT, metric: int = METRIC_IDIV,
              alphamax: float = 1.0, threads: int = 0, work=None) -> DwoOpts:
    """dwo_opts from keyword options; ``bg=None`` means automatic background
    (bg_auto); ``work`` optionally gives a padded job size (Wx, Wy, Wz) for the
    port (bq=2 only)."""
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
    return o


def deconvolve(im: np.ndarray, psf: np.ndarray, *, impl: str = "port", **kw) -> Result:
    """Run the CPU checker on ``im`` (P, N, M) float32 with ``psf`` (pP, pN, pM);
    options as :func:`make_opts`."""
    im = np.ascontiguousarray(im, dtype=np.float32)
    psf = np.ascontiguousarray(psf, dtype=np.float32)
    P, N, M = im.shape
    pP, pN, pM = psf.shape
    o = make_opts(**kw)
    cap = max(o.maxiter, o.n_iter, 1)
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


def psf_prepare(psf: np.ndarray, shape, border_quality: int = 2, xycropfactor: float = 0.001) -> np.ndarray:
    """dw_run's normalise / psf_autocrop / normalise (oracle/dwo.c)."""
    p = np.ascontiguousarray(psf, dtype=np.float32)
    P, N, M = shape
    pP, pN, pM = p.shape
    out = np.empty(p.size, dtype=np.float32)
    dims = (ctypes.c_int64 * 3)()
    _lib("port").dwo_psf_prepare(p.ctypes.data, pM, pN, pP, M, N, P, border_quality,
                                 ctypes.c_float(xycropfactor), out.ctypes.data, dims)
    return out[: dims[0] * dims[1] * dims[2]].reshape(dims[2], dims[1], dims[0]).copy()


def tiling_create(shape, max_size: int, overlap: int = 20, impl: str = "port") -> np.ndarray:
    """Tiles as an (n, 18) int64 array: size[3], pos[6], xpos[6], xsize[3]
    (x, y, z order); ``impl="reference"`` runs the reference's tiling.c."""
    P, N, M = shape
    lib = _lib(impl)
    fn = lib.dwo_tiling_create if impl == "port" else lib.dwref_tiling_create
    n = fn(M, N, P, max_size, overlap, None, 0)
    t = np.zeros((n, 18), dtype=np.int64)
    fn(M, N, P, max_size, overlap, t.ctypes.data, n)
    return t


def tiling_weights(shape, max_size: int, overlap: int, tid: int):
    """The reference's tile_getWeight for tile ``tid`` and tiling_getWeights,
    over the (N, M) plane (tiling.c:169-223)."""
    P, N, M = shape
    wt = np.zeros((N, M), np.float32)
    ws = np.zeros((N, M), np.float32)
    _lib("reference").dwref_tiling_weights(M, N, P, max_size, overlap, tid, wt.ctypes.data, ws.ctypes.data)
    return wt, ws


def deconvolve_tiled(im: np.ndarray, psf: np.ndarray, tile_size: int, overlap: int = 20, offset: float = 5.0,
                     xycropfactor: float = 0.001, impl: str = "port", **kw) -> Result:
    """deconvolve_tiles (dw.c:2001-2229) in memory; ``psf`` as dw_run hands it
    over; options as :func:`make_opts`."""
    im = np.ascontiguousarray(im, dtype=np.float32)
    psf = np.ascontiguousarray(psf, dtype=np.float32)
    P, N, M = im.shape
    pP, pN, pM = psf.shape
    o = make_opts(**kw)
    out = np.empty_like(im)
    lib = _lib(impl)
    fn = lib.dwo_deconvolve_tiled if impl == "port" else lib.dwref_deconvolve_tiled
    rc = fn(im.ctypes.data, M, N, P, psf.ctypes.data, pM, pN, pP, tile_size, overlap, ctypes.c_float(offset),
            ctypes.c_float(xycropfactor), ctypes.byref(o), out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle ({impl}) rejected the tiled input: code {rc}")
    return Result(out, np.zeros(0, np.float32), o)


def iteration_seconds() -> np.ndarray:
    """Per-iteration wall seconds of the last reference run (its iterator's
    timestamps)."""
    buf = np.zeros(4096, np.float64)
    n = _lib("reference").dwref_iteration_seconds(buf.ctypes.data, len(buf))
    return buf[:n].copy()


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
