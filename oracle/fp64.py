"""FP64 restatement of deconwolf's SHB / RL deconvolution (test infrastructure).

TEST INFRASTRUCTURE ONLY: the error reference of the parity tests.  It runs
the same iteration as deconwolf's CPU methods with every value and every
transform in float64 (NumPy + scipy.fft), so a float32 result's distance to
it is that result's own arithmetic error.  Nothing in the product imports it.

Follows, step by step:
  deconvolve_shb        src/method_shb.c:77-424   (loop :298-382, result :385-413)
  iter_shb              src/method_shb.c:10-74
  deconvolve_rl         src/method_rl.c:105-400   (result :393)
  iter_rl               src/method_rl.c:28-102
  job size by bq        src/method_shb.c:137-153
  OTF                   src/method_shb.c:185-212 (fim_insert fim.c:585-623,
                        fim_argmax fim.c:269-332, fim_circshift fim.c:982-1057)
  Bertero weights       src/method_shb.c:216-253, initial_guess dw.c:2497-2520
  start FLAT / IDENTITY src/method_shb.c:255-294
  get_fIdiv / get_fMSE  src/dw.c:1492-1524 / 1461-1490 (here with log, not logf)

Differences from the reference, all on purpose: float64 everywhere; the
I-divergence uses the double log; iterations are a fixed count (the caller
passes the count the float32 run made, so both runs take the same steps).
Arrays are NumPy (P, N, M), x fastest, as in the fim layout.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np


@dataclass
class Fp64Result:
    out: np.ndarray        # (P, N, M) float64
    trace: np.ndarray      # I-divergence (or MSE) per iteration, float64
    bg: float
    work: tuple            # job size (wP, wN, wM)


def job_size(shape, psf_shape, bq: int):
    """method_shb.c:137-153 (same rule in method_rl.c)."""
    out = []
    for s, p in zip(shape, psf_shape):
        if bq == 2:
            out.append(s + p - 1)
        elif bq == 1:
            out.append(s + (p + 1) // 2)
        else:
            out.append(max(s, p))
    return tuple(out)


def _idiv(y, g):
    """get_fIdiv (dw.c:1492-1524) in double: mean over the image of
    g*log(g/y) - (g - y) where y > 0 and g > 0."""
    m = (y > 0) & (g > 0)
    gm, ym = g[m], y[m]
    return float((gm * np.log(gm / ym) - (gm - ym)).sum() / g.size)


def _mse(y, g):
    """get_fMSE (dw.c:1461-1490)."""
    d = y - g
    return float((d * d).sum() / g.size)


def deconvolve_fp64(im: np.ndarray, psf: np.ndarray, method: str = "shb", n_iter: int = 50, bq: int = 2,
                    bg: float | None = None, positivity: bool = True, alphamax: float = 1.0,
                    start: str = "flat", metric: str = "idiv", workers: int | None = None) -> Fp64Result:
    import scipy.fft as sfft
    workers = workers or os.cpu_count() or 1
    g = np.asarray(im, dtype=np.float64)
    P, N, M = g.shape
    if n_iter == 0:  # method_shb.c:101-105
        return Fp64Result(g.copy(), np.zeros(0), float(bg or 0), g.shape)
    if bg is None:  # method_shb.c:108-117
        bg = max(float(g.min()), 0.01)
    w = job_size(g.shape, psf.shape, bq)
    img = (slice(0, P), slice(0, N), slice(0, M))

    # OTF: PSF at the corner, argmax (lowest index) moved to the origin
    Z = np.zeros(w, dtype=np.float64)
    pP, pN, pM = psf.shape
    Z[:pP, :pN, :pM] = psf
    c, b, a = np.unravel_index(int(np.argmax(Z)), w)
    Z = np.roll(Z, shift=(-c, -b, -a), axis=(0, 1, 2))
    K = sfft.rfftn(Z, workers=workers)
    Kc = np.conj(K)
    del Z

    def conv(X, H):
        return sfft.irfftn(sfft.rfftn(X, workers=workers) * H, s=w, workers=workers)

    W = None
    if bq > 0:  # Bertero weights: 1/P1 where P1 = K^T 1_image > 0.01
        one = np.zeros(w)
        one[img] = 1.0
        P1 = conv(one, Kc)
        W = np.where(P1 > 0.01, 1.0 / np.where(P1 > 0.01, P1, 1.0), 0.0)
        del one, P1

    if start == "flat":
        x = np.full(w, g.sum() / float(np.prod(w)))
    elif start == "identity":
        x = np.zeros(w)
        x[img] = g
    else:
        raise ValueError("start must be 'flat' or 'identity'")
    xp = x.copy()
    err_of = _idiv if metric == "idiv" else _mse
    trace = np.zeros(n_iter)
    shb = method == "shb"
    for it in range(n_iter):
        if shb:
            # method_shb.c:325-339
            alpha = min(max((it - 1.0) / (it + 2.0), 0.0), alphamax)
            p = np.maximum(x + alpha * (x - xp), bg)
            # iter_shb
            y = conv(p, K)
            ys = y[img]
            trace[it] = err_of(ys, g)
            ys = np.where(np.abs(ys) < 1e-6, np.copysign(1e-6, ys), ys)
            r = np.zeros(w)
            r[img] = g / ys
            xn = conv(r, Kc) * (p * W if W is not None else p)
            xp, x = x, xn
            if positivity:
                x = np.maximum(x, bg)
        else:
            # iter_rl: f = current guess
            f = x
            y = conv(f, K)
            ys = y[img]
            trace[it] = err_of(ys, g)
            r = np.full(w, 1e-6)
            pos = ys > 0
            r[img] = np.where(pos, g / np.where(pos, ys, 1.0), bg)
            xn = conv(r, Kc) * (f * W if W is not None else f)
            if bg > 0:  # method_rl.c:362-372
                xn = np.maximum(xn, bg)
            x = xn
    # SHB returns the iterate before the last update (method_shb.c:385-413),
    # RL the newest one (method_rl.c:393)
    res = xp if shb else x
    return Fp64Result(np.ascontiguousarray(res[img]), trace, float(bg), w)
