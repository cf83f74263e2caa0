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


def deconvolve_fp64_torch(im: np.ndarray, psf: np.ndarray, method: str = "shb", n_iter: int = 50, bq: int = 2,
                          bg: float | None = None, positivity: bool = True, alphamax: float = 1.0,
                          device: str = "cpu") -> Fp64Result:
    """deconvolve_fp64 with torch float64 tensors and transforms (on ``device``,
    e.g. a GPU for volumes too large for host memory in float64); the same
    steps, flat start, I-divergence.  Returns the result on the host."""
    import torch
    g = torch.as_tensor(np.asarray(im, dtype=np.float64), device=device)
    P, N, M = g.shape
    if n_iter == 0:
        return Fp64Result(g.cpu().numpy(), np.zeros(0), float(bg or 0), tuple(g.shape))
    if bg is None:
        bg = max(float(g.min()), 0.01)
    w = job_size(tuple(g.shape), psf.shape, bq)
    Z = torch.zeros(w, dtype=torch.float64, device=device)
    pP, pN, pM = psf.shape
    Z[:pP, :pN, :pM] = torch.as_tensor(np.asarray(psf, dtype=np.float64), device=device)
    c, b, a = np.unravel_index(int(torch.argmax(Z).item()), w)
    Z = torch.roll(Z, shifts=(-int(c), -int(b), -int(a)), dims=(0, 1, 2))
    K = torch.fft.rfftn(Z)
    del Z
    Kc = torch.conj(K)

    def conv(X, H):
        return torch.fft.irfftn(torch.fft.rfftn(X) * H, s=w)

    W = None
    if bq > 0:
        one = torch.zeros(w, dtype=torch.float64, device=device)
        one[:P, :N, :M] = 1.0
        P1 = conv(one, Kc)
        del one
        W = torch.where(P1 > 0.01, 1.0 / torch.where(P1 > 0.01, P1, torch.ones_like(P1)), torch.zeros_like(P1))
        del P1
    x = torch.full(w, float(g.sum().item()) / float(np.prod(w)), dtype=torch.float64, device=device)
    xp = x.clone()
    trace = np.zeros(n_iter)
    shb = method == "shb"

    def idiv(ys):
        m = (ys > 0) & (g > 0)
        gm, ym = g[m], ys[m]
        return float(((gm * torch.log(gm / ym)) - (gm - ym)).sum().item() / g.numel())

    for it in range(n_iter):
        if shb:
            alpha = min(max((it - 1.0) / (it + 2.0), 0.0), alphamax)
            p = torch.clamp(x + alpha * (x - xp), min=bg)
            y = conv(p, K)
            ys = y[:P, :N, :M]
            trace[it] = idiv(ys)
            ys = torch.where(ys.abs() < 1e-6, torch.copysign(torch.full_like(ys, 1e-6), ys), ys)
            r = torch.zeros(w, dtype=torch.float64, device=device)
            r[:P, :N, :M] = g / ys
            del y, ys
            xn = conv(r, Kc) * (p * W if W is not None else p)
            del r, p
            xp, x = x, xn
            if positivity:
                x = torch.clamp(x, min=bg)
        else:
            f = x
            y = conv(f, K)
            ys = y[:P, :N, :M]
            trace[it] = idiv(ys)
            r = torch.full(w, 1e-6, dtype=torch.float64, device=device)
            pos = ys > 0
            r[:P, :N, :M] = torch.where(pos, g / torch.where(pos, ys, torch.ones_like(ys)), torch.full_like(ys, bg))
            del y, ys
            xn = conv(r, Kc) * (f * W if W is not None else f)
            if bg > 0:
                xn = torch.clamp(xn, min=bg)
            x = xn
    res = xp if shb else x
    return Fp64Result(res[:P, :N, :M].contiguous().cpu().numpy(), trace, float(bg), w)
