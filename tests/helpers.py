"""Shared test inputs: small seeded images and PSFs (synthetic, deterministic)."""
import numpy as np


def gauss_psf(shape, sigma, seed=0, jitter=0.0):
    """Anisotropic Gaussian PSF with its maximum at the centre (odd shape)."""
    pP, pN, pM = shape
    z = np.arange(pP) - (pP - 1) / 2
    y = np.arange(pN) - (pN - 1) / 2
    x = np.arange(pM) - (pM - 1) / 2
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    sz, sy, sx = sigma
    p = np.exp(-0.5 * ((Z / sz) ** 2 + (Y / sy) ** 2 + (X / sx) ** 2))
    if jitter:
        rng = np.random.default_rng(seed)
        p *= 1 + jitter * rng.random(p.shape)
        c = tuple((s - 1) // 2 for s in shape)
        p[c] = p.max() * 1.01
    p /= p.sum()
    return p.astype(np.float32)


def poisson_image(shape, psf, seed=1, bg=100.0, npts=40, amp=2000.0):
    """Poisson(bg + points convolved with the PSF), stored as uint16 values."""
    from scipy.signal import fftconvolve
    rng = np.random.default_rng(seed)
    obj = np.zeros(shape, dtype=np.float64)
    idx = tuple(rng.integers(0, s, npts) for s in shape)
    obj[idx] += amp * rng.lognormal(0, 0.5, npts)
    blur = fftconvolve(obj, psf.astype(np.float64), mode="same")
    img = rng.poisson(np.clip(bg + blur, 0, None))
    return np.clip(img, 0, 65535).astype(np.uint16).astype(np.float32)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
