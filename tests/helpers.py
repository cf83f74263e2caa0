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


# ---------------------------------------------------------------- sketches
# A full-volume check for outputs too large to store as a fixture: k rows of
# pseudo-random +-1 signs (a seeded integer hash of the voxel index, the same
# on every device) projected onto the flattened volume, summed in float64.
# For any vector d, ||S d||^2 / k estimates ||d||^2 without bias (relative
# spread about sqrt(2 / k)), so ||S a - S b|| / (sqrt(k) ||b||) estimates the
# relative L2 distance of a and b over every voxel.
_P31 = 2147483647
SKETCH_ROWS = 32


def _sketch_consts(k):
    rng = np.random.default_rng(20240611)
    return (rng.integers(1, _P31, k), rng.integers(0, _P31, k), rng.integers(0, _P31, k))


def sketch(v, k: int = SKETCH_ROWS, device: str = "cpu", chunk: int = 1 << 24) -> np.ndarray:
    """S v for the flattened volume v (NumPy or torch), as float64[k]."""
    import torch
    t = v if isinstance(v, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(v))
    t = t.reshape(-1).to(device)
    A, B, C = _sketch_consts(k)
    out = np.zeros(k, dtype=np.float64)
    n = t.numel()
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        i = torch.arange(s, e, dtype=torch.int64, device=device)
        vv = t[s:e].to(torch.float64)
        for j in range(k):
            h = (i * int(A[j]) + int(B[j])) % _P31       # < 2^62: no overflow
            h = (h * h + int(C[j])) % _P31
            sgn = ((h >> 16) & 1).to(torch.float64) * 2 - 1
            out[j] += float((sgn * vv).sum())
    return out


def sketch_rel_l2(sk_a, sk_b, norm_b: float) -> float:
    """Estimated relative L2 distance of a to b from their sketches."""
    k = len(sk_a)
    return float(np.linalg.norm(np.asarray(sk_a) - np.asarray(sk_b)) / (np.sqrt(k) * norm_b))
