"""Seeded synthetic microscopy inputs (benchmarks and tests).

Born-Wolf PSF
    Restates the model of deconwolf's PSF generator ``dw_bw``
    (src/dw_bwpsf.c:538-775, src/bw_gsl.c:79-111): the intensity at lateral
    distance r and defocus z is
        |int_0^1 J0(k0 NA r rho) exp(-i k0 NA^2 z rho^2 / (2 ni)) rho drho|^2,
    k0 = 2 pi / lambda, sampled as a radial profile with 17 samples per pixel
    (dw_bwpsf.c:658-690), integrated over each pixel (here: 5 x 5 sub-pixel
    samples instead of adaptive quadrature), mirrored in z, and normalised
    to sum 1.  The reference's adaptive GSL quadrature is replaced by a fixed
    Gauss-Legendre rule; fidelity to dw_bw is not pinned (the reference ships
    no PSF fixture) and does not affect deconvolution parity, which compares
    both engines on the same PSF array.

Image
    object = K point sources at uniform random voxels with lognormal(7, 0.5)
    intensities + B isotropic Gaussian blobs (sigma 8 px, peak 200);
    image = Poisson(background + object (*) PSF), clipped to [0, 65535] and
    stored as uint16 values in float32 -- the generator stated for the
    benchmark configurations (object, PSF and seeds per configuration below).
"""
from __future__ import annotations

import os

import numpy as np


def _gauss_legendre(n: int):
    x, w = np.polynomial.legendre.leggauss(n)
    return 0.5 * (x + 1.0), 0.5 * w  # on [0, 1]


def bw_radial(r_nm: np.ndarray, z_nm: float, lam: float, NA: float, ni: float, nq: int = 400) -> np.ndarray:
    from scipy.special import j0
    rho, w = _gauss_legendre(nq)
    k0 = 2.0 * np.pi / lam
    W = k0 * (NA ** 2) * z_nm * rho ** 2 / (2.0 * ni)
    B = j0(k0 * NA * np.outer(r_nm, rho))  # (nr, nq)
    re = B @ (np.cos(W) * rho * w)
    im = -(B @ (np.sin(W) * rho * w))
    return re * re + im * im


def bw_psf(shape=(79, 127, 127), lam=466.0, NA=1.4, ni=1.515, dxy=130.0, dz=300.0,
           oversampling: int = 17, subpix: int = 5) -> np.ndarray:
    """Born-Wolf PSF, array (P, N, M) float32 with sum 1, maximum at the centre."""
    P, N, M = shape
    if P % 2 == 0 or N % 2 == 0 or M % 2 == 0:
        raise ValueError("PSF sizes must be odd")
    cy, cx = (N - 1) / 2, (M - 1) / 2
    rmax = np.hypot(cx + 1, cy + 1)
    nr = int(np.ceil(rmax * oversampling)) + 4
    r_pix = np.arange(nr) / oversampling
    # sub-pixel sample offsets inside each pixel
    o = (np.arange(subpix) + 0.5) / subpix - 0.5
    yy = (np.arange(N) - cy)[:, None, None, None] + o[None, None, :, None]
    xx = (np.arange(M) - cx)[None, :, None, None] + o[None, None, None, :]
    rr = np.sqrt(yy ** 2 + xx ** 2)  # (N, M, s, s) in pixels
    V = np.empty((P, N, M), dtype=np.float64)
    for z in range((P + 1) // 2):
        defocus = dz * (z - (P - 1) / 2.0)
        prof = bw_radial(r_pix * dxy, defocus, lam, NA, ni)
        V[z] = np.interp(rr, r_pix, prof).mean(axis=(2, 3))
    for z in range((P - 1) // 2):
        V[P - 1 - z] = V[z]
    V /= V.sum()
    return V.astype(np.float32)


# configurations of the benchmark workloads (image size, PSF, counts, seed)
CONFIGS = {
    "shb-256x256x40": dict(shape=(40, 256, 256), psf_shape=(79, 127, 127), lam=466.0, K=1500, B=40, bg=100.0, seed=1),
    "shb-2048x2048x60": dict(shape=(60, 2048, 2048), psf_shape=(119, 181, 181), lam=670.0, K=40000, B=600, bg=100.0,
                             seed=2),
    # a mid-size case of the same kernels (per-voxel work as above, device
    # buffers > L2, a few GB on the device): used for hardware-counter captures
    "shb-1024x1024x20": dict(shape=(20, 1024, 1024), psf_shape=(39, 181, 181), lam=670.0, K=3300, B=50, bg=100.0,
                             seed=3),
}


def _add_blobs(obj: np.ndarray, rng, B: int, sigma: float = 8.0, amp: float = 200.0) -> None:
    P, N, M = obj.shape
    h = int(np.ceil(4 * sigma))
    g1 = np.exp(-0.5 * (np.arange(-h, h + 1) / sigma) ** 2)
    cz = rng.integers(0, P, B)
    cy = rng.integers(0, N, B)
    cx = rng.integers(0, M, B)
    for z0, y0, x0 in zip(cz, cy, cx):
        z1, z2 = max(0, z0 - h), min(P, z0 + h + 1)
        y1, y2 = max(0, y0 - h), min(N, y0 + h + 1)
        x1, x2 = max(0, x0 - h), min(M, x0 + h + 1)
        gz = g1[z1 - z0 + h:z2 - z0 + h]
        gy = g1[y1 - y0 + h:y2 - y0 + h]
        gx = g1[x1 - x0 + h:x2 - x0 + h]
        obj[z1:z2, y1:y2, x1:x2] += (amp * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]).astype(obj.dtype)


def synth_image(shape, psf: np.ndarray, K: int, B: int, bg: float, seed: int, workers: int | None = None) -> np.ndarray:
    """Poisson(bg + object (*) psf), 'same' linear convolution, uint16 values as float32."""
    import scipy.fft as sfft
    rng = np.random.default_rng(seed)
    P, N, M = shape
    obj = np.zeros(shape, dtype=np.float32)
    idx = (rng.integers(0, P, K), rng.integers(0, N, K), rng.integers(0, M, K))
    np.add.at(obj, idx, rng.lognormal(7.0, 0.5, K).astype(np.float32))
    _add_blobs(obj, rng, B)
    pP, pN, pM = psf.shape
    full = [sfft.next_fast_len(s + p - 1, real=True) for s, p in zip(shape, psf.shape)]
    workers = workers or os.cpu_count() or 1
    Fo = sfft.rfftn(obj, s=full, workers=workers)
    del obj
    Fo *= sfft.rfftn(psf, s=full, workers=workers)
    conv = sfft.irfftn(Fo, s=full, workers=workers)
    del Fo
    a, b, c = (pP - 1) // 2, (pN - 1) // 2, (pM - 1) // 2
    blur = conv[a:a + P, b:b + N, c:c + M]
    lam = np.clip(bg + blur.astype(np.float64), 0, None)
    del conv
    img = rng.poisson(lam)
    return np.clip(img, 0, 65535).astype(np.uint16).astype(np.float32)


def config_inputs(name: str, cache_dir: str | None = None):
    """(image, psf) of a named configuration, generated from its seed; cached
    as .npy under cache_dir when given."""
    c = CONFIGS[name]
    if cache_dir:
        os.makedirs(cache_dir, exist_ok=True)
        fi = os.path.join(cache_dir, f"{name}_image.npy")
        fp = os.path.join(cache_dir, f"{name}_psf.npy")
        if os.path.exists(fi) and os.path.exists(fp):
            return np.load(fi), np.load(fp)
    psf = bw_psf(c["psf_shape"], lam=c["lam"])
    im = synth_image(c["shape"], psf, c["K"], c["B"], c["bg"], c["seed"])
    if cache_dir:
        np.save(fi, im)
        np.save(fp, psf)
    return im, psf
