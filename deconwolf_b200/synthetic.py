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
    # small cases whose x, y or z transform length is that of the 2048^2 x 60
    # workload (2240, 2240, 180), so one axis's kernel is exactly the one it
    # runs, on ~1 GB of device memory: hardware-counter captures
    "shb-2048x256x20": dict(shape=(20, 256, 2048), psf_shape=(39, 181, 181), lam=670.0, K=800, B=12, bg=100.0,
                            seed=4),
    "shb-256x2048x20": dict(shape=(20, 2048, 256), psf_shape=(39, 181, 181), lam=670.0, K=800, B=12, bg=100.0,
                            seed=5),
    "shb-256x256x60": dict(shape=(60, 256, 256), psf_shape=(119, 181, 181), lam=670.0, K=600, B=9, bg=100.0,
                           seed=6),
    # one interior tile of the 4096^2 x 60 image at tile size 1024 and
    # overlap 50 (1124^2 x 60, job 1344^2 x 180)
    "shb-1124x1124x60": dict(shape=(60, 1124, 1124), psf_shape=(119, 181, 181), lam=670.0, K=12000, B=180,
                             bg=100.0, seed=7),
    # one tile of the same image at tile size 512 and overlap 50 (612 x 562 x
    # 60, job 792 x 742 x 178 -> 800 x 750 x 180)
    "shb-612x562x60": dict(shape=(60, 562, 612), psf_shape=(119, 181, 181), lam=670.0, K=3300, B=50, bg=100.0,
                           seed=8),
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


def synth_image_blocked(shape, psf: np.ndarray, K: int, B: int, bg: float, seed: int, block: int = 512,
                        workers: int | None = None) -> np.ndarray:
    """synth_image for large volumes: the same object model (K points, B
    blobs, from ``seed``), convolved block by block in x/y (each output block
    from the object block grown by the PSF half-widths, so the result equals
    the whole-volume 'same' convolution up to FFT rounding), then Poisson
    noise per block (a per-block stream derived from ``seed``)."""
    import scipy.fft as sfft
    rng = np.random.default_rng(seed)
    P, N, M = shape
    obj = np.zeros(shape, dtype=np.float32)
    idx = (rng.integers(0, P, K), rng.integers(0, N, K), rng.integers(0, M, K))
    np.add.at(obj, idx, rng.lognormal(7.0, 0.5, K).astype(np.float32))
    _add_blobs(obj, rng, B)
    pP, pN, pM = psf.shape
    hz, hy, hx = (pP - 1) // 2, (pN - 1) // 2, (pM - 1) // 2
    workers = workers or os.cpu_count() or 1
    out = np.empty(shape, dtype=np.float32)
    # object zero-padded by the PSF half widths on every side
    objp = np.zeros((P + 2 * hz, N + 2 * hy, M + 2 * hx), dtype=np.float32)
    objp[hz:hz + P, hy:hy + N, hx:hx + M] = obj
    del obj
    Fp = {}
    for y0 in range(0, N, block):
        for x0 in range(0, M, block):
            by, bx = min(block, N - y0), min(block, M - x0)
            sub = objp[:, y0:y0 + by + 2 * hy, x0:x0 + bx + 2 * hx]
            full = [sfft.next_fast_len(s, real=True) for s in sub.shape]
            key = tuple(full)
            if key not in Fp:
                Fp[key] = sfft.rfftn(psf, s=full, workers=workers)
            conv = sfft.irfftn(sfft.rfftn(sub, s=full, workers=workers) * Fp[key], s=full, workers=workers)
            blur = conv[2 * hz:2 * hz + P, 2 * hy:2 * hy + by, 2 * hx:2 * hx + bx]
            lam = np.clip(bg + blur.astype(np.float64), 0, None)
            brng = np.random.default_rng([seed, y0, x0])
            out[:, y0:y0 + by, x0:x0 + bx] = np.clip(brng.poisson(lam), 0, 65535).astype(np.uint16)
    return out


def _save_atomic(path: str, a: np.ndarray) -> None:
    """np.save through a private temporary file and a rename, so that
    processes sharing the cache (one per GPU) never read a partial file."""
    tmp = f"{path}.{os.getpid()}.tmp.npy"
    np.save(tmp, a)
    os.replace(tmp, path)


def cached(name: str, cache_dir: str | None, make):
    """(image, psf) from ``make()``, cached as .npy under cache_dir."""
    if cache_dir:
        os.makedirs(cache_dir, exist_ok=True)
        fi = os.path.join(cache_dir, f"{name}_image.npy")
        fp = os.path.join(cache_dir, f"{name}_psf.npy")
        if os.path.exists(fi) and os.path.exists(fp):
            return np.load(fi), np.load(fp)
    im, psf = make()
    if cache_dir:
        _save_atomic(fi, im)
        _save_atomic(fp, psf)
    return im, psf


def tiled_inputs(cache_dir: str | None = None):
    """The 4096 x 4096 x 60 tiled workload: the generator of the 2048 x 2048
    x 60 workload scaled by area (K = 160000, B = 2400), seed 3, PSF
    Born-Wolf 670 nm 181 x 181 x 119."""
    def make():
        psf = bw_psf((119, 181, 181), lam=670.0)
        return synth_image_blocked((60, 4096, 4096), psf, 160000, 2400, 100.0, 3), psf
    return cached("tiles-4096x4096x60", cache_dir, make)


def tiled_pair_inputs(cache_dir: str | None = None):
    """A 2048 x 1024 x 60 image that tiling splits into two tiles at tile
    size 1024 and overlap 50: the generator of the 2048 x 2048 x 60 workload
    scaled by area (K = 20000, B = 300), seed 9; PSF Born-Wolf 670 nm
    181 x 181 x 119."""
    def make():
        psf = bw_psf((119, 181, 181), lam=670.0)
        return synth_image_blocked((60, 1024, 2048), psf, 20000, 300, 100.0, 9), psf
    return cached("tiles-2048x1024x60", cache_dir, make)


CHANNEL_LAMBDAS = (405.0, 466.0, 525.0, 595.0, 670.0, 750.0)
CHANNEL_ITERS = (20, 40, 60, 80, 100, 150)


def channel_spec(c: int):
    """Channel c of the multi-channel field of view: xy side from 512 to 2048,
    z from 30 to 80 slices and background 80-150, drawn with seed 40 + c; PSF
    Born-Wolf at the channel's wavelength, 181 x 181 x (2P - 1)."""
    rng = np.random.default_rng(40 + c)
    side = int(rng.choice([512, 768, 1024, 1536, 2048]))
    P = int(rng.integers(30, 81))
    bg = float(rng.integers(80, 151))
    area = side * side * P / (2048 * 2048 * 60)
    return dict(shape=(P, side, side), psf_shape=(2 * P - 1, 181, 181), lam=CHANNEL_LAMBDAS[c],
                iters=CHANNEL_ITERS[c], bg=bg, K=max(1, int(40000 * area)), B=max(1, int(600 * area)), seed=40 + c)


def channel_inputs(c: int, cache_dir: str | None = None):
    sp = channel_spec(c)

    def make():
        psf = bw_psf(sp["psf_shape"], lam=sp["lam"])
        return synth_image_blocked(sp["shape"], psf, sp["K"], sp["B"], sp["bg"], sp["seed"]), psf
    return cached(f"channel{c}", cache_dir, make)


SERVE_SIZES = ((20, 256, 256), (40, 512, 512), (60, 1024, 1024), (80, 2048, 2048))


def serve_requests(n: int, rate: float = 2.0, seed: int = 5):
    """The serving stream: Poisson arrivals at ``rate`` per second; size class
    uniform over SERVE_SIZES, wavelength uniform over CHANNEL_LAMBDAS,
    iterations uniform in [20, 200], SHB or RL with probability 1/2."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    t -= t[0]
    out = []
    for i in range(n):
        out.append(dict(arrival=float(t[i]), size=int(rng.integers(0, len(SERVE_SIZES))),
                        lam=float(rng.choice(CHANNEL_LAMBDAS)), iters=int(rng.integers(20, 201)),
                        method="shb" if rng.random() < 0.5 else "rl"))
    return out


def serve_image(size: int, variant: int, cache_dir: str | None = None):
    """Image ``variant`` (0 or 1) of size class ``size`` (seed 5000 + 10*size
    + variant), blurred with the 525 nm PSF of that size."""
    shape = SERVE_SIZES[size]
    P, N, M = shape
    area = N * M * P / (2048 * 2048 * 60)

    def make():
        psf = bw_psf((2 * P - 1, 181, 181), lam=525.0)
        im = synth_image_blocked(shape, psf, max(1, int(40000 * area)), max(1, int(600 * area)), 100.0,
                                 5000 + 10 * size + variant)
        return im, psf
    return cached(f"serve{size}_{variant}", cache_dir, make)


def serve_psf(size: int, lam: float, cache_dir: str | None = None) -> np.ndarray:
    P = SERVE_SIZES[size][0]
    if cache_dir:
        f = os.path.join(cache_dir, f"servepsf{size}_{int(lam)}.npy")
        if os.path.exists(f):
            return np.load(f)
    psf = bw_psf((2 * P - 1, 181, 181), lam=lam)
    if cache_dir:
        os.makedirs(cache_dir, exist_ok=True)
        _save_atomic(f, psf)
    return psf


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
        _save_atomic(fi, im)
        _save_atomic(fp, psf)
    return im, psf
