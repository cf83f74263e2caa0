"""The periodic-margin scheme of the engine for border_quality 0/1 at job
sizes without an exact transform (CPU, numpy): a field of period w is
transformed at a length W >= w + 2h with [w, w+h) and [W-h, W) holding
copies of [0, h) and [w-h, w) and zeros between; its convolution with a PSF
of half-width h (shifted so that its centre is at the origin), and the
adjoint (correlation), then equal the period-w circular ones on [0, w).
The OTF itself is not wrapped."""
import numpy as np
import pytest


def _margins(f, W, h):
    w = f.shape[0]
    g = np.zeros((W,) + f.shape[1:], f.dtype)
    g[:w] = f
    g[w:w + h] = f[:h]
    g[W - h:] = f[w - h:]
    return g


def _embed_psf(p, n):
    # centre at the origin, negative offsets wrapped to the end
    h = (p.shape[0] - 1) // 2
    k = np.zeros(n)
    for d in range(-h, h + 1):
        k[d % n] = p[d + h]
    return k


@pytest.mark.parametrize("w,p,W", [(25, 5, 36), (26, 7, 32), (37, 11, 48), (61, 7, 72), (13, 13, 40)])
def test_margins_give_the_circular_convolution(w, p, W):
    rng = np.random.default_rng(w * 100 + p)
    h = (p - 1) // 2
    assert W >= w + 2 * h
    f = rng.random(w)
    psf = rng.random(p)
    circ = np.real(np.fft.ifft(np.fft.fft(f) * np.fft.fft(_embed_psf(psf, w))))
    circ_t = np.real(np.fft.ifft(np.fft.fft(f) * np.conj(np.fft.fft(_embed_psf(psf, w)))))
    K = np.fft.fft(_embed_psf(psf, W))  # the OTF at the longer length, not wrapped
    g = _margins(f, W, h)
    lin = np.real(np.fft.ifft(np.fft.fft(g) * K))[:w]
    lin_t = np.real(np.fft.ifft(np.fft.fft(g) * np.conj(K)))[:w]
    np.testing.assert_allclose(lin, circ, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(lin_t, circ_t, rtol=1e-12, atol=1e-12)


def test_three_axes_at_once():
    """Margins along every axis (y and z margins as whole rows copied after
    the x margins) give the 3-D circular convolution."""
    rng = np.random.default_rng(7)
    w = (9, 13, 11)
    p = (5, 7, 3)
    W = (16, 24, 14)
    f = rng.random(w)
    circ_k = np.ones(w, complex)
    lin_k = np.ones(W, complex)
    # a separable PSF for brevity: the product of one profile per axis
    prof = [rng.random(n) for n in p]
    for ax in range(3):
        shape = [1, 1, 1]
        shape[ax] = -1
        circ_k = circ_k * np.fft.fft(_embed_psf(prof[ax], w[ax])).reshape(shape)
        lin_k = lin_k * np.fft.fft(_embed_psf(prof[ax], W[ax])).reshape(shape)
    g = f
    for ax in range(3):
        g = np.moveaxis(_margins(np.moveaxis(g, ax, 0), W[ax], (p[ax] - 1) // 2), 0, ax)
    circ = np.real(np.fft.ifftn(np.fft.fftn(f) * circ_k))
    lin = np.real(np.fft.ifftn(np.fft.fftn(g) * lin_k))[: w[0], : w[1], : w[2]]
    np.testing.assert_allclose(lin, circ, rtol=1e-12, atol=1e-12)
