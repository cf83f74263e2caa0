"""CPU tests of the oracle: the C restatement (port) is pinned against
deconwolf's own method code compiled unmodified (oracle/_ref), and the FFT
underneath both against the known-answer tests of the reference's fft.c."""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from tests.helpers import gauss_psf, poisson_image, rel_l2

pytestmark = pytest.mark.skipif(not po.available("port"), reason="oracle not built (make -C oracle)")

need_ref = pytest.mark.skipif(not po.available("reference"),
                              reason="oracle/_ref not built (needs the reference sources at build time)")


def small_case(seed=1, shape=(9, 22, 19), psf_shape=(5, 7, 9)):
    psf = gauss_psf(psf_shape, (1.2, 1.5, 1.7), seed=seed, jitter=0.2)
    im = poisson_image(shape, psf, seed=seed, bg=50.0, npts=15)
    return im, psf


CASES = [
    dict(method="shb", iter_type=po.ITER_FIXED, n_iter=12),
    dict(method="rl", iter_type=po.ITER_FIXED, n_iter=12),
    dict(method="shb", iter_type=po.ITER_REL, err_rel=0.002),
    dict(method="rl", iter_type=po.ITER_REL, err_rel=0.002),
    dict(method="shb", iter_type=po.ITER_ABS, err_abs=1.5, maxiter=30),
    dict(method="shb", iter_type=po.ITER_FIXED, n_iter=7, border_quality=1),
    dict(method="rl", iter_type=po.ITER_FIXED, n_iter=7, border_quality=0),
    dict(method="shb", iter_type=po.ITER_FIXED, n_iter=6, start=po.START_IDENTITY),
    dict(method="rl", iter_type=po.ITER_FIXED, n_iter=6, metric=po.METRIC_MSE),
    dict(method="shb", iter_type=po.ITER_FIXED, n_iter=6, bg=3.0, positivity=False),
    dict(method="shb", iter_type=po.ITER_FIXED, n_iter=8, alphamax=0.3),
    dict(method="shb", iter_type=po.ITER_FIXED, n_iter=1),
    dict(method="shb", iter_type=po.ITER_FIXED, n_iter=0),
    dict(method="rl", iter_type=po.ITER_FIXED, n_iter=0),
]


@need_ref
@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}={v}" for k, v in c.items()))
def test_port_matches_reference(case):
    """The restatement reproduces deconwolf's compiled method code exactly
    (output, iteration count, error trace and automatic background)."""
    im, psf = small_case()
    a = po.deconvolve(im, psf, impl="port", threads=1, **case)
    b = po.deconvolve(im, psf, impl="reference", threads=1, **case)
    assert a.iterations == b.iterations
    np.testing.assert_array_equal(a.trace, b.trace)
    np.testing.assert_array_equal(a.out, b.out)
    assert a.bg == b.bg


@need_ref
def test_port_matches_reference_odd_shapes_threads():
    im, psf = small_case(seed=3, shape=(1, 17, 23), psf_shape=(1, 5, 7))  # a 2-D image
    for m in ("shb", "rl"):
        a = po.deconvolve(im, psf, method=m, n_iter=9, impl="port", threads=4)
        b = po.deconvolve(im, psf, method=m, n_iter=9, impl="reference", threads=4)
        np.testing.assert_array_equal(a.out, b.out)
        assert np.allclose(a.trace, b.trace, rtol=1e-6, atol=0)


def test_shb_semantics():
    """n_iter == 0 copies; SHB with one iteration returns its start estimate
    (the iterate before the last update, method_shb.c:385-395)."""
    im, psf = small_case()
    r0 = po.deconvolve(im, psf, method="shb", n_iter=0)
    np.testing.assert_array_equal(r0.out, im)
    r1 = po.deconvolve(im, psf, method="shb", n_iter=1)
    P, N, M = im.shape
    pP, pN, pM = psf.shape
    wmnp = (M + pM - 1) * (N + pN - 1) * (P + pP - 1)
    flat = np.float32(np.float32(im.astype(np.float64).sum()) / np.float32(wmnp))
    assert np.all(r1.out == flat)
    # the RL output after one iteration is not the start
    rl1 = po.deconvolve(im, psf, method="rl", n_iter=1)
    assert not np.all(rl1.out == flat)


def test_shb_alpha_sequence():
    """alpha_k = (k-1)/(k+2) clamped to [0, alphamax] (method_shb.c:328-330):
    with alphamax = 0 SHB is plain RL with a bg floor, shifted by one output
    (up to RL's 1e-6 ratio outside the image, method_rl.c:63, where SHB has 0)."""
    im, psf = small_case()
    shb = po.deconvolve(im, psf, method="shb", n_iter=6, alphamax=0.0, bg=1e-6, positivity=False)
    rl = po.deconvolve(im, psf, method="rl", n_iter=5, bg=1e-6)
    assert rel_l2(shb.out, rl.out) < 1e-4
    assert np.allclose(shb.trace[:5], rl.trace, rtol=1e-5)
    full = po.deconvolve(im, psf, method="shb", n_iter=6)
    assert rel_l2(full.out, shb.out) > 1e-3  # the extrapolation does change the result


def test_padding_is_exact_for_bq2():
    """Padding the job to a larger (7-smooth) size leaves the result unchanged
    up to FFT rounding when border_quality is 2 (both methods)."""
    im, psf = small_case()
    P, N, M = im.shape
    pP, pN, pM = psf.shape
    w = (M + pM - 1, N + pN - 1, P + pP - 1)
    for m in ("shb", "rl"):
        a = po.deconvolve(im, psf, method=m, n_iter=15)
        b = po.deconvolve(im, psf, method=m, n_iter=15, work=(w[0] + 9, w[1] + 4, w[2] + 7))
        assert rel_l2(b.out, a.out) < 1e-5
        assert np.max(np.abs(b.trace - a.trace) / a.trace) < 1e-6


def test_fft_round_trip_kat():
    """fft.c:708-780: fft -> ifft round trip, max relative error < 1e-5 on
    sizes 51-60 x 25-34 x 20-29."""
    rng = np.random.default_rng(5)
    for _ in range(6):
        M, N, P = int(rng.integers(51, 61)), int(rng.integers(25, 35)), int(rng.integers(20, 30))
        x = (5 + rng.random((P, N, M))).astype(np.float32)
        y = po.irfftn(po.rfftn(x), M) / np.float32(M * N * P)
        big = np.abs(x) > 1e-5
        assert np.max(np.abs((x[big] - y[big]) / x[big])) < 1e-5


def test_fft_flip_conj_kat():
    """fft.c:576-628: flip(X) (*) A == ifft(conj(fft(X)) fft(A)), MSE < 1e-5
    on 12 x 13 x 15.  The identity holds for the circular flip
    x[(-n) mod N]; fim_flipall (fim.c:568-583) reverses x[N-1-n], which is the
    circular flip shifted by one sample, so the flip is rolled by one here."""
    rng = np.random.default_rng(6)
    M, N, P = 12, 13, 15
    A = rng.random((P, N, M)).astype(np.float32)
    B = A.copy()
    Bf = np.empty_like(B)
    # fim_flipall: T[a,b,c] = A[M-1-a, N-1-b, P-1-c]
    Bf[:, :, :] = np.roll(B[::-1, ::-1, ::-1], 1, axis=(0, 1, 2))
    FA, FB, FBf = po.rfftn(A), po.rfftn(B), po.rfftn(Bf)
    Y1 = po.irfftn(FA * FBf, M) / np.float32(M * N * P)
    Y2 = po.irfftn(np.conj(FB) * FA, M) / np.float32(M * N * P)
    assert float(np.mean((Y1 - Y2) ** 2)) < 1e-5


def test_fft_matches_numpy():
    rng = np.random.default_rng(7)
    for shape in [(7, 9, 10), (3, 5, 382 // 2), (5, 6, 14)]:
        x = rng.random(shape).astype(np.float32)
        a = po.rfftn(x)
        b = np.fft.rfftn(x.astype(np.float64))
        assert np.max(np.abs(a - b)) / np.max(np.abs(b)) < 1e-6


def test_argmax_first_maximum():
    """fim_argmax_max (fim.c:269-332): ties resolve to the lowest index."""
    import ctypes
    lib = po._lib("port")
    a = np.zeros((4, 5, 6), dtype=np.float32)
    a[2, 3, 1] = 7
    a[1, 4, 5] = 7
    a[3, 0, 0] = 7
    m, n, p = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    lib.dwo_argmax(a.ctypes.data, 6, 5, 4, ctypes.byref(m), ctypes.byref(n), ctypes.byref(p))
    assert (p.value, n.value, m.value) == (1, 4, 5)


def test_idiv_definition():
    """get_fIdiv (dw.c:1492-1524) only counts voxels with y > 0 and g > 0."""
    g = np.array([[[0.0, 2.0, 3.0, 5.0]]], dtype=np.float32)
    y = np.array([[[1.0, 0.0, 4.0, 5.0]]], dtype=np.float32)
    ref = (3.0 * np.log(np.float32(3.0 / 4.0)) - (3.0 - 4.0) + 0.0) / 4.0
    assert abs(po.idiv(y, g) - np.float32(ref)) < 1e-7


GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", ["small_shb", "small_rl", "small_shb_rel"])
def test_port_reproduces_golden(name):
    """The committed fixtures were made by the reference build (make_golden.py);
    the port must reproduce them exactly on any machine."""
    f = os.path.join(GOLD, f"{name}.npz")
    if not os.path.exists(f):
        pytest.skip("fixture missing")
    d = np.load(f, allow_pickle=False)
    kw = {k[4:]: (v.item() if v.ndim == 0 else v) for k, v in d.items() if k.startswith("opt_")}
    r = po.deconvolve(d["image"], d["psf"], impl="port", **kw)
    assert r.iterations == int(d["iterations"])
    np.testing.assert_array_equal(r.trace, d["trace"])
    np.testing.assert_array_equal(r.out, d["out"])


@pytest.mark.skipif(not po.available("reference"), reason="oracle/_ref not built")
@pytest.mark.parametrize("shape", [(9, 22, 19), (1, 30, 26), (3, 60, 70), (40, 20, 56)])
@pytest.mark.parametrize("method", ["shb", "rl"])
def test_lp_start_port_equals_reference(shape, method):
    """The low-pass start (fim_gsmooth with sigma 8, fim.c:2240-2278) as
    restated in the port equals the reference's own, bit for bit."""
    psf = gauss_psf((3, 5, 5) if shape[0] < 5 else (5, 7, 9), (1.2, 1.5, 1.7), seed=2, jitter=0.2)
    im = poisson_image(shape, psf, seed=2, bg=50.0, npts=12)
    a = po.deconvolve(im, psf, method=method, n_iter=3, start=po.START_LP)
    b = po.deconvolve(im, psf, method=method, n_iter=3, start=po.START_LP, impl="reference")
    np.testing.assert_array_equal(a.out, b.out)
    np.testing.assert_array_equal(a.trace, b.trace)


@need_ref
@pytest.mark.parametrize("shape,psf_shape,bq", [
    ((9, 22, 20), (5, 7, 9), 1),     # job 25 x 26 x 12: odd x
    ((37, 40, 30), (11, 9, 9), 0),   # z period 37 (prime)
    ((20, 33, 44), (21, 15, 13), 0), # x 44, y 33
    ((12, 26, 31), (7, 9, 11), 1),   # job 37 x 31 x 16
])
def test_port_matches_reference_periodic_sizes(shape, psf_shape, bq):
    """The sizes the GPU runs with periodic margins: the restatement equals
    the reference at the reference's own (exact) job size, bit for bit."""
    im, psf = small_case(seed=6, shape=shape, psf_shape=psf_shape)
    for m in ("shb", "rl"):
        a = po.deconvolve(im, psf, method=m, n_iter=5, border_quality=bq, impl="port", threads=1)
        b = po.deconvolve(im, psf, method=m, n_iter=5, border_quality=bq, impl="reference", threads=1)
        np.testing.assert_array_equal(a.trace, b.trace)
        np.testing.assert_array_equal(a.out, b.out)
