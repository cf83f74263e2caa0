"""GPU parity tests: the sm_100a engine, called through the C ABI, against
the oracle (tests-only CPU checker).

Tolerances (FP32 arithmetic, as in the reference):
  * against the reference at its own job size: relative L2 of the output
    <= 1e-4 and relative error of every I-divergence value <= 1e-5;
  * against the oracle run at the same padded job size as the GPU (which
    isolates FFT rounding): the same bounds, usually met by a wide margin.
"""
import ctypes
import os

import numpy as np
import pytest

import deconwolf_b200 as dw
from oracle import pyoracle as po
from tests.helpers import gauss_psf, poisson_image, rel_l2

pytestmark = pytest.mark.gpu

OUT_TOL = 1e-4
TRACE_TOL = 1e-5


def trace_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.abs(b)))


def case_inputs(seed=1, shape=(9, 22, 19), psf_shape=(5, 7, 9)):
    psf = gauss_psf(psf_shape, (1.2, 1.5, 1.7), seed=seed, jitter=0.2)
    im = poisson_image(shape, psf, seed=seed, bg=50.0, npts=15)
    return im, psf


def checker(**kw):
    return "reference" if po.available("reference") else "port"


CASES = [
    dict(method="shb", n_iter=12),
    dict(method="rl", n_iter=12),
    dict(method="shb", n_iter=30),
    dict(method="shb", iter_type=po.ITER_REL, err_rel=0.002),
    dict(method="rl", iter_type=po.ITER_REL, err_rel=0.002),
    dict(method="shb", iter_type=po.ITER_ABS, err_abs=1.5, maxiter=30),
    dict(method="shb", n_iter=6, start=po.START_IDENTITY),
    dict(method="rl", n_iter=6, metric=po.METRIC_MSE),
    dict(method="shb", n_iter=6, bg=3.0, positivity=False),
    dict(method="shb", n_iter=8, alphamax=0.3),
    dict(method="rl", n_iter=5, bg=0.5),
    dict(method="shb", n_iter=7, start=po.START_LP),
    dict(method="rl", n_iter=7, start=po.START_LP),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}={v}" for k, v in c.items()))
def test_method_matches_oracle(case):
    im, psf = case_inputs()
    g = dw.run_method(im, psf, **case)
    # same padded job size as the GPU
    p = po.deconvolve(im, psf, work=g.work, **case)
    assert g.iterations == p.iterations
    assert rel_l2(g.out, p.out) < OUT_TOL
    assert trace_err(g.trace, p.trace) < TRACE_TOL
    # the reference at its own job size
    r = po.deconvolve(im, psf, impl=checker(), **case)
    assert g.iterations == r.iterations
    assert rel_l2(g.out, r.out) < OUT_TOL
    assert trace_err(g.trace, r.trace) < TRACE_TOL
    assert abs(g.bg - r.bg) <= 1e-6 * max(1.0, abs(r.bg))


@pytest.mark.parametrize("shape,psf_shape,bq", [
    ((1, 30, 26), (1, 7, 9), 2),        # 2-D image: z length 1
    ((6, 17, 31), (3, 5, 5), 2),        # odd sizes
    ((20, 50, 60), (7, 7, 7), 1),       # bq 1 on an exact supported job 64 x 54 x 24
    ((16, 60, 60), (9, 9, 9), 0),       # bq 0: job = image size 60 x 60 x 16
    ((5, 40, 3), (5, 9, 3), 2),         # thin x
])
def test_shapes_and_border_quality(shape, psf_shape, bq):
    im, psf = case_inputs(seed=4, shape=shape, psf_shape=psf_shape)
    for m in ("shb", "rl"):
        g = dw.run_method(im, psf, method=m, n_iter=10, border_quality=bq)
        r = po.deconvolve(im, psf, method=m, n_iter=10, border_quality=bq, impl=checker())
        assert rel_l2(g.out, r.out) < OUT_TOL, m
        assert trace_err(g.trace, r.trace) < TRACE_TOL, m


PERIODIC = [
    ((9, 22, 20), (5, 7, 9), 1),     # bq 1: x 25 (odd) and y 26 periodic, z 12 exact
    ((37, 40, 30), (11, 9, 9), 0),   # bq 0: z period 37 (prime)
    ((20, 33, 44), (21, 15, 13), 0), # bq 0: x 44 (22 = 2*11) and y 33 periodic, z 21 exact
    ((12, 26, 31), (7, 9, 11), 1),   # bq 1: every axis periodic (37, 31, 16 -> x odd, y prime)
]


@pytest.mark.parametrize("shape,psf_shape,bq", PERIODIC)
@pytest.mark.parametrize("kw", [dict(method="shb", n_iter=10), dict(method="rl", n_iter=8),
                                dict(method="shb", iter_type=po.ITER_REL, err_rel=0.005)],
                         ids=["shb", "rl", "shb-rel"])
def test_periodic_sizes_match_reference(shape, psf_shape, bq, kw):
    """border_quality 0/1 at job sizes without an exact transform: the
    circular convolution of the reference's job size is carried out at a
    longer length with periodic margins; against the reference at its own
    (exact) size."""
    im, psf = case_inputs(seed=6, shape=shape, psf_shape=psf_shape)
    g = dw.run_method(im, psf, border_quality=bq, **kw)
    r = po.deconvolve(im, psf, border_quality=bq, impl=checker(), **kw)
    assert g.iterations == r.iterations
    assert rel_l2(g.out, r.out) < OUT_TOL
    assert trace_err(g.trace, r.trace) < TRACE_TOL


def test_identity_and_first_iteration():
    im, psf = case_inputs()
    np.testing.assert_array_equal(dw.run_method(im, psf, n_iter=0).out, im)
    g = dw.run_method(im, psf, method="shb", n_iter=1)
    r = po.deconvolve(im, psf, method="shb", n_iter=1, impl=checker())
    np.testing.assert_array_equal(g.out, r.out)  # the flat start, bit for bit


@pytest.mark.parametrize("shape", [(9, 22, 19), (1, 30, 26), (3, 60, 70), (40, 20, 56), (80, 64, 60)])
def test_lp_start_equals_reference_bitwise(shape):
    """The low-pass start (fim_gsmooth, sigma 8): SHB's output after one
    iteration is the start estimate itself, equal to the reference's bit for
    bit (thin z trims the kernel; lines shorter than its 49 taps take the
    renormalised branch)."""
    im, psf = case_inputs(seed=5, shape=shape, psf_shape=(3, 5, 5) if shape[0] < 5 else (5, 7, 9))
    g = dw.run_method(im, psf, method="shb", n_iter=1, start=dw.START_LP)
    r = po.deconvolve(im, psf, method="shb", n_iter=1, start=po.START_LP, impl=checker())
    np.testing.assert_array_equal(g.out, r.out)


@pytest.mark.parametrize("name", ["small_shb", "small_rl", "small_shb_rel"])
def test_golden_fixtures(name):
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", f"{name}.npz"))
    kw = {k[4:]: (v.item() if v.ndim == 0 else v) for k, v in d.items() if k.startswith("opt_")}
    g = dw.run_method(d["image"], d["psf"], **kw)
    assert g.iterations == int(d["iterations"])
    assert rel_l2(g.out, d["out"]) < OUT_TOL
    assert trace_err(g.trace, d["trace"]) < TRACE_TOL


def test_config1_golden():
    """256 x 256 x 40, Born-Wolf 127 x 127 x 79 PSF, SHB 50 iterations against
    the reference's own output (sampled voxels, plane sums, full trace)."""
    f = os.path.join(os.path.dirname(__file__), "golden", "config1_shb50.npz")
    if not os.path.exists(f):
        pytest.skip("config1 fixture not generated")
    from deconwolf_b200 import synthetic
    d = np.load(f)
    im, psf = synthetic.config_inputs("shb-256x256x40")
    idx = d["sample_idx"]
    np.testing.assert_array_equal(im.reshape(-1)[idx], d["image_sample"])  # same inputs as the fixture
    g = dw.run_method(im, psf, method="shb", n_iter=50)
    assert g.work == (384, 384, 120)
    assert trace_err(g.trace, d["trace"]) < TRACE_TOL
    assert rel_l2(g.out.reshape(-1)[idx], d["sample_val"]) < OUT_TOL
    assert rel_l2(g.out.astype(np.float64).sum(axis=(1, 2)), d["plane_sums"]) < OUT_TOL
    assert abs(np.linalg.norm(g.out.astype(np.float64)) / d["norm"] - 1) < OUT_TOL


def test_config2_golden():
    """2048 x 2048 x 60, Born-Wolf 181 x 181 x 119 PSF, SHB 50 iterations
    (job 2228 x 2228 x 178, padded here to 2240 x 2240 x 180) against the
    reference's own output: the full I-divergence trace, every plane sum, the
    norm, 262144 sampled voxels and the relative L2 distance over the whole
    volume estimated from a 32-row sketch."""
    f = os.path.join(os.path.dirname(__file__), "golden", "config2_shb50.npz")
    if not os.path.exists(f):
        pytest.skip("config2 fixture not generated")
    from deconwolf_b200 import synthetic
    from tests.helpers import sketch, sketch_rel_l2
    d = np.load(f)
    im, psf = synthetic.config_inputs("shb-2048x2048x60")
    idx = d["sample_idx"]
    np.testing.assert_array_equal(im.reshape(-1)[idx], d["image_sample"])  # same inputs as the fixture
    assert abs(float(im.astype(np.float64).sum()) - float(d["image_sum"])) == 0
    g = dw.run_method(im, psf, method="shb", n_iter=50)
    assert g.work == (2240, 2240, 180)
    assert trace_err(g.trace, d["trace"]) < TRACE_TOL
    assert rel_l2(g.out.reshape(-1)[idx], d["sample_val"]) < OUT_TOL
    assert rel_l2(g.out.astype(np.float64).sum(axis=(1, 2)), d["plane_sums"]) < OUT_TOL
    assert abs(np.linalg.norm(g.out.astype(np.float64)) / d["norm"] - 1) < OUT_TOL
    est = sketch_rel_l2(sketch(g.out, device="cuda"), d["sketch"], float(d["norm"]))
    print(f"\nconfig 2: relative L2 to the reference over the volume (sketch) {est:.3e}, "
          f"on samples {rel_l2(g.out.reshape(-1)[idx], d['sample_val']):.3e}, "
          f"trace {trace_err(g.trace, d['trace']):.2e}")
    assert est < OUT_TOL


@pytest.mark.parametrize("name,fixture,work,method", [
    ("shb-1124x1124x60", "tile1024_shb50.npz", (1344, 1344, 180), "shb"),
    ("shb-612x562x60", "tile512_shb50.npz", (800, 750, 180), "shb"),
    ("shb-612x562x60", "tile512_rl50.npz", (800, 750, 180), "rl"),
])
def test_tile_golden(name, fixture, work, method):
    """Tiles of the 4096 x 4096 x 60 image at tile size 1024 (1124 x 1124 x
    60, job 1304 x 1304 x 178 -> 1344 x 1344 x 180) and 512 (612 x 562 x 60,
    job 792 x 742 x 178 -> 800 x 750 x 180), full 181 x 181 x 119 PSF: the
    tiled workload's transform lengths at full size, SHB 50, against the
    reference's own output."""
    f = os.path.join(os.path.dirname(__file__), "golden", fixture)
    if not os.path.exists(f):
        pytest.skip("tile fixture not generated")
    from deconwolf_b200 import synthetic
    from tests.helpers import sketch, sketch_rel_l2
    d = np.load(f)
    im, psf = synthetic.config_inputs(name)
    idx = d["sample_idx"]
    np.testing.assert_array_equal(im.reshape(-1)[idx], d["image_sample"])
    g = dw.run_method(im, psf, method=method, n_iter=50)
    assert g.work == work
    assert trace_err(g.trace, d["trace"]) < TRACE_TOL
    assert rel_l2(g.out.reshape(-1)[idx], d["sample_val"]) < OUT_TOL
    assert rel_l2(g.out.astype(np.float64).sum(axis=(1, 2)), d["plane_sums"]) < OUT_TOL
    est = sketch_rel_l2(sketch(g.out, device="cuda"), d["sketch"], float(d["norm"]))
    print(f"\n{name} {method}: relative L2 to the reference over the volume (sketch) {est:.3e}, "
          f"trace {trace_err(g.trace, d['trace']):.2e}")
    assert est < OUT_TOL


def test_deterministic():
    im, psf = case_inputs(seed=7, shape=(12, 40, 36), psf_shape=(7, 9, 9))
    a = dw.run_method(im, psf, n_iter=15)
    b = dw.run_method(im, psf, n_iter=15)
    np.testing.assert_array_equal(a.out, b.out)
    np.testing.assert_array_equal(a.trace, b.trace)


def test_graph_and_eager_agree():
    im, psf = case_inputs(seed=8, shape=(12, 40, 36), psf_shape=(7, 9, 9))
    a = dw.run_method(im, psf, n_iter=9, use_graph=True)
    b = dw.run_method(im, psf, n_iter=9, use_graph=False)
    np.testing.assert_array_equal(a.out, b.out)


def test_job_steps_equal_one_call():
    im, psf = case_inputs(seed=9, shape=(10, 30, 28), psf_shape=(5, 7, 7))
    ref = dw.run_method(im, psf, n_iter=11)
    job = dw.Job(im.shape, psf.shape, n_iter=11)
    job.setup(im, psf)
    left = 11
    while left:
        left = job.step(3)
    r = job.result()
    job.close()
    np.testing.assert_array_equal(r.out, ref.out)
    np.testing.assert_array_equal(r.trace, ref.trace)


def test_device_api_equals_host_api():
    import torch
    im, psf = case_inputs(seed=10, shape=(10, 30, 28), psf_shape=(5, 7, 7))
    ref = dw.run_method(im, psf, n_iter=7, method="rl")
    d_im = torch.from_numpy(im).cuda()
    d_psf = torch.from_numpy(psf).cuda()
    d_out = torch.empty_like(d_im)
    torch.cuda.synchronize()
    res = dw.run_method_device(d_im.data_ptr(), d_psf.data_ptr(), d_out.data_ptr(), im.shape, psf.shape,
                               n_iter=7, method="rl")
    np.testing.assert_array_equal(d_out.cpu().numpy(), ref.out)
    np.testing.assert_array_equal(res.trace, ref.trace)


def test_input_errors():
    im, psf = case_inputs()
    bad = im.copy()
    bad[1, 2, 3] = np.nan
    with pytest.raises(dw.DwcuError) as e:
        dw.run_method(bad, psf, n_iter=3)
    assert e.value.code == 5
    with pytest.raises(dw.DwcuError) as e:
        # beyond the longest supported x transform
        dw.run_method(np.full((1, 1, 5000), 50, np.float32), np.full((1, 1, 3), 1 / 3, np.float32), n_iter=3)
    assert e.value.code == 2
    with pytest.raises(dw.DwcuError) as e:
        # periodic margins need the PSF maximum at its centre
        off = psf.copy()
        off[0, 0, 0] = off.max() * 2
        dw.run_method(im[:, :, :20].copy(), off, n_iter=3, border_quality=1)
    assert e.value.code == 2
    # the context is still usable afterwards
    assert dw.run_method(im, psf, n_iter=2).iterations == 2


# ---------------------------------------------------------------- FFT

def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("shape", [(12, 20, 16), (5, 9, 14), (1, 1, 2240), (180, 6, 8), (7, 12, 384)])
def test_fft_r2c_matches_oracle(shape):
    import torch
    rng = np.random.default_rng(3)
    x = rng.random(shape).astype(np.float32)
    P, N, M = shape
    d_x = _dev(x)
    d_X = torch.empty((P, N, M // 2 + 1), dtype=torch.complex64, device="cuda")
    torch.cuda.synchronize()
    dw.fft_r2c_device(d_x.data_ptr(), shape, d_X.data_ptr())
    X = d_X.cpu().numpy()
    ref = np.fft.rfftn(x.astype(np.float64))
    assert np.max(np.abs(X - ref)) / np.max(np.abs(ref)) < 2e-6
    # c2r(r2c(x)) / n == x (fft.c:708-780: max relative error < 1e-5)
    d_y = torch.empty_like(d_x)
    dw.fft_c2r_device(d_X.data_ptr(), shape, d_y.data_ptr())
    y = d_y.cpu().numpy() / np.float32(P * N * M)
    xx = x + 5  # the reference's KAT uses values in [5, 6]
    d_x2 = _dev(xx.astype(np.float32))
    dw.fft_r2c_device(d_x2.data_ptr(), shape, d_X.data_ptr())
    dw.fft_c2r_device(d_X.data_ptr(), shape, d_y.data_ptr())
    y2 = d_y.cpu().numpy() / np.float32(P * N * M)
    assert np.max(np.abs(y2 - xx) / xx) < 1e-5
    assert np.max(np.abs(y - x)) < 1e-5


def test_fft_round_trip_on_the_reference_kat_sizes():
    """fft.c:708-780 (`fft_ut`, the reference's FFT unit test): r2c then c2r
    on sizes 51-60 x 25-34 x 20-29 with values in [5, 6], maximum relative
    error < 1e-5.  Here every such size with an even x length (the R2C
    transform's requirement): each one with supported lengths (radices up to
    16 over 2, 3, 5, 7) round trips within the bound and matches a float64
    rfftn; the others are refused with DWCU_ERROR_UNSUPPORTED."""
    import torch
    rng = np.random.default_rng(11)
    done = refused = 0
    for M in range(52, 61, 2):
        for N in range(25, 35):
            for P in range(20, 30):
                x = (5 + rng.random((P, N, M))).astype(np.float32)
                d_x = _dev(x)
                d_X = torch.empty((P, N, M // 2 + 1), dtype=torch.complex64, device="cuda")
                d_y = torch.empty_like(d_x)
                torch.cuda.synchronize()
                try:
                    dw.fft_r2c_device(d_x.data_ptr(), (P, N, M), d_X.data_ptr())
                except dw.DwcuError as e:
                    assert e.code == 2, (M, N, P)  # DWCU_ERROR_UNSUPPORTED
                    refused += 1
                    continue
                X = d_X.cpu().numpy()
                dw.fft_c2r_device(d_X.data_ptr(), (P, N, M), d_y.data_ptr())
                y = d_y.cpu().numpy() / np.float32(P * N * M)
                assert np.max(np.abs(y - x) / x) < 1e-5, (M, N, P)
                ref = np.fft.rfftn(x.astype(np.float64))
                assert np.max(np.abs(X - ref)) / np.max(np.abs(ref)) < 2e-6, (M, N, P)
                done += 1
    assert done == 90 and refused == 410


def test_conjugate_product_is_the_circular_correlation():
    """fft.c:576-628 (`fft_ut_flipall_conj`): ifft(conj(fft(X)) fft(A)) is the
    circular correlation of A with X -- the convention of the
    back-projection with the conjugated OTF -- within an MSE of 1e-5 of a
    float64 computation (relative to the values' scale)."""
    import torch
    shape = (15, 14, 12)
    P, N, M = shape
    rng = np.random.default_rng(12)
    X = rng.random(shape).astype(np.float32)
    A = rng.random(shape).astype(np.float32)
    spec = []
    for v in (X, A):
        d_v = _dev(v)
        d_S = torch.empty((P, N, M // 2 + 1), dtype=torch.complex64, device="cuda")
        torch.cuda.synchronize()
        dw.fft_r2c_device(d_v.data_ptr(), shape, d_S.data_ptr())
        spec.append(d_S)
    d_prod = (torch.conj(spec[0]) * spec[1]).contiguous()
    d_out = torch.empty(shape, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    dw.fft_c2r_device(d_prod.data_ptr(), shape, d_out.data_ptr())
    out = d_out.cpu().numpy() / np.float32(P * N * M)
    ref = np.fft.irfftn(np.conj(np.fft.rfftn(X.astype(np.float64))) * np.fft.rfftn(A.astype(np.float64)), s=shape,
                        axes=(0, 1, 2))
    # the same thing written as a correlation: sum_n X[n] A[n + k] (circular)
    k = (3, 5, 7)
    corr = float(np.sum(X.astype(np.float64) * np.roll(A.astype(np.float64), shift=[-s for s in k], axis=(0, 1, 2))))
    assert abs(ref[k] - corr) < 1e-9 * abs(corr)
    assert np.mean((out - ref) ** 2) / np.mean(ref ** 2) < 1e-5
    assert np.max(np.abs(out - ref)) / np.max(np.abs(ref)) < 1e-5


def test_block_reuse_and_release():
    """Jobs of neighbouring sizes reuse cached device blocks; results do not
    depend on which block a job got, and freeing the cache changes nothing."""
    im, psf = case_inputs(seed=8, shape=(12, 40, 44), psf_shape=(5, 7, 9))
    a = dw.run_method(im, psf, method="shb", n_iter=6)
    b = dw.run_method(im[:, :38, :42], psf, method="shb", n_iter=6)  # smaller job, may take a's block
    c = dw.run_method(im, psf, method="shb", n_iter=6)
    dw.release_cache()
    d = dw.run_method(im[:, :38, :42], psf, method="shb", n_iter=6)
    np.testing.assert_array_equal(a.out, c.out)
    np.testing.assert_array_equal(b.out, d.out)




EVEN_CASES = [
    # (image, PSF, border_quality, method): PSFs even about their centre, as
    # the Born-Wolf and Gaussian models are
    ((12, 40, 44), (7, 9, 11), 2, "shb"),
    ((12, 40, 44), (7, 9, 11), 2, "rl"),
    ((9, 22, 20), (5, 7, 9), 1, "shb"),     # periodic margins in x and y
    ((20, 33, 44), (21, 15, 13), 0, "shb"),
    ((1, 64, 60), (1, 9, 9), 2, "shb"),     # a single plane
]


@pytest.mark.parametrize("shape,psf_shape,bq,method", EVEN_CASES)
def test_even_psf(shape, psf_shape, bq, method):
    """Exactly even PSFs (unjittered Gaussians): results as the reference's."""
    psf = gauss_psf(psf_shape, (1.3, 1.6, 1.9))
    assert np.array_equal(psf, psf[::-1, ::-1, ::-1])
    im = poisson_image(shape, psf, seed=11, bg=40.0, npts=12)
    g = dw.run_method(im, psf, border_quality=bq, method=method, n_iter=8)
    r = po.deconvolve(im, psf, border_quality=bq, method=method, n_iter=8, impl=checker())
    assert rel_l2(g.out, r.out) < OUT_TOL
    assert trace_err(g.trace, r.trace) < TRACE_TOL
