"""The FP64 error reference (oracle/fp64.py) against the reference build.

The FP64 restatement runs deconwolf's SHB / RL iteration with every value in
float64.  The reference's own float32 result must sit within float32
rounding of it: relative L2 of the output <= 2e-5 and every I-divergence
value within 1e-5 relative.  These bounds pin the restatement (a wrong step
would move the outputs by far more than rounding) and give the scale
against which the GPU's distance to FP64 is judged in the GPU tests.
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from oracle.fp64 import deconvolve_fp64, deconvolve_fp64_torch, job_size
from tests.helpers import gauss_psf, poisson_image, rel_l2, sketch, sketch_rel_l2

pytestmark = pytest.mark.skipif(not po.available("port"), reason="oracle not built (make -C oracle)")

FP64_OUT_TOL = 2e-5
FP64_TRACE_TOL = 1e-5


def _impl():
    return "reference" if po.available("reference") else "port"


def _inputs(seed, shape, psf_shape):
    psf = gauss_psf(psf_shape, (1.2, 1.5, 1.7), seed=seed, jitter=0.2)
    return poisson_image(shape, psf, seed=seed, bg=50.0, npts=15), psf


CASES = [
    dict(method="shb", n_iter=20),
    dict(method="rl", n_iter=20),
    dict(method="shb", n_iter=10, border_quality=1),
    dict(method="rl", n_iter=10, border_quality=0),
    dict(method="shb", n_iter=8, start=po.START_IDENTITY),
    dict(method="shb", n_iter=8, bg=3.0, positivity=False),
    dict(method="shb", n_iter=8, alphamax=0.3),
    dict(method="rl", n_iter=6, bg=0.5),
]


def _fp64_kw(case):
    kw = dict(method=case["method"], n_iter=case["n_iter"], bq=case.get("border_quality", 2))
    if "bg" in case:
        kw["bg"] = case["bg"]
    if "positivity" in case:
        kw["positivity"] = bool(case["positivity"])
    if "alphamax" in case:
        kw["alphamax"] = case["alphamax"]
    if case.get("start") == po.START_IDENTITY:
        kw["start"] = "identity"
    return kw


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}={v}" for k, v in c.items()))
def test_reference_within_rounding_of_fp64(case):
    im, psf = _inputs(3, (9, 22, 19), (5, 7, 9))
    r = po.deconvolve(im, psf, impl=_impl(), **case)
    f = deconvolve_fp64(im, psf, **_fp64_kw(case))
    assert r.iterations == case["n_iter"]
    assert abs(r.bg - f.bg) <= 1e-6 * max(1.0, f.bg)
    assert rel_l2(r.out, f.out) < FP64_OUT_TOL
    assert np.max(np.abs(r.trace - f.trace) / np.abs(f.trace)) < FP64_TRACE_TOL


def test_job_size_rule():
    # method_shb.c:137-153
    assert job_size((40, 256, 256), (79, 127, 127), 2) == (118, 382, 382)
    assert job_size((40, 256, 256), (79, 127, 127), 1) == (80, 320, 320)
    assert job_size((40, 256, 256), (79, 127, 127), 0) == (79, 256, 256)


def test_identity_and_first_iteration():
    im, psf = _inputs(4, (6, 17, 15), (3, 5, 5))
    np.testing.assert_array_equal(deconvolve_fp64(im, psf, n_iter=0).out, im.astype(np.float64))
    # one SHB iteration returns the flat start: sum(g) / job voxels
    f = deconvolve_fp64(im, psf, method="shb", n_iter=1)
    w = job_size(im.shape, psf.shape, 2)
    assert np.allclose(f.out, im.astype(np.float64).sum() / np.prod(w), rtol=0, atol=1e-12)


def test_sketch_estimates_relative_l2():
    rng = np.random.default_rng(5)
    b = (rng.random(200000) * 1000).astype(np.float32)
    for d in (rng.normal(size=b.size), np.ones(b.size), np.linspace(-1, 1, b.size)):
        a = b.astype(np.float64) + 1e-3 * d
        true = rel_l2(a, b)
        est = sketch_rel_l2(sketch(a), sketch(b), float(np.linalg.norm(b.astype(np.float64))))
        assert 0.6 < est / true < 1.5
    # exact zero distance
    assert sketch_rel_l2(sketch(b), sketch(b.copy()), 1.0) == 0.0


@pytest.mark.parametrize("method,bq", [("shb", 2), ("rl", 2), ("shb", 1), ("rl", 0)])
def test_torch_twin_equals_numpy(method, bq):
    """The torch form (used on the GPU for volumes too large for host memory
    in float64) takes the same steps: equal to rounding in float64."""
    im, psf = _inputs(3, (9, 22, 19), (5, 7, 9))
    a = deconvolve_fp64(im, psf, method=method, n_iter=15, bq=bq)
    b = deconvolve_fp64_torch(im, psf, method=method, n_iter=15, bq=bq)
    assert np.max(np.abs(a.out - b.out)) <= 1e-12 * np.max(np.abs(a.out))
    assert np.max(np.abs(a.trace - b.trace) / a.trace) < 1e-12
