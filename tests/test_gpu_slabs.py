"""One image split over several GPUs by z planes (dwcu_deconvolve_slabs),
with every part on one GPU (the parts, their exchanges and the ordering
between them run as they would on several GPUs; only the data stays in one
GPU's memory).  Both forms of the z pass's exchange run: in place through
the plane table (the default where the GPUs have peer access) and on
gathered copies (DWCU_SLAB_TRANSPOSE=copy, the form for GPUs without).

* One part runs the whole job's kernels on the same data: equal to
  dwcu_deconvolve bit for bit.
* With n parts the kernels see the same values; only the sums combined
  across parts (image sum, I-divergence) are added in another order, so the
  result stays within SPLIT_TOL of the whole job and the error trace within
  SPLIT_TRACE_TOL, and within the parity tolerances of the oracle.
"""
import numpy as np
import pytest

import deconwolf_b200 as dw
from oracle import pyoracle as po
from tests.helpers import gauss_psf, poisson_image, rel_l2

pytestmark = pytest.mark.gpu

OUT_TOL = 1e-4
TRACE_TOL = 1e-5
SPLIT_TOL = 1e-5
SPLIT_TRACE_TOL = 1e-6

ERROR_UNSUPPORTED = 2


@pytest.fixture(params=["direct", "copy"])
def transpose(request, monkeypatch):
    if request.param == "copy":
        monkeypatch.setenv("DWCU_SLAB_TRANSPOSE", "copy")
    else:
        monkeypatch.delenv("DWCU_SLAB_TRANSPOSE", raising=False)
    return request.param


def _inputs(shape=(9, 22, 19), psf_shape=(5, 7, 9), seed=7):
    psf = gauss_psf(psf_shape, (1.2, 1.5, 1.7), seed=seed, jitter=0.2)
    im = poisson_image(shape, psf, seed=seed, bg=50.0, npts=15)
    return im, psf


def _trace_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.abs(b)))


@pytest.mark.parametrize("method", ["shb", "rl"])
def test_one_part_equals_the_whole_job(method, transpose):
    im, psf = _inputs()
    a = dw.run_method(im, psf, method=method, n_iter=12)
    b = dw.run_slabs(im, psf, parts=1, method=method, n_iter=12)
    np.testing.assert_array_equal(b.out, a.out)
    np.testing.assert_array_equal(b.trace, a.trace)
    assert b.bg == a.bg and b.work == a.work


CASES = [
    (dict(method="shb", n_iter=12), (9, 22, 19), (5, 7, 9)),
    (dict(method="rl", n_iter=12), (9, 22, 19), (5, 7, 9)),
    (dict(method="shb", n_iter=20), (20, 64, 70), (9, 11, 13)),
    (dict(method="rl", n_iter=15), (20, 64, 70), (9, 11, 13)),
    (dict(method="shb", iter_type=po.ITER_REL, err_rel=0.002), (9, 22, 19), (5, 7, 9)),
    (dict(method="shb", iter_type=po.ITER_ABS, err_abs=1.5, maxiter=30), (9, 22, 19), (5, 7, 9)),
    (dict(method="shb", n_iter=8, start=po.START_IDENTITY), (9, 22, 19), (5, 7, 9)),
    (dict(method="rl", n_iter=8, metric=po.METRIC_MSE), (9, 22, 19), (5, 7, 9)),
    (dict(method="shb", n_iter=10, border_quality=1), (9, 20, 19), (5, 7, 9)),
    (dict(method="rl", n_iter=10, border_quality=0), (10, 24, 20), (5, 7, 9)),
    (dict(method="shb", n_iter=8, bg=3.0, positivity=False), (9, 22, 19), (5, 7, 9)),
    (dict(method="shb", n_iter=7, start=po.START_LP), (9, 22, 19), (5, 7, 9)),
    (dict(method="rl", n_iter=7, start=po.START_LP), (20, 64, 70), (9, 11, 13)),
    # periodic margins along y (job 24 x 32 x 12), along x (30 x 24 x 12), both (bq 0, 30 x 32 x 10)
    (dict(method="shb", n_iter=10, border_quality=1), (9, 22, 19), (5, 7, 9)),
    (dict(method="rl", n_iter=10, border_quality=1), (9, 20, 17), (5, 7, 9)),
    (dict(method="shb", n_iter=10, border_quality=0), (10, 26, 22), (5, 7, 9)),
]


def _id(v):
    if isinstance(v, dict):
        return "-".join(f"{k}={x}" for k, x in v.items())
    return "x".join(map(str, v))


@pytest.mark.parametrize("parts", [2, 3, 5])
@pytest.mark.parametrize("case,shape,psf_shape", CASES, ids=_id)
def test_parts_match_the_whole_job(case, shape, psf_shape, parts, transpose):
    im, psf = _inputs(shape, psf_shape)
    a = dw.run_method(im, psf, **case)
    b = dw.run_slabs(im, psf, parts=parts, **case)
    assert b.iterations == a.iterations and b.work == a.work
    assert rel_l2(b.out, a.out) < SPLIT_TOL
    assert _trace_err(b.trace, a.trace) < SPLIT_TRACE_TOL


def test_parts_without_image_planes(transpose):
    # 3 image planes, a 7-plane job: parts 3..6 hold no image plane
    im, psf = _inputs((3, 30, 31), (5, 7, 9))
    assert dw.plan_size(im.shape, psf.shape)[0][2] == 7
    for method in ("shb", "rl"):
        a = dw.run_method(im, psf, method=method, n_iter=10)
        b = dw.run_slabs(im, psf, parts=7, method=method, n_iter=10)
        assert rel_l2(b.out, a.out) < SPLIT_TOL
        assert _trace_err(b.trace, a.trace) < SPLIT_TRACE_TOL


@pytest.mark.parametrize("method", ["shb", "rl"])
def test_parts_match_the_oracle(method, transpose):
    im, psf = _inputs((20, 64, 70), (9, 11, 13))
    impl = "reference" if po.available("reference") else "port"
    r = po.deconvolve(im, psf, impl=impl, method=method, n_iter=20)
    g = dw.run_slabs(im, psf, parts=4, method=method, n_iter=20)
    assert g.iterations == r.iterations
    assert rel_l2(g.out, r.out) < OUT_TOL
    assert _trace_err(g.trace, r.trace) < TRACE_TOL


def test_unsupported_splits_are_refused():
    # periodic margins along z (job z size 13 at bq 1: transformed at 20)
    im, psf = _inputs((9, 22, 19), (7, 7, 9))
    assert dw.plan_size(im.shape, psf.shape, border_quality=1)[0][2] == 20
    with pytest.raises(dw.DwcuError) as e:
        dw.run_slabs(im, psf, parts=2, method="shb", n_iter=4, border_quality=1)
    assert e.value.code == ERROR_UNSUPPORTED
    im, psf = _inputs()
    Z = dw.plan_size(im.shape, psf.shape)[0][2]
    with pytest.raises(dw.DwcuError) as e:
        dw.run_slabs(im, psf, parts=Z + 1, method="shb", n_iter=4)
    assert e.value.code == ERROR_UNSUPPORTED
    # the library carries on
    assert dw.run_slabs(im, psf, parts=2, method="shb", n_iter=4).iterations == 4
