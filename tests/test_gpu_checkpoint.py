"""Checkpoints of a job between iterations (dwcu_job_snapshot /
dwcu_job_restore): a job stopped after k iterations, its state copied to
the host and the job destroyed, then continued in a new job set up with the
same inputs, ends with the uninterrupted job's result.  With the autotuner
off every x pass uses one plan, and the recomputed spectrum equals the one
the fused update pass would have written, so the results are equal bit for
bit."""
import numpy as np
import pytest

import deconwolf_b200 as dw
from oracle import pyoracle as po
from tests.helpers import gauss_psf, poisson_image

pytestmark = pytest.mark.gpu


@pytest.fixture
def heuristic_plans():
    dw.tune_set_mode(dw.TUNE_OFF)
    dw.tune_clear()
    yield
    dw.tune_set_mode(dw.TUNE_MEASURE)
    dw.tune_clear()


def _inputs():
    psf = gauss_psf((7, 9, 11), (1.3, 1.6, 1.9), seed=61, jitter=0.2)
    im = poisson_image((12, 40, 44), psf, seed=61, bg=60.0, npts=20)
    return im, psf


def _job(im, psf, **kw):
    j = dw.Job(im.shape, psf.shape, **kw)
    j.setup(im, psf)
    return j


CASES = [
    dict(method="shb", n_iter=20),
    dict(method="rl", n_iter=20),
    dict(method="shb", n_iter=15, border_quality=1),
    dict(method="shb", iter_type=po.ITER_REL, err_rel=0.002, maxiter=60),
    dict(method="rl", iter_type=po.ITER_REL, err_rel=0.002, maxiter=60),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}={v}" for k, v in c.items()))
@pytest.mark.parametrize("stop_after", [0, 1, 7])
def test_resumed_job_ends_like_the_uninterrupted_one(case, stop_after, heuristic_plans):
    im, psf = _inputs()
    a = _job(im, psf, **case)
    a.step(1 << 30)
    ref = a.result()
    a.close()

    b = _job(im, psf, **case)
    if stop_after:
        b.step(stop_after)
    snap = b.snapshot()
    b.close()
    assert snap["done_iters"] == stop_after and snap["next_iter"] == stop_after
    assert (snap["x_prev"] is not None) == (case["method"] == "shb")

    c = _job(im, psf, **case)
    c.restore(snap)
    c.step(1 << 30)
    res = c.result()
    c.close()
    assert res.iterations == ref.iterations
    np.testing.assert_array_equal(res.trace, ref.trace)
    np.testing.assert_array_equal(res.out, ref.out)


def test_a_finished_job_restores_to_its_result():
    im, psf = _inputs()
    a = _job(im, psf, method="shb", n_iter=9)
    a.step(1 << 30)
    snap = a.snapshot()
    ref = a.result()
    a.close()
    assert snap["next_iter"] == -1 and snap["done_iters"] == 9
    c = _job(im, psf, method="shb", n_iter=9)
    c.restore(snap)
    assert c.done()
    res = c.result()
    np.testing.assert_array_equal(res.out, ref.out)
    np.testing.assert_array_equal(res.trace, ref.trace)


def test_a_snapshot_of_another_job_is_refused():
    im, psf = _inputs()
    a = _job(im, psf, method="shb", n_iter=6)
    a.step(3)
    snap = a.snapshot()
    a.close()
    other = _job(im[:, :30, :30].copy(), psf, method="shb", n_iter=6)
    with pytest.raises(dw.DwcuError):
        other.restore(snap)                       # another job size
    other.close()
    c = _job(im * 2.0, psf, method="shb", n_iter=6)
    with pytest.raises(dw.DwcuError):
        c.restore(snap)                           # another background (another image)
    c.close()
