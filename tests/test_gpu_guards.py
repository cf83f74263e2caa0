"""Guard bands around every buffer of a job's device block (the library's
debugging aid in place of a memory checker, which is not available on the
GPU machines): every kind of job runs with 4 KB of a fixed pattern before
and after each of its buffers, and no band may change -- no kernel writes
outside the buffer it was given.  The results equal those of the same jobs
without guards, bit for bit.  A positive control (a band overwritten by the
host) shows that the check finds a change."""
import numpy as np
import pytest

import deconwolf_b200 as dw
from tests.helpers import gauss_psf, poisson_image

pytestmark = pytest.mark.gpu


def _violations():
    return int(dw.lib().dwcu_debug_guard_violations())


def _inputs(shape, psf_shape, seed):
    psf = gauss_psf(psf_shape, (1.2, 1.5, 1.7), seed=seed, jitter=0.2)
    return poisson_image(shape, psf, seed=seed, bg=50.0, npts=15), psf


@pytest.fixture
def guarded():
    dw.release_cache()
    assert dw.lib().dwcu_debug_guards(1) == 0
    yield
    dw.lib().dwcu_debug_guards(0)
    dw.release_cache()


def test_the_check_finds_a_changed_band(guarded):
    im, psf = _inputs((9, 22, 19), (5, 7, 9), 51)
    v0 = _violations()
    dw.lib().dwcu_debug_guards(2)
    dw.run_method(im, psf, n_iter=3)
    assert _violations() == v0 + 1
    dw.lib().dwcu_debug_guards(1)
    dw.run_method(im, psf, n_iter=3)
    assert _violations() == v0 + 1


JOBS = [
    ((9, 22, 19), (5, 7, 9), dict(method="shb", n_iter=8)),
    ((9, 22, 19), (5, 7, 9), dict(method="rl", n_iter=8)),
    ((9, 22, 19), (5, 7, 9), dict(method="shb", iter_type=dw.ITER_REL, err_rel=0.01)),
    ((9, 22, 19), (5, 7, 9), dict(method="shb", n_iter=5, start=dw.START_LP)),
    ((9, 22, 19), (5, 7, 9), dict(method="rl", n_iter=5, metric=dw.METRIC_MSE)),
    ((9, 22, 20), (5, 7, 9), dict(method="shb", n_iter=6, border_quality=1)),     # periodic x and y
    ((37, 40, 30), (11, 9, 9), dict(method="rl", n_iter=6, border_quality=0)),    # periodic z
    ((12, 26, 31), (7, 9, 11), dict(method="shb", n_iter=6, border_quality=1)),   # every axis periodic
    ((1, 30, 26), (1, 7, 9), dict(method="shb", n_iter=6)),                       # a single plane
    ((5, 40, 3), (5, 9, 3), dict(method="rl", n_iter=6)),                         # thin x
    ((12, 70, 200), (7, 9, 11), dict(method="shb", n_iter=6)),                    # x alternates, R = 1 update
    ((20, 256, 300), (39, 41, 41), dict(method="shb", n_iter=4)),                 # larger transforms
]


def test_no_job_writes_outside_its_buffers():
    plain = []
    for shape, psf_shape, kw in JOBS:
        im, psf = _inputs(shape, psf_shape, 52)
        plain.append(dw.run_method(im, psf, **kw))
    dw.release_cache()
    dw.lib().dwcu_debug_guards(1)
    try:
        v0 = _violations()
        for (shape, psf_shape, kw), ref in zip(JOBS, plain):
            im, psf = _inputs(shape, psf_shape, 52)
            g = dw.run_method(im, psf, **kw)
            np.testing.assert_array_equal(g.out, ref.out)
            np.testing.assert_array_equal(g.trace, ref.trace)
        # tiles, a batch, the server and a split job
        im, psf = _inputs((8, 70, 64), (7, 9, 9), 53)
        pp = dw.psf_prepare(psf, im.shape)
        dw.deconvolve_tiled(im, pp, 30, 6, method="shb", n_iter=6)
        jobs = []
        for n_iter in (4, 7):
            j = dw.Job(im.shape, psf.shape, method="rl", n_iter=n_iter)
            j.setup(im, psf)
            jobs.append(j)
        dw.batch_run(jobs)
        for j in jobs:
            j.result()
            j.close()
        sv = dw.Server(hbm_budget=0.0, max_active=2, iters_per_turn=3)
        ids = [sv.submit(im, psf, method=m, n_iter=5) for m in ("shb", "rl", "shb")]
        for i in ids:
            sv.wait(i)
        sv.close()
        # one image split into parts (including parts without image planes)
        for parts in (3, 7):
            dw.run_slabs(im, psf, parts=parts, method="shb", n_iter=5)
        dw.run_slabs(im, psf, parts=4, method="rl", n_iter=5)
        assert _violations() == v0
    finally:
        dw.lib().dwcu_debug_guards(0)
        dw.release_cache()
