"""The request server (dwcu_server_*): results of requests served together
equal dwcu_deconvolve on the same inputs, bit for bit; cancellation,
failing requests and a tight memory budget leave the other requests intact."""
import numpy as np
import pytest

import deconwolf_b200 as dw
from tests.helpers import gauss_psf, poisson_image

pytestmark = pytest.mark.gpu

CASES = [
    ((9, 22, 19), (5, 7, 9), dict(method="shb", n_iter=12)),
    ((6, 40, 31), (3, 5, 5), dict(method="rl", n_iter=7)),
    ((12, 30, 44), (7, 7, 7), dict(method="shb", iter_type=dw.ITER_REL, err_rel=0.002, maxiter=30)),
    ((1, 30, 26), (1, 7, 9), dict(method="shb", n_iter=20)),
    ((10, 64, 60), (9, 11, 11), dict(method="shb", n_iter=23)),
    ((7, 33, 35), (5, 9, 7), dict(method="rl", n_iter=3)),
]


def _inputs(k, shape, pshape):
    psf = gauss_psf(pshape, (1.2, 1.5, 1.7), seed=k, jitter=0.2)
    im = poisson_image(shape, psf, seed=k, bg=40.0, npts=12)
    return im, psf


@pytest.mark.parametrize("iters_per_turn", [1, 4])
def test_served_results_equal_alone(iters_per_turn):
    inputs = [_inputs(k, s, p) for k, (s, p, _) in enumerate(CASES)]
    refs = [dw.run_method(im, psf, **kw) for (im, psf), (_, _, kw) in zip(inputs, CASES)]
    sv = dw.Server(max_active=4, iters_per_turn=iters_per_turn)
    ids = [sv.submit(im, psf, **kw) for (im, psf), (_, _, kw) in zip(inputs, CASES)]
    for rid, ref in zip(ids, refs):
        r = sv.wait(rid, timeout=120)
        assert r.iterations == ref.iterations
        np.testing.assert_array_equal(r.out, ref.out)
        np.testing.assert_array_equal(r.trace, ref.trace)
    st = sv.stats()
    sv.close()
    assert st["completed"] == len(CASES) and st["failed"] == 0
    assert 0 < st["latency_p50_s"] <= st["latency_p99_s"]
    assert st["voxel_iterations"] == sum(np.prod(s) * r.iterations for (s, _, _), r in zip(CASES, refs))


def test_cancel_and_failure_leave_others_intact():
    im, psf = _inputs(1, (10, 64, 60), (9, 11, 11))
    ref = dw.run_method(im, psf, n_iter=15)
    bad = im.copy()
    bad[2, 3, 4] = np.nan
    sv = dw.Server(max_active=2, iters_per_turn=2)
    a = sv.submit(im, psf, n_iter=400)   # cancelled while it runs
    b = sv.submit(bad, psf, n_iter=5)    # rejected at setup
    c = sv.submit(im, psf, n_iter=15)
    d = sv.submit(im, psf, n_iter=15)    # cancelled while queued or running
    sv.cancel(a)
    sv.cancel(d)
    with pytest.raises(dw.DwcuError) as e:
        sv.wait(a, timeout=120)
    assert e.value.code == 7
    with pytest.raises(dw.DwcuError) as e:
        sv.wait(b, timeout=120)
    assert e.value.code == 5
    r = sv.wait(c, timeout=120)
    np.testing.assert_array_equal(r.out, ref.out)
    with pytest.raises(dw.DwcuError) as e:
        sv.wait(d, timeout=120)
    assert e.value.code == 7
    st = sv.stats()
    sv.close()
    assert st["completed"] == 1 and st["failed"] == 1 and st["cancelled"] == 2
    assert st["active"] == 0 and st["device_bytes_in_use"] == 0


def test_tight_budget_runs_one_at_a_time():
    inputs = [_inputs(k, (8, 40, 36), (5, 7, 7)) for k in range(3)]
    refs = [dw.run_method(im, psf, n_iter=6) for im, psf in inputs]
    sv = dw.Server(hbm_budget=1.0, max_active=8)  # every job exceeds the budget: admitted only when idle
    ids = [sv.submit(im, psf, n_iter=6) for im, psf in inputs]
    for rid, ref in zip(ids, refs):
        np.testing.assert_array_equal(sv.wait(rid, timeout=120).out, ref.out)
    sv.close()
