"""The autotuner on the GPU: every candidate plan of a job's transform lengths
gives the oracle's result within the parity tolerances, and a measured
choice is recorded with its candidate times."""
import numpy as np
import pytest

import deconwolf_b200 as dw
from oracle import pyoracle as po
from tests.helpers import gauss_psf, poisson_image, rel_l2

pytestmark = pytest.mark.gpu

OUT_TOL = 1e-4
TRACE_TOL = 1e-5


def _case():
    psf = gauss_psf((7, 9, 11), (1.3, 1.6, 1.9), seed=31, jitter=0.2)
    im = poisson_image((12, 70, 200), psf, seed=31, bg=60.0, npts=20)
    return im, psf


def _lengths(work):
    X, Y, Z = work
    return [(dw.PLAN_X, X // 2), (dw.PLAN_Y, Y), (dw.PLAN_LINES, Y), (dw.PLAN_LINES, Z)]


@pytest.mark.parametrize("method", ["shb", "rl"])
def test_every_candidate_matches_the_oracle(method):
    im, psf = _case()
    work = dw.plan_size(im.shape, psf.shape)[0]
    ref = po.deconvolve(im, psf, method=method, n_iter=10, work=work)
    tried = 0
    try:
        for kind, n in _lengths(work):
            plans = dw.tune_plans(kind, n)
            for c in range(len(plans)):
                dw.tune_force(kind, n, c)
                g = dw.run_method(im, psf, method=method, n_iter=10)
                assert g.work == work
                assert rel_l2(g.out, ref.out) < OUT_TOL, (kind, n, c, plans[c])
                assert np.max(np.abs(g.trace - ref.trace) / ref.trace) < TRACE_TOL, (kind, n, c)
                tried += 1
            dw.tune_force(kind, n, -1)
    finally:
        dw.tune_clear()
    assert tried >= 6


def test_measured_choice_is_recorded():
    im, psf = _case()
    work = dw.plan_size(im.shape, psf.shape)[0]
    dw.tune_clear()
    dw.tune_set_mode(dw.TUNE_MEASURE)
    try:
        g = dw.run_method(im, psf, method="shb", n_iter=5)
        X, Y, Z = work
        for kind, n in ((dw.PLAN_X, X // 2), (dw.PLAN_Y, Y), (dw.PLAN_LINES, Z)):
            cnt = len(dw.tune_plans(kind, n))
            cand, ms = dw.tune_query(kind, n)
            if cnt > 1:
                assert 0 <= cand < cnt and len(ms) == cnt and all(t > 0 for t in ms), (kind, n, cand, ms)
                assert cand == dw.tune_select(ms)
        # the tuned plans give the heuristic plans' result within the tolerance
        dw.tune_set_mode(dw.TUNE_OFF)
        dw.tune_clear()
        h = dw.run_method(im, psf, method="shb", n_iter=5)
        assert rel_l2(g.out, h.out) < OUT_TOL
    finally:
        dw.tune_set_mode(dw.TUNE_MEASURE)
        dw.tune_clear()


def test_workload_lengths_are_tuned():
    """Times every candidate of the transform lengths of the 2048 x 2048 x 60
    job (x 1120, y 2240, z 180) and of the tiles of the 4096 x 4096 x 60 image
    (1260, 1344; 750, 800 at tile size 512) and prints the table."""
    rows = []
    try:
        for kind, n in ((dw.PLAN_X, 1120), (dw.PLAN_Y, 2240), (dw.PLAN_LINES, 180), (dw.PLAN_X, 630),
                        (dw.PLAN_X, 672), (dw.PLAN_Y, 1260), (dw.PLAN_Y, 1344), (dw.PLAN_X, 375),
                        (dw.PLAN_X, 400), (dw.PLAN_Y, 750), (dw.PLAN_Y, 800)):
            dw.tune_run(kind, n)
            cand, ms = dw.tune_query(kind, n)
            plans = dw.tune_plans(kind, n)
            assert 0 <= cand < len(plans) and len(ms) == len(plans)
            rows.append((["lines", "y", "x"][kind], n, cand, plans, ms))
    finally:
        dw.tune_clear()
    print()
    for kind, n, cand, plans, ms in rows:
        print(f"tune {kind} {n}: chose {cand} " + "  ".join(f"{p[0]}/{p[1]}:{t:.4f}ms" for p, t in zip(plans, ms)))
