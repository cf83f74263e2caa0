"""The autotuner's host logic (CPU): the selection rule on given candidate
times, the candidate table, and the plan-table file round trip (the
analogue of FFTW wisdom files, src/fft.c:299-316, 355)."""
import math

import pytest

import deconwolf_b200 as dw


def test_select_keeps_the_heuristic_plan_within_the_margin():
    assert dw.tune_select([1.00, 0.99, 1.20]) == 0       # 1 % faster: noise
    assert dw.tune_select([1.00, 0.97, 1.20]) == 1       # 3 % faster: taken
    assert dw.tune_select([1.00, 0.97, 0.90]) == 2       # the fastest
    assert dw.tune_select([1.00, 0.97, 0.90], margin=0.15) == 0
    assert dw.tune_select([2.0]) == 0


def test_select_skips_candidates_that_did_not_run():
    assert dw.tune_select([math.inf, 1.0, 2.0]) == 1     # candidate 0 failed: the fastest that ran
    assert dw.tune_select([1.0, -1.0, math.nan]) == 0
    assert dw.tune_select([-1.0, -1.0]) == 0


def test_candidates_of_the_workload_lengths():
    # candidate 0 is the generator's heuristic choice; the line pass also has
    # a narrower column tile; the x pass an alternate radix list
    for n in (180, 1120, 2240, 1260, 1344, 750, 800):
        plans = dw.tune_plans(dw.PLAN_LINES, n)
        assert len(plans) >= 2
        for rad, tile in plans:
            assert math.prod(rad) == n and all(r <= 16 for r in rad)
        assert plans[-1][0] == plans[0][0] and plans[-1][1] == plans[0][1] // 2
    for n in (1120, 630, 672, 375, 400):
        plans = dw.tune_plans(dw.PLAN_X, n)
        assert len(plans) == 2 and plans[0][1] == plans[1][1]   # same rows per tile
        assert plans[0][0] != plans[1][0] and math.prod(plans[1][0]) == n
    assert dw.tune_plans(dw.PLAN_Y, 2240)[0][0] == (16, 10, 14)
    assert dw.tune_plans(dw.PLAN_X, 11) == []                    # 11 has a prime factor > 7
    with pytest.raises(dw.DwcuError):
        dw.tune_force(dw.PLAN_X, 1120, 5)                      # no such candidate


def test_force_query_export_import_round_trip(tmp_path):
    dw.tune_clear()
    try:
        assert dw.tune_query(dw.PLAN_LINES, 180) == (-1, [])
        dw.tune_force(dw.PLAN_LINES, 180, 2)
        dw.tune_force(dw.PLAN_X, 1120, 1)
        assert dw.tune_query(dw.PLAN_LINES, 180)[0] == 2
        f = tmp_path / "plans.txt"
        dw.tune_export(str(f))
        text = f.read_text()
        assert "lines 180 2" in text and "x 1120 1" in text
        dw.tune_clear()
        assert dw.tune_query(dw.PLAN_X, 1120)[0] == -1
        dw.tune_import(str(f))
        assert dw.tune_query(dw.PLAN_LINES, 180)[0] == 2 and dw.tune_query(dw.PLAN_X, 1120)[0] == 1
        # forgetting a length
        dw.tune_force(dw.PLAN_LINES, 180, -1)
        assert dw.tune_query(dw.PLAN_LINES, 180)[0] == -1
        # a file naming a plan the library does not have is refused as a whole
        bad = tmp_path / "bad.txt"
        bad.write_text("lines 120 1\nx 1120 7\n")
        with pytest.raises(dw.DwcuError):
            dw.tune_import(str(bad))
        assert dw.tune_query(dw.PLAN_LINES, 120)[0] == -1
        with pytest.raises(dw.DwcuError):
            dw.tune_import(str(tmp_path / "missing.txt"))
    finally:
        dw.tune_clear()


def test_mode_switch():
    dw.tune_set_mode(dw.TUNE_OFF)
    try:
        m = dw.ctypes.c_int32()
        assert dw.lib().dwcu_tune_get_mode(dw.ctypes.byref(m)) == 0 and m.value == dw.TUNE_OFF
    finally:
        dw.tune_set_mode(dw.TUNE_MEASURE)
    with pytest.raises(dw.DwcuError):
        dw.tune_set_mode(7)
