"""CPU tests of the C ABI: the library loads, exports every declared entry
point, plans job sizes, and fails loudly (no CPU fallback) without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import deconwolf_b200 as dw

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "dwcu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dwcu_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = dw.lib()
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/dwcu.h but not exported"
    assert sorted(dw.EXPORTS) == names


def test_abi_version():
    assert dw.lib().dwcu_abi_version() == 1


def test_opts_defaults_match_dw_opts_new():
    o = dw.Opts()
    dw.lib().dwcu_opts_init(ctypes.byref(o))
    # dw.c:340-413
    assert o.method == dw.METHOD_SHB and o.iter_type == dw.ITER_REL and o.maxiter == 250
    assert abs(o.err_rel - 0.02) < 1e-9 and o.bg_auto == 1 and o.positivity == 1
    assert o.border_quality == 2 and o.start_condition == dw.START_FLAT and o.metric == dw.METRIC_IDIV
    assert o.alphamax == 1.0 and o.n_iter == 1


def test_plan_sizes_of_the_workloads():
    # 256x256x40 with a 127x127x79 PSF: job 382x382x118 -> 384x384x120
    assert dw.plan_size((40, 256, 256), (79, 127, 127))[0] == (384, 384, 120)
    # 2048x2048x60 with a 181x181x119 PSF: job 2228x2228x178 -> 2240x2240x180
    work, nbytes = dw.plan_size((60, 2048, 2048), (119, 181, 181))
    assert work == (2240, 2240, 180)
    assert 15e9 < nbytes < 25e9


def test_exact_sizes_for_bq_0_and_1():
    # bq 1/0 wrap around inside the job: exact sizes where supported,
    # 256 + 64 = 320 (x, 160 = 16*10), 256 + 64 = 320, 40 + 40 = 80
    assert dw.plan_size((40, 256, 256), (79, 127, 127), border_quality=1)[0] == (320, 320, 80)
    # bq 0: max(M, pM): z period 13 is prime -> periodic z at the next
    # supported length >= 13 + 2*2
    assert dw.plan_size((13, 64, 64), (5, 5, 5), border_quality=0)[0] == (64, 64, 18)


def test_bq1_exact_supported_size():
    # M + (pM+1)/2 = 60 + 4 = 64 (x), 50 + 4 = 54, 20 + 4 = 24: all supported and exact
    work, _ = dw.plan_size((20, 50, 60), (7, 7, 7), border_quality=1)
    assert work == (64, 54, 24)
    # 61 + 4 = 65 is odd: x is transformed at a length >= 65 + 2*3 with
    # periodic margins (72); y and z stay exact
    work, _ = dw.plan_size((20, 50, 61), (7, 7, 7), border_quality=1)
    assert work == (72, 54, 24)
    # bq 0 with a prime z period: 37 + 2*5 -> the next supported length
    work, _ = dw.plan_size((37, 40, 30), (11, 9, 9), border_quality=0)
    assert work[:2] == (30, 40) and work[2] >= 37 + 2 * 5
    with pytest.raises(dw.DwcuError) as e:
        dw.plan_size((1, 1, 5000), (1, 1, 3))  # beyond the longest x transform
    assert e.value.code == 2


def test_invalid_options_rejected():
    with pytest.raises(dw.DwcuError) as e:
        dw.plan_size((0, 5, 5), (3, 3, 3))
    assert e.value.code == 1


@pytest.mark.skipif(dw.lib().dwcu_device_count() > 0, reason="a GPU is present")
def test_no_gpu_no_fallback():
    """Without a device every compute call fails with DWCU_ERROR_CUDA."""
    im = np.ones((4, 8, 8), np.float32) * 100
    psf = np.ones((3, 3, 3), np.float32) / 27
    with pytest.raises(dw.DwcuError) as e:
        dw.run_method(im, psf, n_iter=3)
    assert e.value.code == 4
    assert "no CUDA device" in str(e.value)


@pytest.mark.skipif(dw.lib().dwcu_device_count() > 0, reason="a GPU is present")
def test_no_gpu_server_and_tiles_fail():
    with pytest.raises(dw.DwcuError) as e:
        dw.Server()
    assert e.value.code == 4
    im = np.ones((4, 40, 40), np.float32) * 100
    psf = np.ones((3, 3, 3), np.float32) / 27
    with pytest.raises(dw.DwcuError) as e:
        dw.deconvolve_tiled(im, psf, 20, 4, n_iter=2)
    assert e.value.code == 4


def test_release_cache_without_blocks():
    dw.release_cache()
    dw.release_cache(0)


def test_output_buffer_validation():
    """A caller's result buffer must be a C-contiguous float32 array of the
    image's shape; anything else is rejected before the library is called."""
    im = np.ones((4, 8, 8), np.float32)
    psf = np.ones((3, 3, 3), np.float32) / 27
    for bad in (np.empty((4, 8, 9), np.float32), np.empty((4, 8, 8), np.float64),
                np.empty((4, 8, 16), np.float32)[:, :, ::2]):
        with pytest.raises(ValueError):
            dw.run_method(im, psf, out=bad, n_iter=2)
        with pytest.raises(ValueError):
            dw.deconvolve_tiled(im, psf, 4, 1, out=bad, n_iter=2)
