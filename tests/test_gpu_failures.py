"""Failure detection without faulting the GPU.

* A device-side bounded wait (the mbarrier waits every pass uses for its
  bulk copies) that runs out of polls reports DWCU_ERROR_TIMEOUT through the
  error word the host reads; the device stays usable and later results are
  unchanged.
* A job that needs more device memory than the GPU has is refused with
  DWCU_ERROR_OUT_OF_MEMORY (the allocation fails; nothing is launched).
"""
import numpy as np
import pytest

import deconwolf_b200 as dw
from tests.helpers import gauss_psf, poisson_image

pytestmark = pytest.mark.gpu

ERROR_OUT_OF_MEMORY = 3
ERROR_TIMEOUT = 8


def _small():
    psf = gauss_psf((5, 7, 9), (1.2, 1.5, 1.7), seed=41, jitter=0.2)
    im = poisson_image((9, 22, 19), psf, seed=41, bg=50.0, npts=15)
    return im, psf


def test_bounded_wait_gives_up_and_the_device_stays_usable():
    im, psf = _small()
    ref = dw.run_method(im, psf, n_iter=6)
    assert dw.lib().dwcu_selftest_bounded_wait(0, 1, 1 << 12) == 0   # the phase completes
    rc = dw.lib().dwcu_selftest_bounded_wait(0, 0, 1 << 12)          # nothing completes it
    assert rc == ERROR_TIMEOUT
    assert "gave up" in dw.lib().dwcu_last_error().decode()
    again = dw.run_method(im, psf, n_iter=6)
    np.testing.assert_array_equal(again.out, ref.out)
    np.testing.assert_array_equal(again.trace, ref.trace)


def test_allocation_failure_is_reported():
    im, psf = _small()
    shape, psf_shape = (3900, 3900, 3900), (9, 9, 9)
    need = dw.plan_size(shape, psf_shape)[1]
    assert need > 1e12  # far beyond any GPU
    with pytest.raises(dw.DwcuError) as e:
        dw.Job(shape, psf_shape, method="shb", n_iter=2)
    assert e.value.code == ERROR_OUT_OF_MEMORY
    # the library and the device carry on
    assert dw.run_method(im, psf, n_iter=4).iterations == 4
