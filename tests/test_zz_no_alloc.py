"""dwcu_fft_r2c_noalloc against dwcu_fft_r2c: the same transform from the
library's fixed work space, two calls in a row, within the FFT tolerance
(relative to the largest coefficient, 1e-6); sizes beyond the work space are
rejected.  Named to be collected after the other GPU tests."""
import numpy as np
import pytest

import deconwolf_b200 as dw

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("shape", [(12, 20, 16), (5, 9, 14), (7, 12, 384), (1, 1, 2240), (40, 64, 60)])
def test_noalloc_equals_fft_r2c(shape):
    import torch
    rng = np.random.default_rng(11)
    x = rng.random(shape).astype(np.float32)
    P, N, M = shape
    d_x = _dev(x)
    d_ref = torch.empty((P, N, M // 2 + 1), dtype=torch.complex64, device="cuda")
    d_a = torch.empty_like(d_ref)
    d_b = torch.empty_like(d_ref)
    torch.cuda.synchronize()
    dw.fft_r2c_device(d_x.data_ptr(), shape, d_ref.data_ptr())
    dw.fft_r2c_noalloc_device(d_x.data_ptr(), shape, d_a.data_ptr())
    dw.fft_r2c_noalloc_device(d_x.data_ptr(), shape, d_b.data_ptr())
    ref = d_ref.cpu().numpy()
    scale = np.max(np.abs(ref))
    for out in (d_a.cpu().numpy(), d_b.cpu().numpy()):
        assert np.max(np.abs(out - ref)) / scale < TOL
        # same kernels, and twiddle tables built on the device by the same
        # double-precision series the host uses: the results are identical
        np.testing.assert_array_equal(out, ref)
    np.testing.assert_array_equal(d_a.cpu().numpy(), d_b.cpu().numpy())
    # and against the FP64 transform
    exact = np.fft.rfftn(x.astype(np.float64))
    assert np.max(np.abs(d_a.cpu().numpy() - exact)) / np.max(np.abs(exact)) < 2e-6


def test_noalloc_rejects_oversized():
    import torch
    shape = (64, 256, 256)  # spectrum + staged input > 32 MiB
    P, N, M = shape
    d_x = torch.zeros(shape, dtype=torch.float32, device="cuda")
    d_y = torch.empty((P, N, M // 2 + 1), dtype=torch.complex64, device="cuda")
    with pytest.raises(dw.DwcuError) as e:
        dw.fft_r2c_noalloc_device(d_x.data_ptr(), shape, d_y.data_ptr())
    assert e.value.code == 1
    assert "work space" in str(e.value)
    # still usable afterwards
    small = (4, 6, 8)
    d_s = torch.ones(small, dtype=torch.float32, device="cuda")
    d_S = torch.empty((4, 6, 5), dtype=torch.complex64, device="cuda")
    dw.fft_r2c_noalloc_device(d_s.data_ptr(), small, d_S.data_ptr())
    S = d_S.cpu().numpy()
    assert abs(S[0, 0, 0] - 4 * 6 * 8) < 1e-3 and np.max(np.abs(S.reshape(-1)[1:])) < 1e-3
