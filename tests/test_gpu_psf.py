"""PSF preparation on the device (dwcu_psf_prepare_device) against the host
version and against deconwolf's own dw.c (psf_autocrop compiled unmodified
into oracle/_ref/libdwpsf.so), bit for bit."""
import numpy as np
import pytest

import deconwolf_b200 as dw
from oracle import pyoracle as po
from tests.helpers import gauss_psf

pytestmark = pytest.mark.gpu

CASES = [
    # (psf shape, image shape, bq, xycropfactor)
    ((119, 181, 181), (60, 2048, 2048), 2, 0.001),
    ((79, 127, 127), (40, 256, 256), 2, 0.001),
    ((41, 31, 31), (10, 12, 14), 2, 0.001),
    ((41, 31, 31), (10, 12, 14), 0, 0.001),
    ((41, 31, 31), (10, 12, 14), 1, 0.0),
    ((9, 31, 31), (10, 12, 14), 2, 0.001),
    ((15, 25, 25), (8, 40, 40), 2, 0.05),
]


def _device(psf, ishape, bq, xy):
    import torch
    d_in = torch.from_numpy(np.ascontiguousarray(psf)).cuda()
    d_out = torch.empty(psf.size, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    shape = dw.psf_prepare_device(d_in.data_ptr(), psf.shape, ishape, d_out.data_ptr(), bq, xy)
    out = d_out[: int(np.prod(shape))].cpu().numpy().reshape(shape)
    np.testing.assert_array_equal(d_in.cpu().numpy(), psf)  # the input is not modified
    return out


@pytest.mark.parametrize("pshape,ishape,bq,xy", CASES)
def test_device_prepare_equals_host_and_reference(pshape, ishape, bq, xy):
    psf = gauss_psf(pshape, (pshape[0] / 6, pshape[1] / 8, pshape[2] / 7), seed=2, jitter=0.1)
    d = _device(psf, ishape, bq, xy)
    np.testing.assert_array_equal(d, dw.psf_prepare(psf, ishape, bq, xy))
    ref = po.psf_prepare_reference(psf, ishape, bq, xy)
    if ref is not None:
        np.testing.assert_array_equal(d, ref)


def test_device_prepare_born_wolf():
    from deconwolf_b200 import synthetic
    big = synthetic.bw_psf((119, 181, 181), lam=670.0)
    for psf, ishape in ((synthetic.bw_psf((79, 127, 127), lam=466.0), (40, 256, 256)), (big, (60, 1124, 1124)),
                        (big, (60, 562, 612))):
        d = _device(psf, ishape, 2, 0.001)
        np.testing.assert_array_equal(d, dw.psf_prepare(psf, ishape, 2, 0.001))
        ref = po.psf_prepare_reference(psf, ishape, 2, 0.001)
        if ref is not None:
            np.testing.assert_array_equal(d, ref)
