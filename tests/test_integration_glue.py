"""The reference-side binding (deconwolf_b200/glue/method_shb_cu.c): it
compiles against the reference's src/dw.h with -Wall -Wextra -Werror and links
against libdwcu.so with no undefined symbol (oracle/Makefile builds it into
oracle/_ref/libdwglue.so together with tests/glue_driver.c); on a GPU the
dw_function it provides returns exactly what dwcu_deconvolve returns."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import deconwolf_b200 as dw
from tests.helpers import gauss_psf, poisson_image

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GLUE = os.path.join(ROOT, "oracle", "_ref", "libdwglue.so")


def _glue():
    lib = ctypes.CDLL(GLUE)
    i64, vp = ctypes.c_int64, ctypes.c_void_p
    lib.glue_run.argtypes = [vp, i64, i64, i64, vp, i64, i64, i64, ctypes.c_int, ctypes.c_int, vp,
                             ctypes.POINTER(ctypes.c_float)]
    lib.glue_run.restype = ctypes.c_int
    return lib


@pytest.mark.skipif(not os.path.exists(dw.LIB_PATH), reason="needs libdwcu.so")
def test_glue_compiles_and_links():
    # the recipe builds the glue wherever the reference sources are present
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True,
                   stdout=subprocess.DEVNULL)
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libdwref.so")):
        pytest.skip("reference sources absent: the glue cannot be compiled here")
    assert os.path.exists(GLUE)
    lib = _glue()
    for name in ("deconvolve_shb_cu", "deconvolve_rl_cu", "glue_run"):
        assert hasattr(lib, name)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(GLUE), reason="glue library not built")
@pytest.mark.parametrize("method", ["shb", "rl"])
def test_glue_dw_function_equals_abi(method):
    psf = gauss_psf((5, 7, 9), (1.2, 1.5, 1.7), seed=2, jitter=0.2)
    im = poisson_image((9, 22, 19), psf, seed=2, bg=50.0, npts=15)
    ref = dw.run_method(im, psf, method=method, n_iter=9, iter_type=dw.ITER_FIXED)
    out = np.empty_like(im)
    bg = ctypes.c_float()
    P, N, M = im.shape
    pP, pN, pM = psf.shape
    rc = _glue().glue_run(im.ctypes.data, M, N, P, psf.ctypes.data, pM, pN, pP, 0 if method == "rl" else 2, 9,
                          out.ctypes.data, ctypes.byref(bg))
    assert rc == 0
    np.testing.assert_array_equal(out, ref.out)
    assert bg.value == ref.bg
