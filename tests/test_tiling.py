"""Tiling and PSF preparation (CPU): the host side of dw_run around the method
call, and the oracle's tiled deconvolution, pinned against the reference's
tiling.c compiled into oracle/_ref.

* tiling_create (tiling.c:70-130): the C ABI's dwcu_tiling_create and the
  oracle's restatement equal the reference's tiles exactly;
* the blend weights and the whole in-memory deconvolve_tiles of the oracle
  equal the reference's tiling_get_tile / tiling_put_tile path bit for bit;
* dwcu_psf_prepare equals the oracle's restatement of dw_run's PSF
  preparation (normalise, psf_autocrop, normalise) bit for bit.
"""
import numpy as np
import pytest

import deconwolf_b200 as dw
from oracle import pyoracle as po
from tests.helpers import gauss_psf, poisson_image

needs_ref = pytest.mark.skipif(not po.available("reference"), reason="oracle/_ref not built")


def _abi_tiles(shape, max_size, overlap):
    t = dw.tiling_create(shape, max_size, overlap)
    return np.array([list(d["size"]) + list(d["pos"]) + list(d["xpos"]) + list(d["xsize"]) for d in t],
                    dtype=np.int64)


TILINGS = [
    ((5, 100, 90), 40, 7),
    ((3, 2048, 2048), 1024, 50),
    ((2, 4096, 4096), 1024, 50),
    ((2, 4096, 4096), 512, 50),
    ((1, 333, 101), 100, 20),
    ((4, 1000, 999), 333, 0),
    ((6, 77, 1500), 700, 90),
    ((60, 3001, 2999), 1000, 50),
]


@needs_ref
@pytest.mark.parametrize("shape,max_size,overlap", TILINGS)
def test_tiling_equals_reference(shape, max_size, overlap):
    ref = po.tiling_create(shape, max_size, overlap, impl="reference")
    np.testing.assert_array_equal(po.tiling_create(shape, max_size, overlap), ref)
    np.testing.assert_array_equal(_abi_tiles(shape, max_size, overlap), ref)


def test_tiling_properties():
    rng = np.random.default_rng(5)
    for _ in range(40):
        M, N = (int(v) for v in rng.integers(10, 5000, 2))
        ms = int(rng.integers(5, 2000))
        ov = int(rng.integers(0, 100))
        t = _abi_tiles((3, N, M), ms, ov)
        nx = int(np.ceil(M / ms))
        ny = int(np.ceil(N / ms))
        assert len(t) == nx * ny
        # owned regions partition the image; x-section outer, y-section inner
        cover = np.zeros((N, M), np.int32)
        for k, r in enumerate(t):
            pos, xpos = r[3:9], r[9:15]
            cover[pos[2]:pos[3] + 1, pos[0]:pos[1] + 1] += 1
            assert xpos[0] == max(0, pos[0] - ov) and xpos[1] == min(M - 1, pos[1] + ov)
            assert pos[0] == t[(k // ny) * ny][3] and pos[2] == t[k % ny][5]
        assert cover.min() == 1 and cover.max() == 1


@needs_ref
def test_weights_equal_reference():
    shape, ms, ov = (2, 61, 77), 20, 5
    t = po.tiling_create(shape, ms, ov)
    for tid in (0, 4, len(t) - 1):
        wt, ws = po.tiling_weights(shape, ms, ov, tid)
        assert ws.min() >= 1.0 - 1e-6  # every pixel is owned by one tile (weight 1)
        assert wt.max() == 1.0


@needs_ref
@pytest.mark.parametrize("method", ["shb", "rl"])
def test_tiled_oracle_equals_reference(method):
    psf = gauss_psf((7, 9, 9), (1.2, 1.5, 1.7), seed=3, jitter=0.2)
    im = poisson_image((8, 60, 50), psf, seed=3, bg=50.0, npts=20)
    pp = po.psf_prepare(psf, im.shape)
    a = po.deconvolve_tiled(im, pp, 25, 6, method=method, n_iter=6)
    b = po.deconvolve_tiled(im, pp, 25, 6, method=method, n_iter=6, impl="reference")
    np.testing.assert_array_equal(a.out, b.out)
    assert a.iterations == b.iterations == 6


def test_tiled_one_tile_rejected():
    psf = gauss_psf((3, 5, 5), (1, 1, 1))
    im = np.full((4, 20, 20), 10, np.float32)
    with pytest.raises(RuntimeError):
        po.deconvolve_tiled(im, psf, 40, 5, n_iter=2)


PSF_CASES = [
    # (psf shape, image shape, bq, xycropfactor)
    ((119, 181, 181), (60, 2048, 2048), 2, 0.001),   # z crop 119 -> 119, XY crop of a wide PSF
    ((79, 127, 127), (40, 256, 256), 2, 0.001),      # z crop 79 -> 79
    ((41, 31, 31), (10, 12, 14), 2, 0.001),          # crop to 2*size-1 in x, y and z
    ((41, 31, 31), (10, 12, 14), 0, 0.001),          # bq 0: crop to the image size
    ((41, 31, 31), (10, 12, 14), 1, 0.0),            # no XY crop
    ((9, 31, 31), (10, 12, 14), 2, 0.001),           # too few slices: returned as is
    ((15, 25, 25), (8, 40, 40), 2, 0.05),            # strong XY crop
]


@pytest.mark.parametrize("pshape,ishape,bq,xy", PSF_CASES)
def test_psf_prepare_equals_reference(pshape, ishape, bq, xy):
    """dwcu_psf_prepare against deconwolf's own dw.c (psf_autocrop compiled
    unmodified into oracle/_ref/libdwpsf.so), bit for bit."""
    psf = gauss_psf(pshape, (pshape[0] / 6, pshape[1] / 8, pshape[2] / 7), seed=2, jitter=0.1)
    ref = po.psf_prepare_reference(psf, ishape, bq, xy)
    if ref is None:
        pytest.skip("reference PSF preparation not built (needs deconwolf's sources)")
    np.testing.assert_array_equal(dw.psf_prepare(psf, ishape, bq, xy), ref)


def test_psf_prepare_born_wolf_equals_reference():
    """The Born-Wolf PSFs of the benchmark workloads, prepared for their images."""
    from deconwolf_b200 import synthetic
    for pshape, ishape, lam in (((79, 127, 127), (40, 256, 256), 466.0), ((39, 121, 121), (20, 256, 256), 525.0)):
        psf = synthetic.bw_psf(pshape, lam=lam)
        ref = po.psf_prepare_reference(psf, ishape, 2, 0.001)
        if ref is None:
            pytest.skip("reference PSF preparation not built (needs deconwolf's sources)")
        np.testing.assert_array_equal(dw.psf_prepare(psf, ishape, 2, 0.001), ref)


@pytest.mark.parametrize("pshape,ishape,bq,xy", PSF_CASES)
def test_psf_prepare_equals_oracle(pshape, ishape, bq, xy):
    psf = gauss_psf(pshape, (pshape[0] / 6, pshape[1] / 8, pshape[2] / 7), seed=2, jitter=0.1)
    a = dw.psf_prepare(psf, ishape, bq, xy)
    b = po.psf_prepare(psf, ishape, bq, xy)
    np.testing.assert_array_equal(a, b)
    assert abs(float(a.sum(dtype=np.float64)) - 1.0) < 1e-5
    # byImage crop keeps the centre: size - 2 * ((size - opt) // 2) (dw.c:1815-1830)
    P, N, M = ishape
    opt = (P, N, M) if bq == 0 else (2 * P - 1, 2 * N - 1, 2 * M - 1)
    if pshape[0] < opt[0]:
        assert a.shape == pshape
    else:
        want = tuple(s - 2 * ((s - o) // 2) if s > o else s for s, o in zip(pshape, opt))
        assert a.shape[0] == want[0]
        if xy == 0 or bq == 0:
            assert a.shape == want
        else:
            assert a.shape[1] <= want[1] and a.shape[2] <= want[2]
            assert want[1] - a.shape[1] == want[2] - a.shape[2]  # the same planes go in x and y
