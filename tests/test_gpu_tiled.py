"""GPU tests of the batched paths: dwcu_batch_run and the tiled
deconvolution (dwcu_deconvolve_tiled) against the oracle's in-memory
deconvolve_tiles (pinned bit for bit to the reference's tiling.c path on the
CPU) and against the reference itself.

Tolerance as for one image: relative L2 of the blended output <= 1e-4.
"""
import numpy as np
import pytest

import deconwolf_b200 as dw
from oracle import pyoracle as po
from tests.helpers import gauss_psf, poisson_image, rel_l2

pytestmark = pytest.mark.gpu

OUT_TOL = 1e-4


def _inputs(shape=(8, 70, 64), psf_shape=(7, 9, 9), seed=11):
    psf = gauss_psf(psf_shape, (1.2, 1.5, 1.7), seed=seed, jitter=0.2)
    im = poisson_image(shape, psf, seed=seed, bg=60.0, npts=25)
    return im, psf


@pytest.mark.parametrize("method", ["shb", "rl"])
def test_tiled_matches_oracle(method):
    im, psf = _inputs()
    pp = dw.psf_prepare(psf, im.shape)
    g = dw.deconvolve_tiled(im, pp, 30, 6, method=method, n_iter=8)
    p = po.deconvolve_tiled(im, pp, 30, 6, method=method, n_iter=8)
    assert g.iterations == p.iterations == 8
    assert rel_l2(g.out, p.out) < OUT_TOL
    if po.available("reference"):
        r = po.deconvolve_tiled(im, pp, 30, 6, method=method, n_iter=8, impl="reference")
        assert rel_l2(g.out, r.out) < OUT_TOL


def test_tiled_rel_stopping_matches_oracle():
    im, psf = _inputs(shape=(6, 50, 58), seed=12)
    pp = dw.psf_prepare(psf, im.shape)
    kw = dict(method="shb", iter_type=dw.ITER_REL, err_rel=0.01, maxiter=40)
    g = dw.deconvolve_tiled(im, pp, 20, 5, **kw)
    p = po.deconvolve_tiled(im, pp, 20, 5, iter_type=po.ITER_REL, err_rel=0.01, maxiter=40, method="shb")
    assert g.iterations == p.iterations
    assert rel_l2(g.out, p.out) < OUT_TOL


def test_tiled_waves_give_the_same_result():
    """One tile per batch (tiny HBM budget) equals all tiles in one batch."""
    im, psf = _inputs(seed=13)
    pp = dw.psf_prepare(psf, im.shape)
    a = dw.deconvolve_tiled(im, pp, 25, 4, n_iter=6)
    b = dw.deconvolve_tiled(im, pp, 25, 4, n_iter=6, hbm_budget=1.0)
    np.testing.assert_array_equal(a.out, b.out)


def test_tiled_single_tile_rejected():
    im, psf = _inputs(shape=(4, 20, 20), psf_shape=(3, 5, 5))
    with pytest.raises(dw.DwcuError) as e:
        dw.deconvolve_tiled(im, psf, 64, 5, n_iter=2)
    assert e.value.code == 1


def test_dw_run_tiled_and_untiled():
    im, psf = _inputs(seed=14)
    pp = po.psf_prepare(psf, im.shape)
    # untiled: the result keeps the offset (dw_run's result buffer)
    u = dw.dw_run(im, psf, n_iter=5)
    r = po.deconvolve(im + np.float32(5.0), pp, n_iter=5)
    assert rel_l2(u, r.out) < OUT_TOL
    t = dw.dw_run(im, psf, n_iter=5, tilesize=30, tilepad=6)
    rt = po.deconvolve_tiled(im, pp, 30, 6, n_iter=5)
    assert rel_l2(t, rt.out) < OUT_TOL


def test_batch_run_equals_one_at_a_time():
    """Jobs of uneven sizes, methods and stopping rules stepped together by
    dwcu_batch_run give exactly the results of separate calls."""
    cases = [
        ((9, 22, 19), (5, 7, 9), dict(method="shb", n_iter=12)),
        ((6, 40, 31), (3, 5, 5), dict(method="rl", n_iter=7)),
        ((12, 30, 44), (7, 7, 7), dict(method="shb", iter_type=dw.ITER_REL, err_rel=0.002, maxiter=30)),
        ((1, 30, 26), (1, 7, 9), dict(method="shb", n_iter=20)),
    ]
    jobs, refs = [], []
    for k, (shape, pshape, kw) in enumerate(cases):
        psf = gauss_psf(pshape, (1.2, 1.5, 1.7), seed=k, jitter=0.2)
        im = poisson_image(shape, psf, seed=k, bg=40.0, npts=12)
        refs.append(dw.run_method(im, psf, **kw))
        j = dw.Job(im.shape, psf.shape, **kw)
        j.setup(im, psf)
        jobs.append(j)
    dw.batch_run(jobs)
    for j, ref in zip(jobs, refs):
        assert j.done()
        r = j.result()
        j.close()
        assert r.iterations == ref.iterations
        np.testing.assert_array_equal(r.out, ref.out)
        np.testing.assert_array_equal(r.trace, ref.trace)


def test_multi_layer_single_rank_equals_batched():
    """The multi-GPU layer run in one process (tiles one by one through
    dwcu_deconvolve, blended on the device by dwcu_tile_blend) gives the
    batched tiled result exactly."""
    from deconwolf_b200 import multi
    im, psf = _inputs(seed=15)
    pp = dw.psf_prepare(psf, im.shape)
    a = dw.deconvolve_tiled(im, pp, 30, 6, n_iter=7).out
    b = multi.deconvolve_tiled(im, pp, 30, 6, n_iter=7)
    np.testing.assert_array_equal(a, b)
    jobs = [dict(image=im[:, :40, :40].copy(), psf=psf, kw=dict(n_iter=4)),
            dict(image=im[:, 20:, 10:].copy(), psf=psf, kw=dict(n_iter=3, method="rl"))]
    res = multi.run_jobs(jobs)
    for j, r in zip(jobs, res):
        np.testing.assert_array_equal(r, dw.run_method(j["image"], j["psf"], **j["kw"]).out)


def test_tiled_pair_golden():
    """The tiled path at full size: a 2048 x 1024 x 60 image at tile size 1024
    and overlap 50 (two tiles of 1074-1124 x 1024 x 60, each with its own PSF
    crop, weighted blend), SHB 50, against the reference's own tiled path
    (tiling.c with the reference's method code): every plane sum, the norm,
    131072 sampled voxels and the whole-volume sketch."""
    import os
    f = os.path.join(os.path.dirname(__file__), "golden", "tiled2_shb50.npz")
    if not os.path.exists(f):
        pytest.skip("tiled fixture not generated")
    from deconwolf_b200 import synthetic
    from tests.helpers import sketch, sketch_rel_l2
    d = np.load(f)
    im, psf = synthetic.tiled_pair_inputs()
    idx = d["sample_idx"]
    np.testing.assert_array_equal(im.reshape(-1)[idx], d["image_sample"])
    pp = dw.psf_prepare(psf, im.shape)
    assert tuple(pp.shape) == tuple(d["psf_shape"])
    g = dw.deconvolve_tiled(im, pp, 1024, 50, method="shb", n_iter=50)
    assert rel_l2(g.out.reshape(-1)[idx], d["sample_val"]) < OUT_TOL
    assert rel_l2(g.out.astype(np.float64).sum(axis=(1, 2)), d["plane_sums"]) < OUT_TOL
    est = sketch_rel_l2(sketch(g.out, device="cuda"), d["sketch"], float(d["norm"]))
    print(f"\ntiled 2048x1024x60 (2 tiles): relative L2 to the reference tiled path (sketch) {est:.3e}")
    assert est < OUT_TOL


@pytest.mark.parametrize("offset", [0.0, 5.0])
def test_tile_paste_round_trip(offset):
    """tiling_ut (src/tiling_ut.c:88-152): an image of constant 7 cut into
    overlapping tiles and pasted back with the blend weights is 7 again
    within 1e-4 -- here through the device blend (dwcu_tile_blend), each tile
    carrying the offset that the tiled path adds before deconvolving."""
    import torch
    shape = (3, 61, 77)
    tiles = dw.tiling_create(shape, 20, 5)
    arr = dw.tiles_array(tiles)
    d_out = torch.zeros(shape, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    for tid, t in enumerate(tiles):
        m, n, p = t["xsize"]
        d_tile = torch.full((p, n, m), 7.0 + offset, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        dw.tile_blend_device(d_out.data_ptr(), shape, arr, tid, d_tile.data_ptr(), offset=offset)
    out = d_out.cpu().numpy()
    assert len(tiles) == 16
    assert np.max(np.abs(out - 7.0)) < 1e-4
