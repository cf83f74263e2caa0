"""One image split over processes, one part per process
(dwcu_slab_part_*, multi.deconvolve_split).

* Two processes on one GPU with gloo: the ordering points are host barriers
  after a stream synchronisation, so no kernel of one process waits on the
  other's; the peer spectra are mapped through CUDA IPC handles.  The result
  equals the same split run by one process (dwcu_deconvolve_slabs, 2 parts)
  bit for bit, in both exchange forms.
* One process with NCCL: the callbacks' stream-ordered all-reduces on the
  part's stream; the result equals the one-part split bit for bit.
Both with the heuristic plans (the split over processes never measures
plans of its own)."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

import deconwolf_b200 as dw
from oracle import pyoracle as po
from tests.helpers import gauss_psf, poisson_image, rel_l2

pytestmark = pytest.mark.gpu


def _inputs():
    psf = gauss_psf((7, 9, 11), (1.3, 1.6, 1.9), seed=71, jitter=0.2)
    im = poisson_image((12, 40, 44), psf, seed=71, bg=60.0, npts=20)
    return im, psf


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, backend, path, env, case):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    os.environ.update(env)
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    import deconwolf_b200 as dw
    from deconwolf_b200 import multi
    torch.cuda.set_device(0)
    dist.init_process_group(backend, rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        dw.tune_set_mode(dw.TUNE_OFF)
        im, psf = _inputs()
        r = multi.deconvolve_split(im, psf, **case)
        np.savez(f"{path}.{rank}.npz", out=r.out, trace=r.trace, iterations=r.iterations)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run(tmp_path, world, backend, env, case):
    ctx = mp.get_context("spawn")
    port = _free_port()
    path = str(tmp_path / "split")
    procs = [ctx.Process(target=_worker, args=(r, world, port, backend, path, env, case)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=400)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert [p.exitcode for p in procs] == [0] * world
    return [np.load(f"{path}.{r}.npz") for r in range(world)]


@pytest.fixture
def heuristic_plans():
    dw.tune_set_mode(dw.TUNE_OFF)
    dw.tune_clear()
    yield
    dw.tune_set_mode(dw.TUNE_MEASURE)
    dw.tune_clear()


CASES = [
    (dict(method="shb", n_iter=12), {}),
    (dict(method="shb", n_iter=12), {"DWCU_SLAB_TRANSPOSE": "copy"}),
    (dict(method="rl", iter_type=po.ITER_REL, err_rel=0.002, maxiter=40), {}),
    (dict(method="shb", n_iter=8, start=po.START_LP, border_quality=1), {}),
]


@pytest.mark.parametrize("case,env", CASES, ids=lambda v: "-".join(f"{k}={x}" for k, x in v.items()) or "direct")
def test_two_processes_equal_one_process(tmp_path, case, env, heuristic_plans, monkeypatch):
    res = _run(tmp_path, 2, "gloo", env, case)
    im, psf = _inputs()
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    ref = dw.run_slabs(im, psf, parts=2, **case)
    whole = dw.run_method(im, psf, **case)
    for r in res:  # every rank holds the whole result
        assert int(r["iterations"]) == ref.iterations
        np.testing.assert_array_equal(r["out"], ref.out)
        np.testing.assert_array_equal(r["trace"], ref.trace)
    assert rel_l2(res[0]["out"], whole.out) < 1e-5


def test_three_processes_equal_one_process(tmp_path, heuristic_plans):
    case = dict(method="shb", n_iter=9, border_quality=1)
    res = _run(tmp_path, 3, "gloo", {}, case)
    im, psf = _inputs()
    ref = dw.run_slabs(im, psf, parts=3, **case)
    for r in res:
        np.testing.assert_array_equal(r["out"], ref.out)
        np.testing.assert_array_equal(r["trace"], ref.trace)


def test_nccl_single_rank_equals_one_part(tmp_path, heuristic_plans):
    case = dict(method="shb", n_iter=10)
    res = _run(tmp_path, 1, "nccl", {}, case)
    im, psf = _inputs()
    ref = dw.run_slabs(im, psf, parts=1, **case)
    np.testing.assert_array_equal(res[0]["out"], ref.out)
    np.testing.assert_array_equal(res[0]["trace"], ref.trace)


def test_run_before_every_part_is_mapped_is_refused():
    import torch
    im, psf = _inputs()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    part = dw.SlabPart(im.shape, psf.shape, 2, 0, buf.data_ptr(), lambda s: None, lambda s, n, op: None,
                       method="shb", n_iter=3)
    with pytest.raises(dw.DwcuError) as e:
        part.run(im, psf, np.zeros(im.shape, np.float32))
    assert e.value.code == 1  # DWCU_ERROR_INVALID_VALUE: part 1 was never imported
    part.close()
