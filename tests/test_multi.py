"""Host logic of the multi-GPU layer on CPU ranks (gloo, world size 2): the
job assignment, results sent to rank 0, and the tiled deconvolution with
per-rank blending and one reduce -- with the oracle standing in for the GPU
runner and a NumPy blender standing in for the device blend, so that the
orchestration is what is tested."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from deconwolf_b200 import multi


def test_assign_balanced_and_deterministic():
    rng = np.random.default_rng(3)
    costs = list(rng.integers(1, 1000, 37))
    for world in (1, 2, 3, 8):
        a = multi.assign(costs, world)
        assert a == multi.assign(list(costs), world)
        assert set(a) <= set(range(world))
        load = np.zeros(world)
        for c, r in zip(costs, a):
            load[r] += c
        # longest-first greedy: within the largest job of the most even split
        assert load.max() - load.min() <= max(costs)
    assert multi.assign([5, 5, 5, 5], 2) == [0, 1, 0, 1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _weight1d(a, b, c, d, x):
    # getWeight1d, tiling.c:169-197, in float32
    a, b, c, d = (np.float32(v) for v in (a, b, c, d))
    x = np.float32(x)
    w = np.zeros_like(x)
    mid = (x >= b) & (x <= c)
    up = (x >= a) & (x < b)
    down = (x > c) & (x <= d)
    w[mid] = 1
    w[up] = (x[up] - a + np.float32(1)) / (b - a + np.float32(1))
    w[down] = np.float32(1) - (x[down] - c) / (d - c + np.float32(1))
    return w


class NumpyVolume:
    def __init__(self, shape, tiles):
        self.v = np.zeros(shape, np.float32)
        self.tiles = tiles
        P, N, M = shape
        self.M, self.N = M, N

    def _w(self, t, xs, ys):
        wx = _weight1d(t["xpos"][0], t["pos"][0], t["pos"][1], t["xpos"][1], xs)
        wy = _weight1d(t["xpos"][2], t["pos"][2], t["pos"][3], t["xpos"][3], ys)
        return np.minimum(wy[:, None], wx[None, :])

    def blend(self, tid, out, offset):
        t = self.tiles[tid]
        x0, x1, y0, y1, z0, z1 = t["xpos"]
        xs, ys = np.arange(x0, x1 + 1), np.arange(y0, y1 + 1)
        s = out.astype(np.float32)
        if offset > 0:
            s = np.maximum(s - np.float32(offset), np.float32(0))
        wsum = sum(self._w(u, xs, ys) for u in self.tiles)
        w = self._w(t, xs, ys) / wsum
        self.v[z0:z1 + 1, y0:y1 + 1, x0:x1 + 1] += w[None] * s

    def tensor(self):
        import torch
        return torch.from_numpy(self.v)


def _oracle_runner(im, psf, **kw):
    from oracle import pyoracle as po
    return po.deconvolve(im, psf, threads=2, **kw).out


def _inputs():
    from tests.helpers import gauss_psf, poisson_image
    psf = gauss_psf((7, 9, 9), (1.2, 1.5, 1.7), seed=3, jitter=0.2)
    im = poisson_image((8, 60, 50), psf, seed=3, bg=50.0, npts=20)
    return im, psf


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        im, psf = _inputs()
        import deconwolf_b200 as dw
        pp = dw.psf_prepare(psf, im.shape)
        out = multi.deconvolve_tiled(im, pp, 25, 6, runner=_oracle_runner, blender=NumpyVolume, n_iter=5)
        jobs = [dict(image=im[:, :30, :30].copy(), psf=psf, kw=dict(n_iter=3)),
                dict(image=im[:, 30:, 20:].copy(), psf=psf, kw=dict(n_iter=4, method="rl")),
                dict(image=im[:4].copy(), psf=psf[1:6], kw=dict(n_iter=2))]
        res = multi.run_jobs(jobs, runner=_oracle_runner)
        if rank == 0:
            q.put(("ok", out, res))
        else:
            q.put(("ok", out is None and res is None, None))
    except Exception as e:  # reported to the test
        q.put(("error", repr(e), None))
    finally:
        dist.destroy_process_group()


def test_two_ranks_match_one_process():
    from oracle import pyoracle as po
    import deconwolf_b200 as dw
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = [q.get(timeout=300) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    assert all(g[0] == "ok" for g in got), got
    r0 = [g for g in got if g[2] is not None]
    assert len(r0) == 1
    _, out, res = r0[0]
    assert any(g[1] is True for g in got)  # the other rank returned nothing
    im, psf = _inputs()
    pp = dw.psf_prepare(psf, im.shape)
    ref = po.deconvolve_tiled(im, pp, 25, 6, n_iter=5).out
    # exact away from overlaps; a few ulps where the ranks' blends are summed
    assert np.max(np.abs(out - ref) / np.maximum(np.abs(ref), 1)) < 1e-5
    jobs_ref = [_oracle_runner(im[:, :30, :30].copy(), psf, n_iter=3),
                _oracle_runner(im[:, 30:, 20:].copy(), psf, n_iter=4, method="rl"),
                _oracle_runner(im[:4].copy(), psf[1:6], n_iter=2)]
    for a, b in zip(res, jobs_ref):
        np.testing.assert_array_equal(a, b)


# ---------------------------------------------------------------- split over processes

class _FakePart:
    """Stands in for a rank's device part of a split job: its handle names
    the rank, and its run writes the rank's planes (z = rank, rank + world,
    ...) as twice the image."""

    def __init__(self, shape, psf_shape, world, rank):
        self.world, self.rank = world, rank
        self.imported = {}
        self.closed = False

    def export(self):
        return bytes([self.rank]) * 64, 1000 + self.rank

    def import_part(self, q, handle, offset):
        self.imported[q] = (handle[0], offset)

    def run(self, im, psf, out):
        out[self.rank::self.world] = 2 * im[self.rank::self.world]

        class R:
            pass
        r = R()
        r.out = out
        return r

    def close(self):
        self.closed = True


def _split_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        parts = []

        def factory(shape, psf_shape, w, r):
            parts.append(_FakePart(shape, psf_shape, w, r))
            return parts[-1]

        im = np.arange(7 * 5 * 4, dtype=np.float32).reshape(7, 5, 4)
        res = multi.deconvolve_split(im, np.ones((3, 3, 3), np.float32), part=factory)
        q.put((rank, parts[0].imported, parts[0].closed, res.out))
    finally:
        dist.destroy_process_group()


def test_split_over_ranks_exchanges_handles_and_combines_planes():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_split_worker, args=(world, _free_port(), q), nprocs=world, join=True, start_method="spawn")
    got = sorted(q.get() for _ in range(world))
    im = np.arange(7 * 5 * 4, dtype=np.float32).reshape(7, 5, 4)
    for rank, imported, closed, out in got:
        others = [r for r in range(world) if r != rank]
        assert imported == {r: (r, 1000 + r) for r in others}  # every other rank's handle and offset
        assert closed
        np.testing.assert_array_equal(out, 2 * im)  # every rank's planes, on every rank


class _FailingPart(_FakePart):
    def run(self, im, psf, out):
        if self.rank == 1:
            raise RuntimeError("part failed")
        return super().run(im, psf, out)


def _failing_worker(rank, world, port, q):
    from datetime import timedelta
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=10))
    outcome = "finished"
    try:
        im = np.zeros((6, 5, 4), np.float32)
        multi.deconvolve_split(im, np.ones((3, 3, 3), np.float32),
                               part=lambda shape, psf_shape, w, r: _FailingPart(shape, psf_shape, w, r))
    except Exception as e:  # the failing part, or the peer's collective ending with an error
        outcome = type(e).__name__ + ": " + str(e)[:60]
    q.put((rank, outcome))
    if rank == 1:
        return  # leaves without the result's collective, as a crashed rank would
    try:
        dist.destroy_process_group()
    except Exception:
        pass


def test_a_failing_rank_ends_the_split_on_every_rank():
    """A rank whose part fails leaves the split; the other rank's next
    collective ends with an error within the process group's timeout
    instead of waiting for good."""
    import time
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    t0 = time.time()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    alive = [p.is_alive() for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert not any(alive), "a rank waited for good"
    got = dict(q.get() for _ in range(world))
    assert got[1].startswith("RuntimeError: part failed")
    assert got[0] != "finished"
    assert time.time() - t0 < 120
