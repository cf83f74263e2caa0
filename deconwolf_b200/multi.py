"""Independent deconvolution jobs over several GPUs, one process per GPU.

deconwolf deconvolves tiles (deconvolve_tiles, src/dw.c:2001-2229), channels
and whole images independently of each other; the only step that combines
jobs is the tile blend (tiling_put_tile, src/tiling.c:412-439).  So:

* jobs are assigned to ranks by estimated cost (padded job voxels x
  iterations): longest first, each to the least loaded rank, deterministic so
  that every rank computes the same assignment without communicating;
* each rank runs its jobs on its own GPU; there is no collective on the data
  path of a job;
* independent jobs: each result goes to rank 0 point to point;
* tiles: each rank blends its own tiles, in tile order, into a zero volume on
  its GPU (dwcu_tile_blend), and one reduce sums the volumes onto rank 0.
  Away from tile overlaps every voxel has one contribution, so the sum is
  exact there; in overlaps the additions happen in another order than in
  deconvolve_tiles (differences of a few float ulps).

With torch.distributed not initialised, everything runs in this process.
The per-job runner and the blender are parameters so that the host logic can
be exercised on CPU ranks; the defaults are the GPU path.
"""
from __future__ import annotations

import numpy as np

import deconwolf_b200 as _core


def job_cost(shape, psf_shape, iters: int, border_quality: int = 2, method: str = "shb") -> float:
    """Estimated work of one job: the padded job voxels x iterations."""
    work, _ = _core.plan_size(shape, psf_shape, border_quality, method)
    return float(work[0]) * float(work[1]) * float(work[2]) * float(max(1, iters))


def assign(costs, world: int) -> list[int]:
    """Rank of each job: longest job first, to the least loaded rank (the
    lowest rank on ties).  The same on every rank."""
    load = [0.0] * max(1, world)
    owner = [0] * len(costs)
    for i in sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i)):
        r = min(range(len(load)), key=lambda r: (load[r], r))
        owner[i] = r
        load[r] += float(costs[i])
    return owner


def _dist():
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist
    except Exception:
        pass
    return None


def _rank_world(group=None):
    d = _dist()
    if d is None:
        return 0, 1, None
    return d.get_rank(group), d.get_world_size(group), d


def _gpu_runner(im, psf, **kw):
    return _core.run_method(im, psf, **kw).out


def run_jobs(jobs, runner=None, group=None):
    """Run independent jobs, each a dict with ``image``, ``psf`` and ``kw``
    (options of :func:`run_method`, with ``n_iter``), over the ranks.  Rank 0
    returns the list of results in job order; other ranks return None."""
    import torch
    runner = runner or _gpu_runner
    rank, world, d = _rank_world(group)
    costs = [job_cost(j["image"].shape, j["psf"].shape, j["kw"].get("n_iter", 50),
                      j["kw"].get("border_quality", 2), j["kw"].get("method", "shb")) for j in jobs]
    owner = assign(costs, world)
    mine = {i: runner(j["image"], j["psf"], **j["kw"]) for i, j in enumerate(jobs) if owner[i] == rank}
    if world == 1:
        return [mine[i] for i in range(len(jobs))]
    dev = _transfer_device(d, group)
    if rank == 0:
        out = []
        for i, j in enumerate(jobs):
            if owner[i] == 0:
                out.append(mine[i])
            else:
                t = torch.empty(j["image"].shape, dtype=torch.float32, device=dev)
                d.recv(t, src=owner[i], group=group)
                out.append(t.cpu().numpy())
        return out
    for i in sorted(mine):
        d.send(torch.from_numpy(np.ascontiguousarray(mine[i])).to(dev), dst=0, group=group)
    return None


def _transfer_device(d, group):
    import torch
    return torch.device("cuda", torch.cuda.current_device()) if d.get_backend(group) == "nccl" else torch.device("cpu")


class _GpuVolume:
    """The default blender: a zero volume on this rank's GPU, tiles blended by
    dwcu_tile_blend."""

    def __init__(self, shape, tiles):
        import torch
        self.shape = shape
        self.tiles = _core.tiles_array(tiles)
        self.dev = torch.cuda.current_device()
        self.vol = torch.zeros(shape, dtype=torch.float32, device=f"cuda:{self.dev}")

    def blend(self, tid, tile_out, offset):
        import torch
        t = torch.from_numpy(np.ascontiguousarray(tile_out)).to(self.vol.device)
        torch.cuda.synchronize(self.vol.device)
        _core.tile_blend_device(self.vol.data_ptr(), self.shape, self.tiles, tid, t.data_ptr(), offset, self.dev)

    def tensor(self):
        return self.vol


def deconvolve_tiled(im: np.ndarray, psf: np.ndarray, tile_size: int, overlap: int = 20, offset: float = 5.0,
                     xycropfactor: float = 0.001, runner=None, blender=None, group=None, **kw):
    """deconvolve_tiles over the ranks: ``psf`` as dw_run hands it over.  Rank
    0 returns the blended volume (numpy), other ranks None.  ``blender(shape,
    tiles)`` makes an object with ``blend(tid, tile_out, offset)`` and
    ``tensor()`` (a torch tensor on the device the process group uses)."""
    runner = runner or _gpu_runner
    blender = blender or _GpuVolume
    rank, world, d = _rank_world(group)
    tiles = _core.tiling_create(im.shape, tile_size, overlap)
    if len(tiles) < 2:
        raise ValueError("only one tile: omit the tile size or decrease it")
    bq = kw.get("border_quality", 2)
    shapes = [tuple(t["xsize"][::-1]) for t in tiles]
    psfs = [_core.psf_prepare(psf, s, bq, xycropfactor) for s in shapes]
    costs = [job_cost(s, p.shape, kw.get("n_iter", 50), bq, kw.get("method", "shb")) for s, p in zip(shapes, psfs)]
    owner = assign(costs, world)
    vol = blender(im.shape, tiles)
    for tid, t in enumerate(tiles):
        if owner[tid] != rank:
            continue
        x0, x1, y0, y1, z0, z1 = t["xpos"]
        tile = np.ascontiguousarray(im[z0:z1 + 1, y0:y1 + 1, x0:x1 + 1], dtype=np.float32)
        if offset > 0:
            tile = tile + np.float32(offset)
        vol.blend(tid, runner(tile, psfs[tid], **kw), offset)
    v = vol.tensor()
    if world > 1:
        d.reduce(v, dst=0, group=group)
    return v.cpu().numpy() if rank == 0 else None


def _device_part(shape, psf_shape, world, rank, d, group, **kw):
    """This rank's part on its GPU (dwcu_slab_part_*), with the collectives
    the parts need: NCCL all-reduces on the part's stream, or (gloo) host
    barriers after synchronising that stream."""
    import torch
    dev = torch.cuda.current_device()
    nccl = d.get_backend(group) == "nccl"
    buf = torch.zeros(8, dtype=torch.float64, device=f"cuda:{dev}")
    tok = torch.zeros(1, dtype=torch.float32, device=f"cuda:{dev}")

    def barrier(stream):
        ext = torch.cuda.ExternalStream(stream, device=dev)
        if nccl:
            with torch.cuda.stream(ext):
                d.all_reduce(tok, group=group)
        else:
            ext.synchronize()
            d.barrier(group=group)

    def allreduce(stream, n, op):
        ext = torch.cuda.ExternalStream(stream, device=dev)
        rop = d.ReduceOp.SUM if op == 0 else d.ReduceOp.MIN
        if nccl:
            with torch.cuda.stream(ext):
                d.all_reduce(buf[:n], op=rop, group=group)
        else:
            ext.synchronize()
            t = buf[:n].cpu()
            d.all_reduce(t, op=rop, group=group)
            with torch.cuda.stream(ext):
                buf[:n].copy_(t)
            ext.synchronize()

    part = _core.SlabPart(shape, psf_shape, world, rank, buf.data_ptr(), barrier, allreduce, device=dev, **kw)
    part._keep = (buf, tok)  # the buffers live as long as the part
    return part


def deconvolve_split(im: np.ndarray, psf: np.ndarray, group=None, part=None, **kw):
    """One image split over the ranks of a process group, one GPU per rank
    (dwcu_slab_part_*): rank r holds the z planes r, r + world, ... of the job
    and the z-pass columns of its slab; the spectra are shared through CUDA
    IPC handles (exchanged with all_gather_object), the ordering points are
    stream-ordered all-reduces on the part's stream (NCCL) or host barriers
    after a stream synchronisation (gloo), and the image sum and the
    I-divergence sums are all-reduced.  Every rank passes the whole image
    and PSF and gets the whole result (its own planes plus an all-reduce of
    the others').  Without an initialised process group: one part in this
    process (dwcu_deconvolve_slabs).  ``part``: a factory
    ``part(shape, psf_shape, world, rank)`` of this rank's part (default: the
    GPU part), so that the orchestration can run on CPU ranks."""
    d = _dist()
    if d is None:
        return _core.run_slabs(im, psf, parts=1, **kw)
    rank, world = d.get_rank(group), d.get_world_size(group)
    p = (part(im.shape, psf.shape, world, rank) if part is not None
         else _device_part(im.shape, psf.shape, world, rank, d, group, **kw))
    try:
        mine = p.export()
        handles = [None] * world
        d.all_gather_object(handles, mine, group=group)
        for q in range(world):
            if q != rank:
                p.import_part(q, *handles[q])
        out = np.zeros(im.shape, dtype=np.float32)
        res = p.run(im, psf, out)
    finally:
        p.close()
    # every plane comes from exactly one rank: the sum is the result
    import torch
    if d.get_backend(group) == "nccl":
        t = torch.from_numpy(out).to(f"cuda:{torch.cuda.current_device()}")
        d.all_reduce(t, group=group)
        res.out = t.cpu().numpy()
    else:
        t = torch.from_numpy(out)
        d.all_reduce(t, group=group)
        res.out = t.numpy()
    return res
