"""Benchmark: SHB deconvolution of the 2048 x 2048 x 60 synthetic workload.

One step = one full `dw --method shb --iter 50` deconvolution of the seeded
synthetic 2048 x 2048 x 60 image with a 181 x 181 x 119 Born-Wolf PSF
(lambda 670 nm): setup (background, OTF, Bertero weights, start) and 50 SHB
iterations, on one B200 per rank.  Metric: Mvoxel*iter/s = image voxels x
iterations / seconds, summed over ranks (weak scaling: every rank
deconvolves its own image; no collective on the data path).

  value  device-resident inputs (dwcu_deconvolve_device), CUDA events on the
         engine's stream, max over ranks
  e2e    the host-buffer C-ABI call dwcu_deconvolve from pinned host memory,
         including the image/PSF upload and the result download
  roofline  the dominant kernel class of the timed steps: algorithmic bytes
         per launch / mean event time per launch, against the measured HBM
         copy bandwidth (MEASURED_PEAKS.json)
  cpu_baseline  deconwolf's own CPU SHB (oracle/_ref) on a bounded crop of
         the same workload, extrapolated to the full job size

`python bench.py --impl reference` times the reference CPU path alone (rank
0; other ranks exit).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "shb-2048x2048x60"
SMALL = "shb-256x256x40"
PROFILE_CASE = "shb-1024x1024x20"  # hardware-counter captures (profiles/)
ITERS = 50
# generated inputs are cached between runs on one machine, outside the
# repository (a 2048 x 2048 x 60 image is about 1 GB)
CACHE = os.environ.get("DWCU_INPUT_CACHE", os.path.join(tempfile.gettempdir(), "dwcu_input_cache"))


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.thr = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thr = threading.Thread(target=self._read, daemon=True)
        self.thr.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thr:
            self.thr.join(timeout=5)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---------------------------------------------------------------- reference arm

def cpu_reference(im, psf, n_iter: int, crop: int):
    """deconwolf's CPU SHB (oracle/_ref) on a crop x crop x P corner of the
    image with the full PSF; returns seconds per iteration measured by the
    iterator and the job voxel count of the crop."""
    from oracle import pyoracle as po
    sub = np.ascontiguousarray(im[:, :crop, :crop])
    impl = "reference" if po.available("reference") else "port"
    r = po.deconvolve(sub, psf, method="shb", n_iter=n_iter, impl=impl, threads=os.cpu_count())
    P, N, M = sub.shape
    pP, pN, pM = psf.shape
    job = (M + pM - 1) * (N + pN - 1) * (P + pP - 1)
    return r.loop_seconds / max(1, r.iterations), job, impl


def full_job_voxels(shape, psf_shape):
    P, N, M = shape
    pP, pN, pM = psf_shape
    return (M + pM - 1) * (N + pN - 1) * (P + pP - 1)


def cpu_baseline_entry(im, psf, crop=384, iters=2):
    per_it, job_crop, impl = cpu_reference(im, psf, iters, crop)
    full_job = full_job_voxels(im.shape, psf.shape)
    t_full = per_it * full_job / job_crop
    vox = im.size
    return {
        "value": vox * 1e-6 / t_full, "unit": "Mvoxel*iter/s", "cores": os.cpu_count(),
        "kind": "reference" if impl == "reference" else "port",
        "sample": (f"{iters} SHB iterations of deconwolf's CPU method code ({impl} build, FFTW replaced by the "
                   f"oracle FFT) on a {crop}x{crop}x{im.shape[0]} crop with the full PSF "
                   f"(job {crop + psf.shape[2] - 1}x{crop + psf.shape[1] - 1}x{im.shape[0] + psf.shape[0] - 1}); "
                   f"{per_it:.2f} s/iteration extrapolated per job voxel to the full job"),
    }


def run_reference_arm(args):
    """deconwolf's own CPU SHB (oracle/_ref: the reference's method code,
    FFTW replaced by the oracle FFT) with all host threads, on a bounded crop
    of the workload: warm-up + timed iterations in one run, the timed ones
    read from the reference iterator's per-iteration timestamps, scaled per
    job voxel to the full job (time is linear in job voxels for a fixed PSF)."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    from deconwolf_b200 import synthetic
    im, psf = synthetic.config_inputs(args.workload, CACHE)
    P, N, M = im.shape
    crop = min(M, N, 384 if args.steps + args.warmup <= 12 else 256)
    from oracle import pyoracle as po
    sub = np.ascontiguousarray(im[:, :crop, :crop])
    impl = "reference" if po.available("reference") else "port"
    n = args.warmup + args.steps
    r = po.deconvolve(sub, psf, method="shb", n_iter=n, impl=impl, threads=os.cpu_count())
    if impl == "reference":
        ts = po.iteration_seconds()
        per_it = float(np.mean(ts[args.warmup:n])) if len(ts) >= n else r.loop_seconds / max(1, r.iterations)
    else:
        per_it = r.loop_seconds / max(1, r.iterations)
    job_crop = full_job_voxels(sub.shape, psf.shape)
    t_full = per_it * full_job_voxels(im.shape, psf.shape) / job_crop
    value = im.size * 1e-6 / t_full
    sample = (f"{n} SHB iterations ({args.warmup} warm-up, {args.steps} timed) of deconwolf's CPU method code "
              f"({impl} build, FFTW replaced by the oracle FFT, {os.cpu_count()} threads) on a "
              f"{crop}x{crop}x{P} crop with the full {psf.shape[2]}x{psf.shape[1]}x{psf.shape[0]} PSF "
              f"(job {crop + psf.shape[2] - 1}x{crop + psf.shape[1] - 1}x{P + psf.shape[0] - 1}); "
              f"{per_it:.3f} s/iteration scaled per job voxel to the full job")
    line = {
        "impl": "reference", "metric": "Mvoxel*iter/s (SHB, %s)" % args.workload.split("-", 1)[1],
        "value": value, "unit": "Mvoxel*iter/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_full * ITERS * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded Poisson image, Born-Wolf PSF)",
        "config": {"workload": args.workload, "image": [M, N, P], "psf": list(psf.shape[::-1]), "method": "shb",
                   "iterations_per_step": ITERS, "crop": [crop, crop, P]},
        "cpu_baseline": {"value": value, "unit": "Mvoxel*iter/s", "cores": os.cpu_count(),
                         "kind": "reference" if impl == "reference" else "port", "sample": sample},
        "e2e": {"value": value, "unit": "Mvoxel*iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- batched / served workloads
#
# Each prints one JSON line: the batched (or served) throughput as `value`,
# the plain one-job-at-a-time GPU path on the same inputs as `sequential`.
# Wall-clock timing around host-buffer calls (uploads and downloads inside).

def _common_line(metric, value, args, config, extra):
    line = {"metric": metric, "value": value, "unit": "Mvoxel*iter/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded Poisson images, Born-Wolf PSFs)", "config": config}
    line.update(extra)
    return line


_PINNED = []


def _pinned(a=None, shape=None):
    """A numpy view of page-locked host memory: a copy of ``a``, or an
    uninitialised float32 array of ``shape`` (the host buffers of the
    end-to-end measurements)."""
    import torch
    t = (torch.from_numpy(np.ascontiguousarray(a)).pin_memory() if a is not None
         else torch.empty(shape, dtype=torch.float32, pin_memory=True))
    _PINNED.append(t)
    return t.numpy()


def run_tiles(args):
    import deconwolf_b200 as dw
    from deconwolf_b200 import synthetic
    t0 = time.time()
    im, psf = synthetic.tiled_inputs(CACHE)
    log(f"inputs {im.shape} in {time.time() - t0:.1f}s")
    pp = dw.psf_prepare(psf, im.shape)
    tiles = dw.tiling_create(im.shape, args.tilesize, 50)
    im = _pinned(im)
    outs = {0.0: _pinned(shape=im.shape), 1.0: _pinned(shape=im.shape)}

    def step(budget=0.0):
        return dw.deconvolve_tiled(im, pp, args.tilesize, 50, method="shb", n_iter=ITERS, hbm_budget=budget,
                                   out=outs[budget])

    for _ in range(args.warmup):
        step()
    t = time.perf_counter()
    for _ in range(args.steps):
        res = step()
    dt = (time.perf_counter() - t) / args.steps
    t = time.perf_counter()
    seq = step(1.0)  # one tile per batch: the tiles one after another
    dt_seq = time.perf_counter() - t
    vox_it = float(im.size) * ITERS
    P, N, M = im.shape
    print(json.dumps(_common_line(
        f"Mvoxel*iter/s (SHB, tiled {M}x{N}x{P})", vox_it / dt / 1e6, args,
        {"workload": "tiles-4096x4096x60", "image": [M, N, P], "psf": list(psf.shape[::-1]),
         "tilesize": args.tilesize, "overlap": 50, "tiles": len(tiles), "iterations": ITERS, "method": "shb",
         "host_buffers": "page-locked image and result"},
        {"ms_per_step": dt * 1e3,
         "sequential": {"value": vox_it / dt_seq / 1e6, "ms_per_step": dt_seq * 1e3,
                        "how": "dwcu_deconvolve_tiled with one tile per batch"},
         "batched_equals_sequential": bool(np.array_equal(res.out, seq.out))})), flush=True)
    return 0


def run_channels(args):
    import deconwolf_b200 as dw
    from deconwolf_b200 import synthetic
    t0 = time.time()
    chans = []
    for c in range(6):
        im, psf = synthetic.channel_inputs(c, CACHE)
        sp = synthetic.channel_spec(c)
        chans.append((_pinned(im), dw.psf_prepare(psf, im.shape), sp["iters"]))
    log(f"6 channels in {time.time() - t0:.1f}s: " + ", ".join(str(c[0].shape) for c in chans))
    outs_b = [_pinned(shape=c[0].shape) for c in chans]
    outs_s = [_pinned(shape=c[0].shape) for c in chans]

    def batched():
        jobs = []
        for im, p, it in chans:
            j = dw.Job(im.shape, p.shape, method="shb", n_iter=it)
            j.setup(im, p)
            jobs.append(j)
        dw.batch_run(jobs)
        outs = [j.result(out=o) for j, o in zip(jobs, outs_b)]
        for j in jobs:
            j.close()
        return outs

    def sequential():
        return [dw.run_method(im, p, out=o, method="shb", n_iter=it) for (im, p, it), o in zip(chans, outs_s)]

    for _ in range(args.warmup):
        batched()
    t = time.perf_counter()
    for _ in range(args.steps):
        outs = batched()
    dt = (time.perf_counter() - t) / args.steps
    sequential()
    t = time.perf_counter()
    souts = sequential()
    dt_seq = time.perf_counter() - t
    vox_it = float(sum(im.size * it for im, _, it in chans))
    same = all(np.array_equal(a.out, b.out) for a, b in zip(outs, souts))
    print(json.dumps(_common_line(
        "Mvoxel*iter/s (SHB, 6-channel field of view)", vox_it / dt / 1e6, args,
        {"workload": "channels-6", "channels": [{"image": list(im.shape[::-1]), "psf": list(p.shape[::-1]),
                                                 "iterations": it} for im, p, it in chans], "method": "shb",
         "host_buffers": "page-locked images and results"},
        {"ms_per_step": dt * 1e3,
         "sequential": {"value": vox_it / dt_seq / 1e6, "ms_per_step": dt_seq * 1e3,
                        "how": "dwcu_deconvolve per channel, one after another"},
         "batched_equals_sequential": bool(same)})), flush=True)
    return 0


# jobs per size class of the serving stream (a few seconds of GPU work each)
CLASS_JOBS = (24, 12, 4, 2)


def run_classes(args):
    """Plain vs batched per size class of the serving stream: for each image
    size, CLASS_JOBS jobs of 50 SHB iterations (two seeded images of the
    class alternating, the 525 nm PSF of the class), run one at a time through
    dwcu_deconvolve and as one dwcu_batch_run; page-locked host buffers,
    uploads and downloads inside the timed region, wall clock."""
    import deconwolf_b200 as dw
    from deconwolf_b200 import synthetic
    classes = []
    for size, njobs in enumerate(CLASS_JOBS):
        if args.classes and size not in args.classes:
            continue
        ims = [_pinned(synthetic.serve_image(size, v, CACHE)[0]) for v in range(2)]
        psf = dw.psf_prepare(synthetic.serve_psf(size, 525.0, CACHE), ims[0].shape)
        jobs_in = [ims[i % 2] for i in range(njobs)]
        outs_b = [_pinned(shape=ims[0].shape) for _ in range(njobs)]
        outs_s = [_pinned(shape=ims[0].shape) for _ in range(njobs)]

        def batched():
            jobs = []
            for im in jobs_in:
                j = dw.Job(im.shape, psf.shape, method="shb", n_iter=ITERS)
                j.setup(im, psf)
                jobs.append(j)
            dw.batch_run(jobs)
            res = [j.result(out=o) for j, o in zip(jobs, outs_b)]
            for j in jobs:
                j.close()
            return res

        def sequential():
            return [dw.run_method(im, psf, out=o, method="shb", n_iter=ITERS) for im, o in zip(jobs_in, outs_s)]

        for _ in range(args.warmup):
            batched()
            sequential()
        t = time.perf_counter()
        for _ in range(args.steps):
            rb = batched()
        dt_b = (time.perf_counter() - t) / args.steps
        t = time.perf_counter()
        for _ in range(args.steps):
            rs = sequential()
        dt_s = (time.perf_counter() - t) / args.steps
        vox_it = float(ims[0].size) * ITERS * njobs
        work = dw.plan_size(ims[0].shape, psf.shape)[0]
        same = all(np.array_equal(a.out, b.out) for a, b in zip(rb, rs))
        classes.append({"image": list(ims[0].shape[::-1]), "job": list(work), "psf": list(psf.shape[::-1]),
                        "jobs": njobs, "batched": vox_it / dt_b / 1e6, "sequential": vox_it / dt_s / 1e6,
                        "ratio": dt_s / dt_b, "batched_ms": dt_b * 1e3, "sequential_ms": dt_s * 1e3,
                        "batched_equals_sequential": bool(same)})
        log(f"class {size}: {classes[-1]}")
    tot_b = sum(c["batched_ms"] for c in classes)
    tot_s = sum(c["sequential_ms"] for c in classes)
    vox = sum(c["batched"] * c["batched_ms"] for c in classes)
    print(json.dumps(_common_line(
        "Mvoxel*iter/s (SHB 50 it, batches of one size class)", vox / tot_b, args,
        {"workload": "batch-classes", "method": "shb", "iterations": ITERS,
         "host_buffers": "page-locked images and results"},
        {"ms_per_step": tot_b, "classes": classes,
         "sequential": {"value": vox / tot_s, "ms_per_step": tot_s,
                        "how": "dwcu_deconvolve per job, one after another"}})), flush=True)
    return 0


def _fingerprint(a):
    """(xor, sum) of a float32 volume's bit patterns: equal volumes give equal
    fingerprints; a difference in any voxel changes them."""
    u = np.ascontiguousarray(a).view(np.uint32).reshape(-1)
    return int(np.bitwise_xor.reduce(u)), int(u.sum(dtype=np.uint64))


def run_serve(args):
    import deconwolf_b200 as dw
    from deconwolf_b200 import synthetic
    t0 = time.time()
    reqs = synthetic.serve_requests(args.requests)
    pool = {}
    psfs = {}
    for i, r in enumerate(reqs):
        key = (r["size"], i % 2)
        if key not in pool:
            pool[key] = synthetic.serve_image(*key, cache_dir=CACHE)[0]
        r["image"] = key
        if (r["size"], r["lam"]) not in psfs:
            psfs[(r["size"], r["lam"])] = synthetic.serve_psf(r["size"], r["lam"], CACHE)
    log(f"{len(reqs)} requests, {len(pool)} images, {len(psfs)} PSFs in {time.time() - t0:.1f}s")

    def inputs(r):
        return pool[r["image"]], psfs[(r["size"], r["lam"])]

    # served: a submitter thread replays the arrivals
    sv = dw.Server(hbm_budget=args.hbm_budget, max_active=8, iters_per_turn=8)
    ids = [None] * len(reqs)
    start = time.perf_counter()

    def submitter():
        for i, r in enumerate(reqs):
            delay = start + r["arrival"] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            im, psf = inputs(r)
            ids[i] = sv.submit(im, psf, method=r["method"], n_iter=r["iters"])

    # results are reduced to a fingerprint of their bits as they arrive (the
    # stream's results together would not fit in host memory)
    served = [None] * len(reqs)

    def waiter():
        for i in range(len(reqs)):
            while ids[i] is None:
                time.sleep(0.001)
            served[i] = _fingerprint(sv.wait(ids[i]).out)

    th = threading.Thread(target=submitter)
    tw = threading.Thread(target=waiter)
    th.start()
    tw.start()
    th.join()
    tw.join()
    st = sv.stats()
    sv.close()
    vox_it = float(sum(pool[r["image"]].size * r["iters"] for r in reqs))
    # sequential: one request at a time, each starting at its arrival or when
    # the previous ends; the clock stops while a result is fingerprinted
    lat = []
    start = time.perf_counter()
    seq = []
    for r in reqs:
        delay = start + r["arrival"] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        im, psf = inputs(r)
        res = dw.run_method(im, psf, method=r["method"], n_iter=r["iters"])
        lat.append(time.perf_counter() - (start + r["arrival"]))
        t_fp = time.perf_counter()
        seq.append(_fingerprint(res.out))
        del res
        start += time.perf_counter() - t_fp
    wall_seq = time.perf_counter() - start
    lat = np.sort(np.array(lat))
    same = sum(int(a == b) for a, b in zip(served, seq))
    sizes = [list(s[::-1]) for s in synthetic.SERVE_SIZES]
    print(json.dumps(_common_line(
        "Mvoxel*iter/s (SHB/RL serving stream)", st["voxel_iterations"] / st["wall_s"] / 1e6, args,
        {"workload": "serve-stream", "requests": len(reqs), "arrival_rate_per_s": 2.0, "sizes": sizes,
         "psf": "181x181x(2P-1) Born-Wolf at the request's wavelength", "iterations": "uniform 20-200",
         "methods": "SHB/RL 50/50", "hbm_budget_bytes": args.hbm_budget, "max_active": 8, "iters_per_turn": 8},
        {"latency_p50_s": st["latency_p50_s"], "latency_p99_s": st["latency_p99_s"],
         "latency_mean_s": st["latency_mean_s"], "wall_s": st["wall_s"],
         "sequential": {"value": vox_it / wall_seq / 1e6, "wall_s": wall_seq,
                        "latency_p50_s": float(lat[int(np.ceil(0.5 * len(lat))) - 1]),
                        "latency_p99_s": float(lat[int(np.ceil(0.99 * len(lat))) - 1]),
                        "how": "dwcu_deconvolve per request in arrival order"},
         "served_equals_sequential": f"{same}/{len(reqs)}"})), flush=True)
    return 0


# ---------------------------------------------------------------- B200 arm

def run_split(args):
    """One 2048 x 2048 x 60 image split into --parts slabs of z planes
    (dwcu_deconvolve_slabs), parts dealt round-robin over the visible GPUs,
    beside the whole job on one GPU (dwcu_deconvolve).  With one GPU every
    part shares it, and the difference is the cost of the split itself (the
    column transposes run as copies within one GPU's memory)."""
    import torch
    import deconwolf_b200 as dw
    from deconwolf_b200 import synthetic
    im, psf = synthetic.config_inputs(WORKLOAD, CACHE)
    ngpu = max(1, torch.cuda.device_count())
    parts = args.parts
    devices = [p % ngpu for p in range(parts)]
    im = _pinned(im)
    outs = [_pinned(shape=im.shape), _pinned(shape=im.shape)]

    def split():
        return dw.run_slabs(im, psf, parts=parts, devices=devices, method="shb", n_iter=ITERS, out=outs[0])

    def whole():
        return dw.run_method(im, psf, method="shb", n_iter=ITERS, out=outs[1])

    for _ in range(args.warmup):
        split()
    t = time.perf_counter()
    loop = []
    for _ in range(args.steps):
        res = split()
        loop.append(res.seconds_iterate)
    dt = (time.perf_counter() - t) / args.steps
    whole()
    t = time.perf_counter()
    ref = whole()
    dt_whole = time.perf_counter() - t
    vox_it = float(im.size) * ITERS
    P, N, M = im.shape
    lay = [dw.slab_layout(im.shape, psf.shape, parts, p) for p in range(parts)]
    print(json.dumps(_common_line(
        f"Mvoxel*iter/s (SHB, {M}x{N}x{P} split into {parts} parts)", vox_it / dt / 1e6, args,
        {"workload": "split-2048x2048x60", "image": [M, N, P], "psf": list(psf.shape[::-1]), "parts": parts,
         "devices": devices, "iterations": ITERS, "method": "shb",
         "exchange": "gathered copies" if os.environ.get("DWCU_SLAB_TRANSPOSE") == "copy" else "in place (plane table)",
         "planes_per_part": [q["planes"] for q in lay], "columns_per_part": [q["cols"] for q in lay],
         "host_buffers": "page-locked image and result"},
        {"n_gpus": len(set(devices)), "ms_per_step": dt * 1e3,
         "loop_ms": statistics.median(loop) * 1e3,
         "whole_job": {"value": vox_it / dt_whole / 1e6, "ms_per_step": dt_whole * 1e3,
                       "loop_ms": ref.seconds_iterate * 1e3, "how": "dwcu_deconvolve on GPU 0"},
         "rel_l2_vs_whole": float(np.linalg.norm(res.out.astype(np.float64) - ref.out)
                                  / np.linalg.norm(ref.out.astype(np.float64))),
         "iterations_equal": bool(res.iterations == ref.iterations)})), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=WORKLOAD,
                    choices=[WORKLOAD, SMALL, PROFILE_CASE, "shb-2048x256x20", "shb-256x2048x20", "shb-256x256x60",
                             "shb-1124x1124x60",
                             "tiles-4096x4096x60", "channels-6", "serve-stream", "batch-classes",
                             "split-2048x2048x60"])
    ap.add_argument("--parts", type=int, default=2, help="split-2048x2048x60: slabs of z planes")
    ap.add_argument("--tilesize", type=int, default=1024)
    ap.add_argument("--requests", type=int, default=60, help="serve-stream: number of requests (full stream: 500)")
    ap.add_argument("--hbm-budget", type=float, default=160e9, help="serve-stream: device bytes for admitted jobs")
    ap.add_argument("--classes", type=int, nargs="*", default=None,
                    help="batch-classes: size classes to run (default: all four)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warmup raised to 3 (timing rule)")
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "tiles-4096x4096x60":
        return run_tiles(args)
    if args.workload == "channels-6":
        return run_channels(args)
    if args.workload == "serve-stream":
        return run_serve(args)
    if args.workload == "batch-classes":
        return run_classes(args)
    if args.workload == "split-2048x2048x60":
        return run_split(args)

    import torch
    import torch.distributed as dist
    import deconwolf_b200 as dw
    from deconwolf_b200 import synthetic

    world, rank, local = dist_setup()
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = local

    t0 = time.time()
    im, psf = synthetic.config_inputs(args.workload, CACHE)
    log(f"[rank {rank}] inputs {im.shape} psf {psf.shape} in {time.time() - t0:.1f}s")
    P, N, M = im.shape
    work, nbytes = dw.plan_size(im.shape, psf.shape)

    d_im = torch.from_numpy(im).to(f"cuda:{dev}")
    d_psf = torch.from_numpy(psf).to(f"cuda:{dev}")
    d_out = torch.empty_like(d_im)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize()

    def step():
        return dw.run_method_device(d_im.data_ptr(), d_psf.data_ptr(), d_out.data_ptr(), im.shape, psf.shape,
                                    stream=stream.cuda_stream, method="shb", n_iter=ITERS, device=dev)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(dev)
    clocks.start()
    launches0 = int(dw.lib().dwcu_launch_count())
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    # the production path: each step's iteration loop replays one cached CUDA
    # graph; the steps run back to back and are read at the end
    ev0.record(stream)
    for _ in range(args.steps):
        res = step()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = int(dw.lib().dwcu_launch_count()) - launches0
    if world > 1:
        dist.barrier()
    # per-kernel timing (kernel table and roofline only): the same steps
    # again with CUDA events between the kernels, launched eagerly
    dw.profile_enable(True)
    torch.cuda.synchronize()
    e2a = torch.cuda.Event(enable_timing=True)
    e2b = torch.cuda.Event(enable_timing=True)
    e2a.record(stream)
    for _ in range(args.steps):
        step()
    e2b.record(stream)
    torch.cuda.synchronize()
    ms_prof = e2a.elapsed_time(e2b)
    dw.profile_enable(False)
    stats = dw.profile_collect()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    t_max = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{dev}")
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms_max = float(t_max.item())
    vox_it = float(im.size) * ITERS * args.steps * world
    value = vox_it / (ms_max * 1e-3) / 1e6

    # ---- end to end through the host-buffer C-ABI call
    e2e = None
    if not args.no_e2e:
        h_im = torch.from_numpy(im).pin_memory()
        h_psf = torch.from_numpy(psf).pin_memory()
        h_out = torch.empty(im.shape, dtype=torch.float32).pin_memory()
        o = dw.make_opts(method="shb", n_iter=ITERS, device=dev)

        def e2e_step():
            rc = dw.lib().dwcu_deconvolve(ctypes.c_void_p(h_im.data_ptr()), M, N, P, ctypes.c_void_p(h_psf.data_ptr()),
                                          psf.shape[2], psf.shape[1], psf.shape[0], ctypes.byref(o),
                                          ctypes.c_void_p(h_out.data_ptr()))
            if rc:
                raise dw.DwcuError(rc, dw.lib().dwcu_last_error().decode())

        e2e_step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        cur = torch.cuda.current_stream()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(cur)
        for _ in range(args.steps):
            e2e_step()
        e1.record(cur)
        torch.cuda.synchronize()
        t_e2e = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=f"cuda:{dev}")
        if world > 1:
            dist.all_reduce(t_e2e, op=dist.ReduceOp.MAX)
        e2e = {"value": vox_it / (float(t_e2e.item()) * 1e-3) / 1e6, "unit": "Mvoxel*iter/s",
               "h2d_bytes_per_step": int(im.nbytes + psf.nbytes), "d2h_bytes_per_step": int(im.nbytes)}

    # ---- roofline of the dominant kernel class
    peak, peak_kind = measured_peaks()
    dom = max(stats, key=lambda s: s["ms"]) if stats else None
    roof = None
    if dom:
        avg_s = dom["ms"] / dom["launches"] * 1e-3
        achieved = dom["bytes_per_launch"] / avg_s / 1e9
        roof = {"bound": "hbm", "kernel": dom["name"], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                "algorithmic_bytes_per_launch": dom["bytes_per_launch"], "avg_launch_ms": avg_s * 1e3}
        # ncu DRAM bytes per launch of this kernel class on the capture case,
        # scaled to this launch by the algorithmic bytes (units processed)
        prof_path = os.path.join(ROOT, "profiles", "kernel_traffic.json")
        if os.path.exists(prof_path):
            with open(prof_path) as f:
                tr = json.load(f)
            k = tr["kernels"].get(dom["name"])
            if k:
                roof["traffic"] = k["traffic_over_algorithmic"] * dom["bytes_per_launch"]
                roof["traffic_source"] = (f"ncu dram__bytes_read.sum + dram__bytes_write.sum on "
                                          f"{k.get('workload', tr['capture']['workload'])} "
                                          f"({k['dram_bytes_per_launch']:.4g} B per launch), scaled by algorithmic bytes")
    kernels = sorted(
        ({"name": s["name"], "launches": s["launches"], "ms": round(s["ms"], 3),
          "bytes_per_launch": s["bytes_per_launch"],
          "GBps": round(s["bytes_per_launch"] * s["launches"] / (s["ms"] * 1e-3) / 1e9, 1)} for s in stats),
        key=lambda d: -d["ms"])
    total_k = sum(s["ms"] for s in stats) or 1.0

    line = {
        "metric": "Mvoxel*iter/s (SHB, %s)" % args.workload.split("-", 1)[1],
        "value": value, "unit": "Mvoxel*iter/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded Poisson image, Born-Wolf PSF)",
        "config": {"workload": args.workload, "image": [M, N, P], "psf": list(psf.shape[::-1]), "method": "shb",
                   "iterations_per_step": ITERS, "job": list(work), "device_bytes_per_job": nbytes,
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (~18 GB working set per step)"},
        "roofline": roof,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
        "kernels": kernels[:8],
        "kernel_share": {k["name"]: round(k["ms"] / total_k, 3) for k in kernels[:8]},
        "iteration_ms": (ms_max / args.steps - res.seconds_setup * 1e3) / ITERS if res else None,
        "diagnostics": {"ms_per_step_with_kernel_events": ms_prof / args.steps,
                        "setup_ms": res.seconds_setup * 1e3, "iterate_ms": res.seconds_iterate * 1e3,
                        "host_enqueue_ms": res.seconds_enqueue * 1e3,
                        "kernel_ms_per_step": total_k / args.steps},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline_entry(im, psf)
        except Exception as e:  # the checker build may be absent on a foreign machine
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
