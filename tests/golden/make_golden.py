"""Make the golden fixtures of the parity tests from the reference build.

Every fixture here is produced by deconwolf's own method code (method_shb.c,
method_rl.c, fft.c, fim.c compiled unmodified into oracle/_ref, see
oracle/Makefile) on seeded synthetic inputs.  Run in a checkout that has the
reference sources available to oracle/Makefile:

    make -C oracle && python tests/golden/make_golden.py [--config1]

Small fixtures store inputs and full outputs.  The 256 x 256 x 40 fixture
(--config1, a few minutes of CPU) stores the I-divergence trace, per-plane
sums and a seeded sample of 65536 output voxels; the inputs are regenerated
from their seeds by deconwolf_b200.synthetic.

--config1-fp64 (a few minutes) runs the same 256 x 256 x 40 job through the
reference build and through the FP64 restatement (oracle/fp64.py) and stores
the FP64 result at the same sampled voxels, its trace, norm and sketch
(tests/helpers.sketch), the reference output's sketch and the reference's
exact relative L2 distance to the FP64 result.

--config2 (one to two hours on 8 cores, ~20 GB of RAM) runs the reference's
SHB for 50 iterations on the 2048 x 2048 x 60 workload and stores its trace,
plane sums, norm, 262144 sampled voxels and a sketch of the whole output.
--tile1024 and --tile512 do the same for one tile of the tiled 4096 x 4096 x
60 workload at tile size 1024 (1124 x 1124 x 60) and 512 (612 x 562 x 60),
with the full PSF.

--tile512-rl is the 612 x 562 x 60 tile with RL instead of SHB.

--tiled-pair runs the reference's tiled path (tiling.c, per-tile PSF crop,
weighted blend) on a 2048 x 1024 x 60 image at tile size 1024 (two tiles).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402
from tests.helpers import gauss_psf, poisson_image  # noqa: E402


def small(name, shape, psf_shape, seed, **opts):
    psf = gauss_psf(psf_shape, (1.3, 1.6, 1.9), seed=seed, jitter=0.15)
    im = poisson_image(shape, psf, seed=seed, bg=80.0, npts=25)
    r = po.deconvolve(im, psf, impl="reference", threads=os.cpu_count(), **opts)
    out = {"image": im, "psf": psf, "out": r.out, "trace": r.trace, "iterations": np.int64(r.iterations),
           "bg": np.float32(r.bg)}
    for k, v in opts.items():
        out["opt_" + k] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, r.iterations, r.trace[:3])


def sample_index(shape, n, seed=12345):
    rng = np.random.default_rng(seed)
    return rng.choice(int(np.prod(shape)), size=n, replace=False)


def config1():
    from deconwolf_b200 import synthetic
    name = "shb-256x256x40"
    im, psf = synthetic.config_inputs(name)
    t = time.time()
    r = po.deconvolve(im, psf, method="shb", n_iter=50, impl="reference", threads=os.cpu_count())
    print("reference SHB 256x256x40, 50 it:", time.time() - t, "s; loop", r.loop_seconds)
    idx = sample_index(im.shape, 65536)
    np.savez_compressed(
        os.path.join(HERE, "config1_shb50.npz"),
        trace=r.trace, plane_sums=r.out.astype(np.float64).sum(axis=(1, 2)), sample_idx=idx,
        sample_val=r.out.reshape(-1)[idx], norm=np.float64(np.linalg.norm(r.out.astype(np.float64))),
        image_sum=np.float64(im.astype(np.float64).sum()), psf_sum=np.float64(psf.astype(np.float64).sum()),
        image_sample=im.reshape(-1)[idx], bg=np.float32(r.bg), loop_seconds=np.float64(r.loop_seconds),
        threads=np.int64(os.cpu_count()))


def config1_fp64():
    from deconwolf_b200 import synthetic
    from oracle.fp64 import deconvolve_fp64
    from tests.helpers import sketch
    name = "shb-256x256x40"
    im, psf = synthetic.config_inputs(name)
    r = po.deconvolve(im, psf, method="shb", n_iter=50, impl="reference", threads=os.cpu_count())
    t = time.time()
    f = deconvolve_fp64(im, psf, method="shb", n_iter=50)
    print("FP64 SHB 256x256x40, 50 it:", time.time() - t, "s")
    idx = sample_index(im.shape, 65536)
    ref = r.out.astype(np.float64)
    np.savez_compressed(
        os.path.join(HERE, "config1_fp64.npz"),
        sample_idx=idx, fp64_sample=f.out.reshape(-1)[idx], fp64_trace=f.trace,
        fp64_norm=np.float64(np.linalg.norm(f.out)), fp64_sketch=sketch(f.out), ref_sketch=sketch(ref),
        ref_norm=np.float64(np.linalg.norm(ref)),
        ref_rel_l2_fp64=np.float64(np.linalg.norm(ref - f.out) / np.linalg.norm(f.out)),
        ref_trace_rel_fp64=np.float64(np.max(np.abs(r.trace - f.trace) / f.trace)))
    print("reference vs FP64: rel L2", np.linalg.norm(ref - f.out) / np.linalg.norm(f.out))


def config2():
    from deconwolf_b200 import synthetic
    from tests.helpers import sketch
    name = "shb-2048x2048x60"
    t = time.time()
    im, psf = synthetic.config_inputs(name)
    print("inputs", time.time() - t, "s", flush=True)
    t = time.time()
    r = po.deconvolve(im, psf, method="shb", n_iter=50, impl="reference", threads=os.cpu_count())
    print("reference SHB 2048x2048x60, 50 it:", time.time() - t, "s; loop", r.loop_seconds, flush=True)
    idx = np.sort(sample_index(im.shape, 262144))
    out = r.out
    np.savez_compressed(
        os.path.join(HERE, "config2_shb50.npz"),
        trace=r.trace, plane_sums=out.astype(np.float64).sum(axis=(1, 2)), sample_idx=idx,
        sample_val=out.reshape(-1)[idx], norm=np.float64(np.linalg.norm(out.astype(np.float64))),
        sketch=sketch(out), image_sum=np.float64(im.astype(np.float64).sum()),
        psf_sum=np.float64(psf.astype(np.float64).sum()), image_sample=im.reshape(-1)[idx],
        bg=np.float32(r.bg), loop_seconds=np.float64(r.loop_seconds), threads=np.int64(os.cpu_count()))


def tile_golden(name, fixture, method="shb"):
    """A tile of the 4096 x 4096 x 60 image with the full 181 x 181 x 119 PSF,
    SHB 50 iterations: 1124 x 1124 x 60 (tile size 1024, overlap 50; job
    1304 x 1304 x 178, padded on the GPU to 1344 x 1344 x 180) or 612 x 562 x
    60 (tile size 512; job 792 x 742 x 178 -> 800 x 750 x 180)."""
    from deconwolf_b200 import synthetic
    from tests.helpers import sketch
    im, psf = synthetic.config_inputs(name)
    t = time.time()
    r = po.deconvolve(im, psf, method=method, n_iter=50, impl="reference", threads=os.cpu_count())
    print("reference", method, name, "50 it:", time.time() - t, "s", flush=True)
    idx = np.sort(sample_index(im.shape, 131072))
    out = r.out
    np.savez_compressed(
        os.path.join(HERE, fixture),
        trace=r.trace, plane_sums=out.astype(np.float64).sum(axis=(1, 2)), sample_idx=idx,
        sample_val=out.reshape(-1)[idx], norm=np.float64(np.linalg.norm(out.astype(np.float64))),
        sketch=sketch(out), image_sum=np.float64(im.astype(np.float64).sum()), image_sample=im.reshape(-1)[idx],
        bg=np.float32(r.bg), loop_seconds=np.float64(r.loop_seconds), threads=np.int64(os.cpu_count()))


def tiled_pair():
    """The reference's tiled path (deconvolve_tiles over tiling.c, each tile
    with its own PSF crop, weighted blend) on the 2048 x 1024 x 60 image at
    tile size 1024, overlap 50 (two tiles), SHB 50 iterations; the PSF
    prepared for the whole image as dw_run does."""
    from deconwolf_b200 import synthetic
    from tests.helpers import sketch
    im, psf = synthetic.tiled_pair_inputs()
    pp = po.psf_prepare_reference(psf, im.shape)
    t = time.time()
    r = po.deconvolve_tiled(im, pp, 1024, 50, method="shb", n_iter=50, impl="reference", threads=os.cpu_count())
    print("reference tiled SHB 2048x1024x60, 50 it:", time.time() - t, "s", flush=True)
    idx = np.sort(sample_index(im.shape, 131072))
    out = r.out
    np.savez_compressed(
        os.path.join(HERE, "tiled2_shb50.npz"),
        plane_sums=out.astype(np.float64).sum(axis=(1, 2)), sample_idx=idx, sample_val=out.reshape(-1)[idx],
        norm=np.float64(np.linalg.norm(out.astype(np.float64))), sketch=sketch(out),
        image_sample=im.reshape(-1)[idx], psf_shape=np.array(pp.shape), threads=np.int64(os.cpu_count()))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config1", action="store_true")
    ap.add_argument("--config1-fp64", action="store_true")
    ap.add_argument("--config2", action="store_true")
    ap.add_argument("--tile1024", action="store_true")
    ap.add_argument("--tile512", action="store_true")
    ap.add_argument("--tiled-pair", action="store_true")
    ap.add_argument("--tile512-rl", action="store_true")
    ap.add_argument("--no-small", action="store_true")
    a = ap.parse_args()
    if not a.no_small:
        small("small_shb", (11, 40, 37), (7, 9, 11), seed=11, method="shb", n_iter=20)
        small("small_rl", (11, 40, 37), (7, 9, 11), seed=12, method="rl", n_iter=20)
        small("small_shb_rel", (8, 33, 30), (5, 9, 9), seed=13, method="shb", iter_type=po.ITER_REL,
              err_rel=0.001)
    if a.config1:
        config1()
    if a.config1_fp64:
        config1_fp64()
    if a.config2:
        config2()
    if a.tile1024:
        tile_golden("shb-1124x1124x60", "tile1024_shb50.npz")
    if a.tile512:
        tile_golden("shb-612x562x60", "tile512_shb50.npz")
    if a.tiled_pair:
        tiled_pair()
    if a.tile512_rl:
        tile_golden("shb-612x562x60", "tile512_rl50.npz", method="rl")


if __name__ == "__main__":
    main()
