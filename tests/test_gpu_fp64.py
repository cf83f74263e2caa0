"""Each result's error against an FP64 run of the same iteration.

The FP64 restatement (oracle/fp64.py) runs the reference's SHB / RL
iteration with every value in float64; a float32 result's relative L2
distance to it is that result's own arithmetic error.  For the GPU output
and for the reference build's output the tests print both distances and
require the GPU's to be at most FP64_FACTOR times the reference's (with a
floor of FP64_FLOOR for cases where the reference's is tiny).

The reference build here replaces FFTW by the oracle's FFT, which works in
float64 internally and rounds once per transform, so its distance to FP64
is smaller than deconwolf's with float32 FFTW would be; the factor allows
for the GPU's float32 transforms (about log2(n) roundings per transform).
"""
import os

import numpy as np
import pytest

import deconwolf_b200 as dw
from oracle import pyoracle as po
from oracle.fp64 import deconvolve_fp64, deconvolve_fp64_torch
from tests.helpers import gauss_psf, poisson_image, rel_l2, sketch, sketch_rel_l2

pytestmark = pytest.mark.gpu

FP64_FACTOR = 4.0
FP64_FLOOR = 1e-6


def _impl():
    return "reference" if po.available("reference") else "port"


CASES = [
    (dict(method="shb", n_iter=20), (9, 22, 19), (5, 7, 9)),
    (dict(method="rl", n_iter=20), (9, 22, 19), (5, 7, 9)),
    (dict(method="shb", n_iter=50), (12, 40, 44), (7, 9, 11)),
    (dict(method="rl", n_iter=50), (12, 40, 44), (7, 9, 11)),
    (dict(method="shb", n_iter=15, border_quality=1), (9, 22, 20), (5, 7, 9)),
    (dict(method="shb", n_iter=15, border_quality=0), (20, 33, 44), (21, 15, 13)),
]


@pytest.mark.parametrize("case,shape,psf_shape", CASES,
                         ids=lambda v: "-".join(f"{k}={x}" for k, x in v.items()) if isinstance(v, dict) else None)
def test_error_against_fp64(case, shape, psf_shape):
    psf = gauss_psf(psf_shape, (1.2, 1.5, 1.7), seed=21, jitter=0.2)
    im = poisson_image(shape, psf, seed=21, bg=50.0, npts=15)
    g = dw.run_method(im, psf, **case)
    r = po.deconvolve(im, psf, impl=_impl(), **case)
    f = deconvolve_fp64(im, psf, method=case["method"], n_iter=case["n_iter"], bq=case.get("border_quality", 2))
    e_gpu, e_ref = rel_l2(g.out, f.out), rel_l2(r.out, f.out)
    t_gpu = float(np.max(np.abs(g.trace - f.trace) / f.trace))
    t_ref = float(np.max(np.abs(r.trace - f.trace) / f.trace))
    print(f"\nFP64 distance {case} {shape}: GPU {e_gpu:.3e} (trace {t_gpu:.2e}), "
          f"reference {e_ref:.3e} (trace {t_ref:.2e})")
    assert e_gpu <= FP64_FACTOR * max(e_ref, FP64_FLOOR)
    assert t_gpu <= FP64_FACTOR * max(t_ref, FP64_FLOOR)


def test_config1_error_against_fp64():
    """256 x 256 x 40, SHB 50: the GPU's distance to the FP64 run over the
    whole volume (sketch estimate) and on 65536 sampled voxels, beside the
    reference's exact distance stored with the fixture."""
    f = os.path.join(os.path.dirname(__file__), "golden", "config1_fp64.npz")
    if not os.path.exists(f):
        pytest.skip("config1 FP64 fixture not generated")
    from deconwolf_b200 import synthetic
    d = np.load(f)
    im, psf = synthetic.config_inputs("shb-256x256x40")
    g = dw.run_method(im, psf, method="shb", n_iter=50)
    idx = d["sample_idx"]
    e_gpu_sk = sketch_rel_l2(sketch(g.out), d["fp64_sketch"], float(d["fp64_norm"]))
    e_gpu_sm = rel_l2(g.out.reshape(-1)[idx], d["fp64_sample"])
    e_ref = float(d["ref_rel_l2_fp64"])
    t_gpu = float(np.max(np.abs(g.trace - d["fp64_trace"]) / d["fp64_trace"]))
    print(f"\nFP64 distance config 1: GPU {e_gpu_sk:.3e} (sketch), {e_gpu_sm:.3e} (samples), trace {t_gpu:.2e}; "
          f"reference {e_ref:.3e} (exact), trace {float(d['ref_trace_rel_fp64']):.2e}")
    assert e_gpu_sk <= FP64_FACTOR * max(e_ref, FP64_FLOOR)
    assert e_gpu_sm <= FP64_FACTOR * max(e_ref, FP64_FLOOR)
    assert t_gpu <= FP64_FACTOR * max(float(d["ref_trace_rel_fp64"]), FP64_FLOOR)


def test_config2_error_against_fp64():
    """2048 x 2048 x 60, SHB 50: the FP64 run of the same iteration on the GPU
    (torch float64, the same steps as the NumPy restatement), the GPU
    result's exact distance to it over the whole volume, and the reference's
    distance from its fixture (sketch and samples)."""
    f = os.path.join(os.path.dirname(__file__), "golden", "config2_shb50.npz")
    if not os.path.exists(f):
        pytest.skip("config2 fixture not generated")
    from deconwolf_b200 import synthetic
    d = np.load(f)
    im, psf = synthetic.config_inputs("shb-2048x2048x60")
    g = dw.run_method(im, psf, method="shb", n_iter=50)
    dw.release_cache()  # the engine's cached 19 GB block: the float64 run needs the room
    fr = deconvolve_fp64_torch(im, psf, method="shb", n_iter=50, device="cuda")
    import torch
    torch.cuda.empty_cache()
    e_gpu = rel_l2(g.out, fr.out)
    norm64 = float(np.linalg.norm(fr.out))
    e_ref_sk = sketch_rel_l2(d["sketch"], sketch(fr.out, device="cuda"), norm64)
    idx = d["sample_idx"]
    e_ref_sm = rel_l2(d["sample_val"], fr.out.reshape(-1)[idx])
    t_gpu = float(np.max(np.abs(g.trace - fr.trace) / fr.trace))
    t_ref = float(np.max(np.abs(d["trace"] - fr.trace) / fr.trace))
    print(f"\nFP64 distance config 2: GPU {e_gpu:.3e} (exact, whole volume), trace {t_gpu:.2e}; "
          f"reference {e_ref_sk:.3e} (sketch), {e_ref_sm:.3e} (samples), trace {t_ref:.2e}")
    assert e_gpu <= FP64_FACTOR * max(e_ref_sk, FP64_FLOOR)
    assert t_gpu <= FP64_FACTOR * max(t_ref, FP64_FLOOR)
