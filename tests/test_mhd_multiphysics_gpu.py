"""The MHD multiphysics two-material model on the device (VG_MODEL_MHD_MULTIPHYSICS, 1D): the exact FP64 form against
the golden fixtures made by the reference (its own MHDSecondOrderSolver::solve to t_end on the Dumbser multimaterial
layout, and its per-step functions on a perturbed layout with non-zero hyperbolic wave speeds) and against the oracle
(pinned in test_mhd_multiphysics.py), with every limiter and the first-order loop; the CFL maximum wave speed;
argument checks.

The model scales each material's field by pow(alpha_k, 1/2) and forms the interface field as pow(alpha1 B1^2 + alpha2
B2^2, 1/2); CUDA's pow and glibc's may differ in the last place, so runs are compared plane by plane: the largest
difference within 1e-12 of the plane's largest magnitude.  The CFL maximum takes no pow and is compared bit for bit."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "mhdmultiphysics*.npz")))
PRM = wl.mhd_multiphysics_params(1.4, 0.1, 1.67, 0.0, 0.5, 0.7)
REL = 1e-12


def _matches(a, b):
    assert np.isfinite(a).all()
    d = np.abs(a - b).reshape(b.shape[0], -1).max(axis=1)
    scale = np.maximum(np.abs(b).reshape(b.shape[0], -1).max(axis=1), 1e-300)
    assert (d / scale).max() <= REL, f"max normwise diff {(d / scale).max():.3e} (plane {int(np.argmax(d / scale))})"


def _device(gpu, W, prm, dx, **run):
    with gpu.Solver(gpu.MHD_MULTIPHYSICS, W.shape[-1], 1, prm) as s:
        s.upload(W)
        t, n = s.run(dx, 0.8, **run)
        return s.download(), t, n


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_mhd_multiphysics_golden(gpu, path):
    z = np.load(path)
    steps = int(z["steps"])
    t_end = float(z["t_end"]) if "t_end" in z.files else 0.0
    out, t, n = _device(gpu, z["w0"], z["params"], float(z["dx"]), steps=steps, t_end=t_end, limiter=int(z["limiter"]))
    if steps:
        assert n == steps
    else:
        assert t == t_end
    _matches(out, z["out"])


@pytest.mark.parametrize("limiter", [0, 1, 2])
@pytest.mark.parametrize("prm", [wl.mhd_multiphysics_params(2.0, 0.0, 2.0, 0.0), PRM], ids=["one", "two_glm"])
def test_mhd_multiphysics_matches_oracle(gpu, oracle_lib, limiter, prm):
    W = wl.mhd_multiphysics_dumbser_1d(64, seed=4, noise=1e-2)
    ref = W.copy()
    O.run_two_material(O.MHD_MULTIPHYSICS, ref, 1 / 64, 0.8, steps=25, limiter=limiter, bias=0.1, params=prm)
    out, _, n = _device(gpu, W, prm, 1 / 64, steps=25, limiter=limiter, bias=0.1)
    assert n == 25
    _matches(out, ref)


def test_mhd_multiphysics_time_driven_ignores_source_and_reinit(gpu, oracle_lib):
    # the reference's loop takes subcyclingIterations and reinitialisationFrequency and uses neither
    W = wl.mhd_multiphysics_dumbser_1d(72, seed=5, noise=1e-2)
    ref = W.copy()
    t_ref, n_ref = O.run_two_material(O.MHD_MULTIPHYSICS, ref, 1 / 72, 0.8, t_end=0.04, limiter=0, params=PRM)
    out, t, n = _device(gpu, W, PRM, 1 / 72, t_end=0.04, limiter=0, subcycles=2, reinit=3)
    assert t == t_ref and n == n_ref
    _matches(out, ref)


def test_mhd_multiphysics_first_order(gpu, oracle_lib):
    W = wl.mhd_multiphysics_dumbser_1d(50, seed=8, noise=1e-2)
    ref = W.copy()
    O.run_first_order(O.MHD_MULTIPHYSICS, ref, 1 / 50, 0.8, steps=12, params=PRM)
    out, _, _ = _device(gpu, W, PRM, 1 / 50, steps=12, order=1)
    _matches(out, ref)


def test_mhd_multiphysics_max_wave_speed(gpu, oracle_lib):
    W = wl.mhd_multiphysics_dumbser_1d(40, seed=9, noise=2e-2)
    with gpu.Solver(gpu.MHD_MULTIPHYSICS, 40, 1, PRM) as s:
        s.upload(W)
        got = s.max_wave_speed()
    assert got == O.max_wave(O.MHD_MULTIPHYSICS, W, PRM)


def test_mhd_multiphysics_argument_checks(gpu):
    with pytest.raises(gpu.VgError):
        gpu.Solver(gpu.MHD_MULTIPHYSICS, 16, 1, PRM, precision=gpu.MIXED)
    with pytest.raises(gpu.VgError):
        gpu.Solver(gpu.MHD_MULTIPHYSICS, 16, 8, PRM)  # 1D only, as the reference's model
