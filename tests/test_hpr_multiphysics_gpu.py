"""The HPR multiphysics two-material model on the device (VG_MODEL_HPR_MULTIPHYSICS, 1D): the exact FP64 form against
the golden fixtures made by the reference (its own HPRSecondOrderSolver::solve to t_end, and its per-step functions
with a cold material and the reinitialisation) and against the oracle (pinned in test_hpr_multiphysics.py), with every
limiter, thermal and cold materials, the reinitialisation and the first-order loop; the CFL maximum wave speed;
argument checks.

The model's conserved distortion is pow(alpha_k, 1/3) A_k, and CUDA's pow and glibc's may differ in the last place, so
the runs are compared plane by plane: the largest difference within 1e-12 of the plane's largest magnitude.  The CFL
maximum takes no pow and is compared bit for bit."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "hprmultiphysics*.npz")))
STIFF2 = dict(gamma2=2.0, p_inf2=0.5)
PRM = wl.hpr_reduced_params(**STIFF2)
REL = 1e-12
# solid materials take pow in their equations of state (the ShockMieGruneisen cold curve, the plastic relaxation)
REL_SOLID = 1e-10


def _matches(a, b, rel=REL):
    assert np.isfinite(a).all()
    d = np.abs(a - b).reshape(b.shape[0], -1).max(axis=1)
    scale = np.maximum(np.abs(b).reshape(b.shape[0], -1).max(axis=1), 1e-300)
    assert (d / scale).max() <= rel, f"max normwise diff {(d / scale).max():.3e} (plane {int(np.argmax(d / scale))})"


def _device(gpu, W, prm, dx, **run):
    with gpu.Solver(gpu.HPR_MULTIPHYSICS, W.shape[-1], 1, prm) as s:
        s.upload(W)
        t, n = s.run(dx, 0.8, **run)
        return s.download(), t, n


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_hpr_multiphysics_golden(gpu, path):
    z = np.load(path)
    steps = int(z["steps"])
    t_end = float(z["t_end"]) if "t_end" in z.files else 0.0
    out, t, n = _device(gpu, z["w0"], z["params"], float(z["dx"]), steps=steps, t_end=t_end,
                        limiter=int(z["limiter"]), reinit=int(z["reinit"]), subcycles=int(z["subcycles"]))
    if steps:
        assert n == steps
    else:
        assert t == t_end
    solid = z["params"][12] != 0.0 or z["params"][32] != 0.0
    _matches(out, z["out"], rel=REL_SOLID if solid else REL)


@pytest.mark.parametrize("thermal", [(True, True), (True, False), (False, True), (False, False)],
                         ids=["hot", "cold2", "cold1", "cold"])
@pytest.mark.parametrize("limiter", [0, 1, 2])
def test_hpr_multiphysics_matches_oracle(gpu, oracle_lib, limiter, thermal):
    W = wl.hpr_multiphysics_riemann(64, seed=3, p2_scale=1.1, a2_scale=1.01)
    prm = wl.hpr_reduced_params(thermal=thermal, **STIFF2)
    ref = W.copy()
    O.run_two_material(O.HPR_MULTIPHYSICS, ref, 1 / 64, 0.8, steps=10, limiter=limiter, bias=0.1, params=prm)
    out, _, n = _device(gpu, W, prm, 1 / 64, steps=10, limiter=limiter, bias=0.1)
    assert n == 10
    _matches(out, ref)


@pytest.mark.parametrize("thermal", [(True, True), (True, False), (False, True)], ids=["hot", "cold2", "cold1"])
def test_hpr_multiphysics_reinit_matches_oracle(gpu, oracle_lib, thermal):
    # two reinitialisations in a row: the second mixes the cold material's J that the first one set
    W = wl.hpr_multiphysics_riemann(50, seed=5, p2_scale=1.1, a2_scale=1.01)
    prm = wl.hpr_reduced_params(thermal=thermal, **STIFF2)
    ref = W.copy()
    O.run_two_material(O.HPR_MULTIPHYSICS, ref, 1 / 50, 0.8, steps=2, limiter=2, reinit=1, params=prm)
    out, _, _ = _device(gpu, W, prm, 1 / 50, steps=2, limiter=2, reinit=1)
    _matches(out, ref)


def test_hpr_multiphysics_time_driven(gpu, oracle_lib):
    W = wl.hpr_multiphysics_riemann(72, seed=7, p2_scale=0.9)
    ref = W.copy()
    t_ref, n_ref = O.run_two_material(O.HPR_MULTIPHYSICS, ref, 1 / 72, 0.8, t_end=0.012, limiter=0, params=PRM,
                                      subcycles=2)
    out, t, n = _device(gpu, W, PRM, 1 / 72, t_end=0.012, limiter=0, subcycles=2)
    assert t == t_ref and n == n_ref
    _matches(out, ref)


def test_hpr_multiphysics_first_order(gpu, oracle_lib):
    W = wl.hpr_multiphysics_riemann(50, seed=8)
    ref = W.copy()
    O.run_first_order(O.HPR_MULTIPHYSICS, ref, 1 / 50, 0.8, steps=8, params=PRM)
    out, _, _ = _device(gpu, W, PRM, 1 / 50, steps=8, order=1)
    _matches(out, ref)


def test_hpr_multiphysics_max_wave_speed(gpu, oracle_lib):
    W = wl.hpr_multiphysics_riemann(40, seed=9, p2_scale=1.5, a2_scale=1.02)
    with gpu.Solver(gpu.HPR_MULTIPHYSICS, 40, 1, PRM) as s:
        s.upload(W)
        got = s.max_wave_speed()
    assert got == O.max_wave(O.HPR_MULTIPHYSICS, W, PRM)


def test_hpr_multiphysics_argument_checks(gpu):
    with pytest.raises(gpu.VgError):
        gpu.Solver(gpu.HPR_MULTIPHYSICS, 16, 1, PRM, precision=gpu.MIXED)
    with pytest.raises(gpu.VgError):
        gpu.Solver(gpu.HPR_MULTIPHYSICS, 16, 8, PRM)  # 1D only, as the reference's model
    with gpu.Solver(gpu.HPR_MULTIPHYSICS, 32, 1, PRM) as s:
        s.upload(wl.hpr_multiphysics_riemann(32, seed=9))
        with pytest.raises(gpu.VgError):
            s.run(1 / 32, 0.8, steps=3, stiff=True)
        t, n = s.run(1 / 32, 0.8, steps=3, subcycles=1, reinit=3)
        assert n == 3 and np.isfinite(s.download()).all()
