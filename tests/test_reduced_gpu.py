"""The Euler two-material models on the device (VG_MODEL_EULER_REDUCED, VG_MODEL_EULER_MULTIPHYSICS): the exact FP64 form against the
golden fixtures made by the reference's own SecondOrderSolver::solve{,2D} (tests/golden/make_golden.py) and against
the oracle (pinned to the reference in test_reduced.py), bit for bit, with the volume-fraction reinitialisation;
the mixed form within L1 1e-6 of the mixture density; the first-order loop; argument checks."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "reduced*.npz")) +
                glob.glob(os.path.join(os.path.dirname(__file__), "golden", "multiphysics*.npz")))
MODELS = [O.EULER_REDUCED, O.EULER_MULTIPHYSICS]


def _planes(model, W):
    return W if model == O.EULER_REDUCED else wl.multiphysics_from_reduced(W)


def _bitwise(a, b):
    if not np.array_equal(a, b):
        d = np.abs(a - b)
        raise AssertionError(f"max |diff| {d.max():.3e}; {np.count_nonzero(d)} values differ")


def _device(gpu, W, prm, dx, precision=None, boundary=None, model=O.EULER_REDUCED, **run):
    nx = W.shape[-1]
    ny = 1 if W.ndim == 2 else W.shape[1]
    kw = {}
    if precision is not None:
        kw["precision"] = precision
    if boundary is not None:
        kw["boundary"] = boundary
    with gpu.Solver(model, nx, ny, prm, **kw) as s:
        s.upload(W)
        t, n = s.run(dx, 0.8, **run)
        return s.download(), t, n


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_reduced_golden(gpu, path):
    z = np.load(path)
    out, _, n = _device(gpu, z["w0"], z["params"], float(z["dx"]), model=int(z["model"]), steps=int(z["steps"]),
                        limiter=int(z["limiter"]), reinit=int(z["reinit"]))
    assert n == int(z["steps"])
    _bitwise(out, z["out"])


@pytest.mark.parametrize("model", MODELS)
@pytest.mark.parametrize("reinit", [0, 3])
@pytest.mark.parametrize("limiter", [0, 2])
@pytest.mark.parametrize("ny", [1, 20])
def test_reduced_matches_oracle(gpu, oracle_lib, ny, limiter, reinit, model):
    prm = wl.reduced_params(1.4, 0.0, 1.67, 0.0)
    W = wl.reduced_shock_tube(130, rho=(1.0, 0.1379), p=(2.0, 1.0)) if ny == 1 else wl.reduced_bubble_2d(36, ny)
    W = _planes(model, W)
    dx = 1.0 / W.shape[-1]
    ref = W.copy()
    O.run_two_material(model, ref, dx, 0.8, steps=17, limiter=limiter, params=prm, reinit=reinit)
    out, _, _ = _device(gpu, W, prm, dx, model=model, steps=17, limiter=limiter, reinit=reinit)
    _bitwise(out, ref)


def test_reduced_time_driven_and_periodic(gpu, oracle_lib):
    prm = wl.reduced_params(1.4, 0.0, 1.4, 0.0)
    W = wl.reduced_shock_tube(150)
    ref = W.copy()
    t_ref, n_ref = O.run_reduced(ref, 1 / 150, 0.8, t_end=0.05, limiter=1, params=prm, reinit=5)
    out, t, n = _device(gpu, W, prm, 1 / 150, t_end=0.05, limiter=1, reinit=5)
    assert (t, n) == (t_ref, n_ref)
    _bitwise(out, ref)
    W2 = wl.reduced_bubble_2d(30, 26)
    ref = W2.copy()
    O.run_reduced(ref, 1 / 30, 0.8, steps=9, limiter=0, params=prm, bc=O.PERIODIC)
    out, _, _ = _device(gpu, W2, prm, 1 / 30, boundary=gpu.PERIODIC, steps=9, limiter=0)
    _bitwise(out, ref)


@pytest.mark.parametrize("model", MODELS)
def test_reduced_first_order(gpu, oracle_lib, model):
    prm = wl.reduced_params(1.4, 0.0, 1.67, 0.0)
    W = _planes(model, wl.reduced_bubble_2d(28, 24))
    ref = W.copy()
    O.run_first_order(model, ref, 1 / 28, 0.8, steps=12, params=prm)
    out, _, _ = _device(gpu, W, prm, 1 / 28, model=model, steps=12, order=1)
    _bitwise(out, ref)


def test_multiphysics_has_no_mixed_form(gpu):
    with pytest.raises(gpu.VgError):
        gpu.Solver(gpu.EULER_MULTIPHYSICS, 16, 1, wl.reduced_params(), precision=gpu.MIXED)


@pytest.mark.parametrize("model", [O.EULER_REDUCED])
def test_reduced_mixed_form(gpu, model):
    """Without reinitialisation: the reinitialisation resets whole windows where alpha crosses 0.5, a discontinuous
    decision that last-place differences can flip, so the two forms are compared on the sweeps alone."""
    prm = wl.reduced_params(1.4, 0.0, 1.67, 0.0)
    W = _planes(model, wl.reduced_bubble_2d(64))
    fp64, _, _ = _device(gpu, W, prm, 1 / 64, model=model, steps=30, limiter=0)
    mixed, _, _ = _device(gpu, W, prm, 1 / 64, model=model, precision=gpu.MIXED, steps=30, limiter=0)
    i2 = 5 if model == O.EULER_REDUCED else 6

    def rho(P):
        return P[0] * P[4] + (1.0 - P[0]) * P[i2]

    l1 = np.abs(rho(mixed) - rho(fp64)).mean()
    print(f"reduced mixed L1(rho) {l1:.2e}")
    assert np.isfinite(mixed).all() and l1 <= 1e-6


def test_reduced_argument_checks(gpu):
    prm = wl.reduced_params()
    W = wl.reduced_shock_tube(32)
    W[3, 5] = 0.1  # w != 0
    with gpu.Solver(gpu.EULER_REDUCED, 32, 1, prm) as s:
        with pytest.raises(gpu.VgError):
            s.upload(W)
        s.upload(wl.reduced_shock_tube(32))
        with pytest.raises(gpu.VgError):
            s.run(1 / 32, 0.8, steps=3, order=1, reinit=2)
        with pytest.raises(gpu.VgError):
            s.run(1 / 32, 0.8, steps=3, reinit=-1)
    with gpu.Solver(gpu.EULER, 32, 1, wl.euler_params(1.4)) as s:
        s.upload(wl.sod_1d(32))
        with pytest.raises(gpu.VgError):
            s.run(1 / 32, 0.8, steps=3, reinit=2)
