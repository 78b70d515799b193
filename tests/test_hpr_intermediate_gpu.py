"""The HPR intermediate two-material model on the device (VG_MODEL_HPR_INTERMEDIATE): the exact FP64 form against the
golden fixtures made by the reference (its own HPRSecondOrderSolver::solve and solve2D to t_end, its per-step functions
with cold materials and with the 2D reinitialisation) and against the oracle (pinned in test_hpr_intermediate.py), with
the RK4 relaxation sub-cycles, the reinitialisation of volume fraction, densities and pressures, periodic ghosts and
the first-order loop; the CFL maximum wave speed; argument checks.

Runs without the relaxation source are compared bit for bit; runs with sub-cycles plane by plane (the largest
difference within 1e-12 of the plane's largest magnitude), because the source's theta1 takes pow(det A, 5/3)
(HPR/hprsourceterms.cpp:21-26) and CUDA's pow and glibc's may differ in the last place: a last-place difference in a
cell grows over the steps, and a per-cell relative bound would amplify it in components near zero."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "hprintermediate*.npz")))
STIFF2 = dict(gamma2=2.0, p_inf2=0.5)
PRM = wl.hpr_reduced_params(**STIFF2)
REL = 1e-12
# solid materials take pow in their equations of state (the ShockMieGruneisen cold curve, the plastic relaxation)
REL_SOLID = 1e-10


def _matches(a, b, subcycles, rel=REL):
    """Bit for bit without the relaxation source, else every plane within rel of its largest magnitude."""
    assert np.isfinite(a).all()
    if subcycles == 0:
        if not np.array_equal(a, b):
            d = np.abs(a - b)
            raise AssertionError(f"max |diff| {d.max():.3e}; {np.count_nonzero(d)} values differ")
        return
    d = np.abs(a - b).reshape(b.shape[0], -1).max(axis=1)
    scale = np.maximum(np.abs(b).reshape(b.shape[0], -1).max(axis=1), 1e-300)
    assert (d / scale).max() <= rel, f"max normwise diff {(d / scale).max():.3e}"


def _device(gpu, W, prm, dx, boundary=None, **run):
    nx = W.shape[-1]
    ny = 1 if W.ndim == 2 else W.shape[1]
    kw = {} if boundary is None else {"boundary": boundary}
    with gpu.Solver(gpu.HPR_INTERMEDIATE, nx, ny, prm, **kw) as s:
        s.upload(W)
        t, n = s.run(dx, 0.8, **run)
        return s.download(), t, n


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_hpr_intermediate_golden(gpu, path):
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
    _matches(out, z["out"], int(z["subcycles"]) or solid, rel=REL_SOLID if solid else REL)


@pytest.mark.parametrize("thermal", [(True, True), (True, False), (False, False)], ids=["hot", "mixed", "cold"])
@pytest.mark.parametrize("subcycles", [0, 1])
@pytest.mark.parametrize("limiter", [0, 2])
@pytest.mark.parametrize("ny", [1, 14])
def test_hpr_intermediate_matches_oracle(gpu, oracle_lib, ny, limiter, subcycles, thermal):
    nx = 64 if ny == 1 else 18
    W = wl.hpr_intermediate_riemann(nx, ny, seed=3, p2_scale=1.1)
    prm = wl.hpr_reduced_params(thermal=thermal, **STIFF2)
    steps = 10 if ny == 1 else 5
    ref = W.copy()
    O.run_two_material(O.HPR_INTERMEDIATE, ref, 1 / nx, 0.8, steps=steps, limiter=limiter, params=prm,
                       subcycles=subcycles)
    out, _, n = _device(gpu, W, prm, 1 / nx, steps=steps, limiter=limiter, subcycles=subcycles)
    assert n == steps
    _matches(out, ref, subcycles)


@pytest.mark.parametrize("ny,bubble,reinit", [(1, False, 3), (20, True, 2), (16, False, 3)])
def test_hpr_intermediate_reinit_matches_oracle(gpu, oracle_lib, ny, bubble, reinit):
    nx = 60 if ny == 1 else 20
    W = wl.hpr_intermediate_riemann(nx, ny, seed=nx, bubble=bubble, p2_scale=1.2)
    ref = W.copy()
    kw = dict(steps=9 if ny == 1 else 6, limiter=2, bias=0.0 if ny == 1 else 0.1, reinit=reinit)
    O.run_two_material(O.HPR_INTERMEDIATE, ref, 1 / nx, 0.8, params=PRM, **kw)
    out, _, _ = _device(gpu, W, PRM, 1 / nx, **kw)
    _matches(out, ref, 0)


def test_hpr_intermediate_time_driven_and_periodic(gpu, oracle_lib):
    W = wl.hpr_intermediate_riemann(72, seed=5)
    ref = W.copy()
    t_ref, n_ref = O.run_two_material(O.HPR_INTERMEDIATE, ref, 1 / 72, 0.8, t_end=0.02, limiter=1, params=PRM,
                                      subcycles=1)
    out, t, n = _device(gpu, W, PRM, 1 / 72, t_end=0.02, limiter=1, subcycles=1)
    assert (t, n) == (t_ref, n_ref)
    _matches(out, ref, 1)
    W2 = wl.hpr_intermediate_riemann(18, 16, seed=6, bubble=True)
    ref = W2.copy()
    O.run_two_material(O.HPR_INTERMEDIATE, ref, 1 / 18, 0.8, steps=5, limiter=2, params=PRM, subcycles=1,
                       bc=O.PERIODIC)
    out, _, _ = _device(gpu, W2, PRM, 1 / 18, boundary=gpu.PERIODIC, steps=5, limiter=2, subcycles=1)
    _matches(out, ref, 1)


@pytest.mark.parametrize("ny", [1, 12])
def test_hpr_intermediate_first_order(gpu, oracle_lib, ny):
    nx = 50 if ny == 1 else 16
    W = wl.hpr_intermediate_riemann(nx, ny, seed=7)
    ref = W.copy()
    O.run_first_order(O.HPR_INTERMEDIATE, ref, 1 / nx, 0.8, steps=8, params=PRM)
    out, _, _ = _device(gpu, W, PRM, 1 / nx, steps=8, order=1)
    _matches(out, ref, 0)


@pytest.mark.parametrize("ny", [1, 10])
def test_hpr_intermediate_max_wave_speed(gpu, oracle_lib, ny):
    nx = 40 if ny == 1 else 12
    W = wl.hpr_intermediate_riemann(nx, ny, seed=8, bubble=ny > 1, p2_scale=1.5)
    with gpu.Solver(gpu.HPR_INTERMEDIATE, nx, ny, PRM) as s:
        s.upload(W)
        got = s.max_wave_speed()
    assert got == O.max_wave(O.HPR_INTERMEDIATE, W, PRM)


def test_hpr_intermediate_argument_checks(gpu):
    with pytest.raises(gpu.VgError):
        gpu.Solver(gpu.HPR_INTERMEDIATE, 16, 1, PRM, precision=gpu.MIXED)
    with gpu.Solver(gpu.HPR_INTERMEDIATE, 32, 1, PRM) as s:
        s.upload(wl.hpr_intermediate_riemann(32, seed=9))
        with pytest.raises(gpu.VgError):
            s.run(1 / 32, 0.8, steps=3, order=1, reinit=2)
        with pytest.raises(gpu.VgError):
            s.run(1 / 32, 0.8, steps=3, stiff=True)
        t, n = s.run(1 / 32, 0.8, steps=4, subcycles=1, reinit=2)
        assert n == 4 and np.isfinite(s.download()).all()
