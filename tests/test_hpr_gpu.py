"""HPR (GPR) model on the GPU against the CPU oracle.

Sweeps and the acoustic-tensor CFL are exact-FP64 restatements: compared bit for bit.  The RK4 relaxation
source evaluates pow(det A, 5/3) (HPR/hprsourceterms.cpp:21-26); CUDA's pow and glibc's may differ in the last
place, so runs with the source switched on are compared at a per-cell relative bound of 1e-12.
"""
import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

REL = 1e-12


def _bitwise(a, b):
    if not np.array_equal(a, b):
        d = np.abs(a - b)
        i = np.unravel_index(np.argmax(d), d.shape)
        raise AssertionError(f"max |diff| {d.max():.3e} at {i}; {np.count_nonzero(d)} values differ")


def _rel(a, b):
    scale = np.maximum(np.abs(b), 1e-300)
    r = np.where(a == b, 0.0, np.abs(a - b) / scale)
    return float(r.max())


@pytest.mark.parametrize("bc", [0, 1])
def test_hpr_2d_sweeps_bitwise(gpu, oracle_lib, bc):
    nx, ny = 40, 32
    W = wl.hpr_smooth_2d(nx, ny, seed=5 + bc)
    prm = wl.hpr_params(tau1=1e-2, tau2=1e-2)
    ref = W.copy()
    O.run(O.HPR, ref, 1.0 / nx, 0.8, steps=8, limiter=0, params=prm, bc=bc)
    with gpu.Solver(gpu.HPR, nx, ny, prm, boundary=bc) as s:
        s.upload(W)
        s.run(1.0 / nx, 0.8, steps=8, limiter=0)
        out = s.download()
    _bitwise(out, ref)


@pytest.mark.parametrize("axis", [0, 1])
def test_hpr_single_sweep(gpu, oracle_lib, axis):
    nx, ny = 70, 45
    W = wl.hpr_smooth_2d(nx, ny, seed=9)
    W[3] = 0.02  # a non-zero A01 and J exercise the full 3x3 algebra
    W[14] = 0.05
    prm = wl.hpr_params(tau1=1e-2, tau2=1e-2)
    ref = W.copy()
    O.sweep(O.HPR, ref, axis, 1.0 / nx, 2e-4, limiter=1, params=prm)
    with gpu.Solver(gpu.HPR, nx, ny, prm) as s:
        s.upload(W)
        s.sweep(axis, 1.0 / nx, 2e-4, limiter=1)
        out = s.download()
    _bitwise(out, ref)


def test_hpr_max_wave_speed(gpu, oracle_lib):
    nx, ny = 33, 29
    W = wl.hpr_smooth_2d(nx, ny, seed=12)
    W[2:11] += 0.05 * np.random.default_rng(1).standard_normal((9, ny, nx))
    for thermal in (True, False):
        prm = wl.hpr_params(thermal=thermal)
        with gpu.Solver(gpu.HPR, nx, ny, prm) as s:
            s.upload(W)
            assert s.max_wave_speed() == O.max_wave(O.HPR, W, prm)


def test_hpr_2d_rk4_source(gpu, oracle_lib):
    nx, ny = 24, 20
    W = wl.hpr_smooth_2d(nx, ny, seed=13)
    prm = wl.hpr_params(tau1=1e-2, tau2=1e-2)
    ref = W.copy()
    O.run(O.HPR, ref, 1.0 / nx, 0.8, steps=4, limiter=0, params=prm, subcycles=1)
    with gpu.Solver(gpu.HPR, nx, ny, prm) as s:
        s.upload(W)
        s.run(1.0 / nx, 0.8, steps=4, limiter=0, subcycles=1)
        out = s.download()
    assert _rel(out, ref) <= REL


def test_hpr_1d_heat_conduction_rk4(gpu, oracle_lib):
    n = 100
    W = wl.hpr_heat_conduction_1d(n)
    prm = wl.hpr_params(tau1=1e-1, tau2=1e-1)
    ref = W.copy()
    O.run(O.HPR, ref, 1.0 / n, 0.8, steps=20, limiter=0, params=prm, subcycles=2)
    with gpu.Solver(gpu.HPR, n, 1, prm) as s:
        s.upload(W)
        s.run(1.0 / n, 0.8, steps=20, limiter=0, subcycles=2)
        out = s.download()
    assert _rel(out, ref) <= REL


def test_hpr_golden_rk4(gpu):
    """The committed golden fixture made by the reference's own code (tests/golden/make_golden.py)."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "hpr2d_smooth16_rk4sub1_4.npz"))
    W, out_ref = z["w0"], z["out"]
    ny, nx = W.shape[1:]
    with gpu.Solver(gpu.HPR, nx, ny, z["params"]) as s:
        s.upload(W)
        s.run(float(z["dx"]), float(z["cfl"]), steps=int(z["steps"]), limiter=int(z["limiter"]),
              subcycles=int(z["subcycles"]))
        out = s.download()
    assert _rel(out, out_ref) <= REL


def test_hpr_non_thermal_keeps_heat_flux(gpu, oracle_lib):
    """A non-thermal material: J is not evolved, and setConservedVariableVector leaves it as the cell had it, so a
    non-zero initial J must survive every sweep unchanged, bit for bit with the oracle."""
    nx, ny = 30, 26
    W = wl.hpr_smooth_2d(nx, ny, seed=17)
    rng = np.random.default_rng(5)
    W[14:17] = 0.1 * rng.standard_normal((3, ny, nx))
    prm = wl.hpr_params(thermal=False)
    ref = W.copy()
    O.run(O.HPR, ref, 1.0 / nx, 0.8, steps=6, limiter=0, params=prm)
    assert np.array_equal(ref[14:17], W[14:17])
    for prec in (gpu.FP64, gpu.MIXED):
        with gpu.Solver(gpu.HPR, nx, ny, prm, precision=prec) as s:
            s.upload(W)
            s.run(1.0 / nx, 0.8, steps=6, limiter=0)
            out = s.download()
        assert np.array_equal(out[14:17], W[14:17])
        if prec == gpu.FP64:
            _bitwise(out, ref)
