"""Parity of the CUDA path (through the C ABI) with the CPU oracle on the same inputs.

The plain FP64 form must reproduce the reference's arithmetic exactly: results are compared bit for bit
(np.array_equal), which is stricter than the 1e-12 per-cell relative bound the FP64 form promises.
"""
import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _bitwise(a, b):
    if np.array_equal(a, b):
        return True
    d = np.abs(a - b)
    i = np.unravel_index(np.argmax(d), d.shape)
    raise AssertionError(f"max |diff| {d.max():.3e} at {i}: {a[i]!r} vs {b[i]!r}; "
                         f"{np.count_nonzero(d)} differing values")


def test_sod_1d_time_driven(gpu, oracle_lib):
    """1D Euler shock tube: minbee, CFL 0.9, run to t = 0.25 (613 steps), transmissive."""
    n = 1000
    W = wl.sod_1d(n)
    prm = wl.euler_params(1.4)
    ref = W.copy()
    t_ref, steps_ref = O.run(O.EULER, ref, 1.0 / n, 0.9, t_end=0.25, limiter=O.MINBEE, params=prm)
    with gpu.Solver(gpu.EULER, n, 1, prm) as s:
        s.upload(W)
        t, steps = s.run(1.0 / n, 0.9, t_end=0.25, limiter=gpu.MINBEE)
        out = s.download()
    assert steps == steps_ref == 613
    assert t == t_ref
    _bitwise(out, ref)


@pytest.mark.parametrize("limiter", [0, 1, 2])
@pytest.mark.parametrize("shape", [(64, 64), (130, 67)])
def test_euler_2d_quadrants_steps(gpu, oracle_lib, limiter, shape):
    nx, ny = shape
    W = wl.euler_quadrants_2d(nx, ny, seed=11 + limiter)
    prm = wl.euler_params(1.4)
    ref = W.copy()
    O.run(O.EULER, ref, 1.0 / nx, 0.8, steps=40, limiter=limiter, params=prm)
    with gpu.Solver(gpu.EULER, nx, ny, prm) as s:
        s.upload(W)
        t, steps = s.run(1.0 / nx, 0.8, steps=40, limiter=limiter)
        out = s.download()
    assert steps == 40
    _bitwise(out, ref)


@pytest.mark.parametrize("axis", [0, 1])
def test_euler_single_sweep(gpu, oracle_lib, axis):
    nx, ny = 300, 200
    W = wl.euler_quadrants_2d(nx, ny, seed=5)
    prm = wl.euler_params(1.4)
    ref = W.copy()
    O.sweep(O.EULER, ref, axis, 1.0 / nx, 3e-4, limiter=0, params=prm)
    with gpu.Solver(gpu.EULER, nx, ny, prm) as s:
        s.upload(W)
        s.sweep(axis, 1.0 / nx, 3e-4, limiter=0)
        out = s.download()
    _bitwise(out, ref)


def test_euler_max_wave_speed(gpu, oracle_lib):
    nx, ny = 257, 129
    W = wl.euler_quadrants_2d(nx, ny, seed=9)
    prm = wl.euler_params(1.4)
    with gpu.Solver(gpu.EULER, nx, ny, prm) as s:
        s.upload(W)
        assert s.max_wave_speed() == O.max_wave(O.EULER, W, prm)


@pytest.mark.parametrize("bc", [0, 1])
def test_mhd_2d_vortex(gpu, oracle_lib, bc):
    nx, ny = 96, 80
    W = wl.mhd_vortex_2d(nx, ny, seed=2)
    prm = wl.mhd_params(5.0 / 3.0)
    ref = W.copy()
    O.run(O.MHD, ref, 1.0 / nx, 0.8, steps=30, limiter=0, params=prm, bc=bc)
    with gpu.Solver(gpu.MHD, nx, ny, prm, boundary=bc) as s:
        s.upload(W)
        s.run(1.0 / nx, 0.8, steps=30, limiter=0)
        out = s.download()
    _bitwise(out, ref)


def test_mhd_1d_brio_wu(gpu, oracle_lib):
    n = 400
    W = wl.brio_wu_1d(n)
    prm = wl.mhd_params(2.0)
    ref = W.copy()
    O.run(O.MHD, ref, 1.0 / n, 0.8, steps=100, limiter=0, params=prm)
    with gpu.Solver(gpu.MHD, n, 1, prm) as s:
        s.upload(W)
        s.run(1.0 / n, 0.8, steps=100, limiter=0)
        out = s.download()
    _bitwise(out, ref)


def test_mhd_full_components(gpu, oracle_lib):
    """Non-zero w and Bz select the 9-component variant."""
    nx, ny = 64, 48
    W = wl.mhd_vortex_2d(nx, ny, seed=4)
    W[3] = 0.05 * np.sin(np.linspace(0, 6, nx))[None, :]
    W[7] = 0.1
    prm = wl.mhd_params(5.0 / 3.0)
    ref = W.copy()
    O.run(O.MHD, ref, 1.0 / nx, 0.8, steps=20, limiter=1, params=prm, bc=1)
    with gpu.Solver(gpu.MHD, nx, ny, prm, boundary=1) as s:
        s.upload(W)
        s.run(1.0 / nx, 0.8, steps=20, limiter=1)
        out = s.download()
    _bitwise(out, ref)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("model", [0, 1])
def test_every_launch_config_gives_identical_results(gpu, model, precision):
    """Tile shapes only move work between threads: every configuration yields the same bits."""
    nx, ny = 150, 70
    if model == 0:
        W, prm = wl.euler_quadrants_2d(nx, ny, seed=61), wl.euler_params(1.4)
    else:
        W, prm = wl.mhd_vortex_2d(nx, ny, seed=62), wl.mhd_params(5.0 / 3.0)
    outs = []
    with gpu.Solver(model, nx, ny, prm, precision=precision) as s:
        for xc in range(gpu.NUM_XCFG):
            for yc in range(gpu.NUM_YCFG):
                if xc and yc and xc != yc % gpu.NUM_XCFG:
                    continue  # every X and every Y configuration appears at least once
                s.set_launch_config(xc, yc)
                s.upload(W)
                s.run(1.0 / nx, 0.8, steps=6, limiter=0)
                outs.append(((xc, yc), s.download()))
    for cfg, o in outs[1:]:
        assert np.array_equal(o, outs[0][1]), cfg


def test_autotune_picks_and_keeps_results(gpu, oracle_lib):
    nx, ny = 256, 192
    W, prm = wl.euler_quadrants_2d(nx, ny, seed=63), wl.euler_params(1.4)
    ref = W.copy()
    O.run(O.EULER, ref, 1.0 / nx, 0.8, steps=10, limiter=0, params=prm)
    with gpu.Solver(gpu.EULER, nx, ny, prm) as s:
        s.upload(W)
        xt, yt = s.autotune(1.0 / nx, 0.8, limiter=0)
        assert all(t > 0 for t in xt) and all(t > 0 for t in yt)
        x, y, _, _ = s.launch_config()
        assert xt[x] == min(xt) and yt[y] == min(yt)
        fused, separate = s.schedule_times
        assert fused > 0 and separate > 0
        assert s.schedule() == (1 if separate < fused else 0)
        s.upload(W)
        s.run(1.0 / nx, 0.8, steps=10, limiter=0)
        _bitwise(s.download(), ref)


@pytest.mark.parametrize("model,precision", [(0, 0), (0, 1), (1, 0), (2, 0)])
def test_cfl_schedules_give_identical_results(gpu, oracle_lib, model, precision):
    """The step schedule (the next step's CFL maximum folded into the last X sweep, or a separate reduction pass)
    changes where the maximum is taken, not its value: both schedules give the same bits, time-driven and
    step-driven, and the FP64 form stays bit-equal to the oracle; a separate pass is one more launch per step."""
    nx, ny = 96, 72
    if model == 0:
        W, prm = wl.euler_quadrants_2d(nx, ny, seed=64), wl.euler_params(1.4)
    elif model == 1:
        W, prm = wl.mhd_vortex_2d(nx, ny, seed=65), wl.mhd_params(5.0 / 3.0)
    else:
        W, prm = wl.hpr_smooth_2d(nx, ny, seed=66), wl.hpr_params(tau1=1e-2, tau2=1e-2)
    outs, launches = {}, {}
    with gpu.Solver(model, nx, ny, prm, precision=precision) as s:
        for sched in (0, 1):
            s.set_schedule(sched)
            assert s.schedule() == sched
            s.upload(W)
            t, it = s.run(1.0 / nx, 0.8, steps=9, limiter=0)
            launches[sched] = s.last_launch_count()
            s.upload(W)
            t2, it2 = s.run(1.0 / nx, 0.8, t_end=0.02, limiter=0)
            outs[sched] = (s.download(), t, it, t2, it2)
    a, b = outs[0], outs[1]
    assert np.array_equal(a[0], b[0]) and a[1:] == b[1:]
    assert launches[1] == launches[0] + 9
    if precision == 0:
        ref = W.copy()
        O.run(model, ref, 1.0 / nx, 0.8, t_end=0.02, limiter=0, params=prm)
        _bitwise(a[0], ref)


@pytest.mark.parametrize("bc", [0, 1])
def test_mhd_glm_subcycles_bitwise(gpu, oracle_lib, bc):
    """MHD with GLM damping sub-cycles (MHDForcingSolver's RK4 before and after the sweeps), FP64 bit for bit;
    the mixed form keeps the damping in FP64 and stays within the mixed-form bound."""
    nx, ny = 40, 36
    W = wl.mhd_vortex_2d(nx, ny, seed=6)
    W[8] = 0.01 * np.sin(2 * np.pi * np.arange(nx) / nx)[None, :] * np.ones((ny, 1))
    prm = wl.mhd_params(5.0 / 3.0)
    ref = W.copy()
    O.run(O.MHD, ref, 1.0 / nx, 0.8, steps=12, limiter=0, params=prm, bc=bc, subcycles=2)
    assert np.abs(ref[8] - W[8]).max() > 1e-4
    for prec in (gpu.FP64, gpu.MIXED):
        with gpu.Solver(gpu.MHD, nx, ny, prm, precision=prec, boundary=bc) as s:
            s.upload(W)
            s.run(1.0 / nx, 0.8, steps=12, limiter=0, subcycles=2)
            out = s.download()
        if prec == gpu.FP64:
            assert np.array_equal(out, ref)
        else:
            assert np.abs(out[0] - ref[0]).mean() <= 1e-6
            assert np.abs(out[8] - ref[8]).max() <= 1e-5


def test_mhd_1d_glm_subcycles_bitwise(gpu, oracle_lib):
    n = 120
    W = wl.brio_wu_1d(n)
    W[8] = 0.01 * np.sin(np.arange(n))
    prm = wl.mhd_params(2.0)
    ref = W.copy()
    O.run(O.MHD, ref, 1.0 / n, 0.8, steps=15, limiter=1, params=prm, subcycles=3)
    with gpu.Solver(gpu.MHD, n, 1, prm) as s:
        s.upload(W)
        s.run(1.0 / n, 0.8, steps=15, limiter=1, subcycles=3)
        out = s.download()
    assert np.array_equal(out, ref)
