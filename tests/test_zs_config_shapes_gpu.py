"""Parity at the benchmark configurations' own shapes, against the CPU oracle on the same seeded inputs.

The small-grid tests elsewhere pin every code path; these run the shapes and seeds that bench.py times, so the
numbers it reports are for results that are known to equal the oracle's:

* 2D Euler 4096 x 4096, four-quadrant Riemann data, superbee, CFL 0.8: 5 steps (bitwise), and the mixed form's
  L1/Linf density error against the oracle on the same 5 steps;
* 2D Euler 1024 x 1024 for the configuration's full 200 steps (bitwise);
* 2D MHD 2048 x 2048 periodic vortex with seeded noise: 5 steps (bitwise, and the mixed form's error);
* 2D HPR 1024 x 1024 with the RK4 relaxation forcing at the benchmark's sub-cycle count: 2 steps (<= 1e-12
  relative per cell: the source calls pow, which CUDA and glibc may round differently in the last place);
* the full 4096-instance ragged batch: 5 steps, every instance against its own solve() loop (bitwise);
* single-material Euler with a stiffened-gas p_inf != 0 and a non-zero limiter bias (bitwise).

The oracle runs on the host cores, so these take tens of seconds; the file is named to run after the others.
"""
import math

import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

SEED = 2024          # the seed bench.py uses for every configuration
CFL = 0.8
REL = 1e-12
MIXED_L1 = 1e-6      # the mixed form's density error bar


def _bitwise(a, b):
    if np.array_equal(a, b):
        return
    d = np.abs(a - b)
    i = np.unravel_index(np.argmax(d), d.shape)
    raise AssertionError(f"max |diff| {d.max():.3e} at {i}: {a[i]!r} vs {b[i]!r}; {np.count_nonzero(d)} values differ")


def _run_gpu(gpu, model, W, prm, dx, steps, precision=None, boundary=0, **kw):
    ny, nx = (W.shape[1], W.shape[2]) if W.ndim == 3 else (1, W.shape[1])
    prec = gpu.FP64 if precision is None else precision
    with gpu.Solver(model, nx, ny, prm, precision=prec, boundary=boundary) as s:
        s.upload(W)
        _, it = s.run(dx, CFL, steps=steps, **kw)
        out = s.download()
    assert it == steps
    return out


def test_euler_4096_five_steps(gpu, oracle_lib):
    """The 4096^2 Euler configuration itself: FP64 bit-equal to the oracle after 5 steps; the mixed form within
    the density-error bar of the same oracle result."""
    n = 4096
    W = wl.euler_quadrants_2d(n, n, seed=SEED)
    prm = wl.euler_params(1.4)
    ref = W.copy()
    O.run(O.EULER, ref, 1.0 / n, CFL, steps=5, limiter=O.SUPERBEE, params=prm)
    out = _run_gpu(gpu, gpu.EULER, W, prm, 1.0 / n, 5, limiter=gpu.SUPERBEE)
    _bitwise(out, ref)
    del out
    mixed = _run_gpu(gpu, gpu.EULER, W, prm, 1.0 / n, 5, precision=gpu.MIXED, limiter=gpu.SUPERBEE)
    d = np.abs(mixed[0] - ref[0])
    assert d.mean() <= MIXED_L1, d.mean()
    assert d.max() <= 1e-3, d.max()


def test_euler_1024_full_200_steps(gpu, oracle_lib):
    """The configuration's full step count on a 1024^2 grid of the same quadrant layout."""
    n = 1024
    W = wl.euler_quadrants_2d(n, n, seed=SEED)
    prm = wl.euler_params(1.4)
    ref = W.copy()
    O.run(O.EULER, ref, 1.0 / n, CFL, steps=200, limiter=O.SUPERBEE, params=prm)
    out = _run_gpu(gpu, gpu.EULER, W, prm, 1.0 / n, 200, limiter=gpu.SUPERBEE)
    _bitwise(out, ref)


def test_mhd_2048_periodic_five_steps(gpu, oracle_lib):
    """The 2048^2 periodic MHD vortex (seeded perturbations) after 5 steps: FP64 bitwise, mixed within the bar."""
    n = 2048
    W = wl.mhd_vortex_2d(n, seed=SEED)
    prm = wl.mhd_params()
    ref = W.copy()
    O.run(O.MHD, ref, 1.0 / n, CFL, steps=5, limiter=O.SUPERBEE, params=prm, bc=O.PERIODIC)
    out = _run_gpu(gpu, gpu.MHD, W, prm, 1.0 / n, 5, boundary=gpu.PERIODIC, limiter=gpu.SUPERBEE)
    _bitwise(out, ref)
    del out
    mixed = _run_gpu(gpu, gpu.MHD, W, prm, 1.0 / n, 5, precision=gpu.MIXED, boundary=gpu.PERIODIC,
                     limiter=gpu.SUPERBEE)
    d = np.abs(mixed[0] - ref[0])
    assert d.mean() <= MIXED_L1, d.mean()


def test_hpr_1024_rk4_forcing_two_steps(gpu, oracle_lib):
    """The 1024^2 HPR configuration (seeded relaxation times) with the reference's RK4 forcing at the sub-cycle
    count the benchmark derives from the explicit stability bound, 2 steps."""
    n = 1024
    tau1, tau2 = wl.hpr_relaxation_times(SEED)
    prm = wl.hpr_params(tau1=tau1, tau2=tau2)
    W = wl.hpr_smooth_2d(n, seed=SEED)
    with gpu.Solver(gpu.HPR, n, n, prm) as s:
        s.upload(W)
        S0 = s.max_wave_speed()
    sub = max(1, math.ceil(0.5 * (1.5 * CFL * (1.0 / n) / S0) / (2.5 * min(tau1, tau2))))
    ref = W.copy()
    O.run(O.HPR, ref, 1.0 / n, CFL, steps=2, limiter=O.SUPERBEE, params=prm, subcycles=sub)
    out = _run_gpu(gpu, gpu.HPR, W, prm, 1.0 / n, 2, limiter=gpu.SUPERBEE, subcycles=sub)
    same = out == ref
    scale = np.maximum(np.abs(ref), 1e-300)
    rel = np.where(same, 0.0, np.abs(out - ref) / scale)
    assert rel.max() <= REL, (float(rel.max()), np.unravel_index(np.argmax(rel), rel.shape), sub)


def test_ragged_batch_4096_instances(gpu, oracle_lib):
    """The full ragged batch (4096 instances, cells U{200..4000}, seeded states and gamma) for 5 steps: every
    instance bit-equal to its own solve() loop, and its last dt equal to that loop's."""
    ncell, dx, gamma, theta, W = wl.ragged_riemann_batch(ninst=4096, seed=SEED)
    steps = 5
    with gpu.Batch(ncell, dx, gamma) as b:
        b.upload(W)
        dts = b.run(CFL, steps, limiter=gpu.SUPERBEE)
        out = b.download()
    off = 0
    for k, n in enumerate(ncell):
        ref = W[:, off:off + n].copy()
        _, st, dtl = O.run(O.EULER, ref, dx[k], CFL, steps=steps, limiter=O.SUPERBEE,
                           params=wl.euler_params(gamma[k]), dt_log=True)
        assert st == steps
        if not np.array_equal(out[:, off:off + n], ref):
            _bitwise(out[:, off:off + n], ref)
        assert dts[k] == dtl[-1], k
        off += n


@pytest.mark.parametrize("limiter", [0, 1, 2])
def test_stiffened_gas_with_bias(gpu, oracle_lib, limiter):
    """Single-material Euler with p_inf != 0 (stiffened gas) and a non-zero limiter bias, 2D, 30 steps."""
    nx, ny = 200, 150
    W = wl.euler_quadrants_2d(nx, ny, seed=31 + limiter)
    prm = wl.euler_params(1.9, 0.6)
    for bias in (0.4, -0.7):
        ref = W.copy()
        O.run(O.EULER, ref, 1.0 / nx, CFL, steps=30, bias=bias, limiter=limiter, params=prm)
        out = _run_gpu(gpu, gpu.EULER, W, prm, 1.0 / nx, 30, bias=bias, limiter=limiter)
        _bitwise(out, ref)
