"""The mixed FP32/FP64 form against the FP64 oracle, and conservation of both forms.

Tolerances (stated per config, as the mixed form promises): L1 of density over the grid <= 1e-6 after the
run, and an L-infinity bound that allows a few cells near discontinuities to take another limiter branch.
"""
import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

L1_RHO = 1e-6


def _errors(a, b):
    d = np.abs(a - b)
    return float(d.mean()), float(d.max())


@pytest.mark.parametrize("limiter", [0, 1, 2])
def test_mixed_euler_2d_quadrants(gpu, oracle_lib, limiter):
    nx = ny = 128
    W = wl.euler_quadrants_2d(nx, ny, seed=21 + limiter)
    prm = wl.euler_params(1.4)
    ref = W.copy()
    O.run(O.EULER, ref, 1.0 / nx, 0.8, steps=60, limiter=limiter, params=prm)
    with gpu.Solver(gpu.EULER, nx, ny, prm, precision=gpu.MIXED) as s:
        s.upload(W)
        s.run(1.0 / nx, 0.8, steps=60, limiter=limiter)
        out = s.download()
    l1, linf = _errors(out[0], ref[0])
    print(f"euler2d mixed lim{limiter}: L1(rho) {l1:.3e}  Linf(rho) {linf:.3e}")
    assert l1 <= L1_RHO
    assert linf <= 1e-3


def test_mixed_sod_1d(gpu, oracle_lib):
    n = 1000
    W = wl.sod_1d(n)
    prm = wl.euler_params(1.4)
    ref = W.copy()
    O.run(O.EULER, ref, 1.0 / n, 0.9, t_end=0.25, limiter=O.MINBEE, params=prm)
    with gpu.Solver(gpu.EULER, n, 1, prm, precision=gpu.MIXED) as s:
        s.upload(W)
        s.run(1.0 / n, 0.9, t_end=0.25, limiter=gpu.MINBEE)
        out = s.download()
    l1, linf = _errors(out[0], ref[0])
    print(f"sod mixed: L1(rho) {l1:.3e}  Linf(rho) {linf:.3e}")
    assert l1 <= L1_RHO
    assert linf <= 1e-3


def test_mixed_mhd_vortex(gpu, oracle_lib):
    nx = ny = 96
    W = wl.mhd_vortex_2d(nx, ny, seed=3)
    prm = wl.mhd_params(5.0 / 3.0)
    ref = W.copy()
    O.run(O.MHD, ref, 1.0 / nx, 0.8, steps=50, limiter=0, params=prm, bc=O.PERIODIC)
    with gpu.Solver(gpu.MHD, nx, ny, prm, precision=gpu.MIXED, boundary=gpu.PERIODIC) as s:
        s.upload(W)
        s.run(1.0 / nx, 0.8, steps=50, limiter=0)
        out = s.download()
    l1, linf = _errors(out[0], ref[0])
    print(f"mhd mixed: L1(rho) {l1:.3e}  Linf(rho) {linf:.3e}")
    assert l1 <= L1_RHO
    assert linf <= 1e-3


def _totals(model, W, prm):
    """Grid sums of mass, momentum and energy from primitive planes (cell volume 1)."""
    u = np.zeros((W.shape[0],) + W.shape[1:])
    flat = W.reshape(W.shape[0], -1)
    cons = np.empty_like(flat)
    for k in range(flat.shape[1]):
        cons[:, k] = _cons(model, flat[:, k], prm)
    del u
    return cons.sum(axis=1)


def _cons(model, w, prm):
    out = np.zeros_like(w)
    O.lib().vo_prim_to_cons(model, np.ascontiguousarray(w).ctypes.data_as(O._D), np.ascontiguousarray(prm).ctypes.data_as(O._D),
                            out.ctypes.data_as(O._D))
    return out


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("model", [0, 1])
def test_conservation_periodic(gpu, oracle_lib, precision, model):
    """Periodic boundaries: mass, momentum and energy change by round-off only."""
    nx = ny = 48
    if model == 0:
        W = wl.euler_quadrants_2d(nx, ny, seed=77)
        prm = wl.euler_params(1.4)
    else:
        W = wl.mhd_vortex_2d(nx, ny, seed=78)
        prm = wl.mhd_params(5.0 / 3.0)
    before = _totals(model, W, prm)
    with gpu.Solver(model, nx, ny, prm, precision=precision, boundary=gpu.PERIODIC) as s:
        s.upload(W)
        s.run(1.0 / nx, 0.8, steps=30, limiter=0)
        out = s.download()
    after = _totals(model, out, prm)
    idx = [0, 1, 2, 4] if model == 0 else [0, 1, 2, 4, 5, 6]
    scale = np.abs(before[idx]).max()
    drift = np.abs(after[idx] - before[idx]) / scale
    print(f"model {model} precision {precision}: relative drift {drift}")
    assert drift.max() <= 1e-12


@pytest.mark.parametrize("subcycles", [0, 2])
def test_mixed_hpr_smooth(gpu, oracle_lib, subcycles):
    """HPR mixed form: FP32 flux combinations, FP64 state, pressure recovery, acoustic-tensor CFL and relaxation
    source; against the FP64 oracle (with the RK4 source sub-cycled when subcycles > 0)."""
    nx, ny = 48, 40
    W = wl.hpr_smooth_2d(nx, ny, seed=31)
    prm = wl.hpr_params(tau1=1e-2, tau2=1e-2)
    ref = W.copy()
    O.run(O.HPR, ref, 1.0 / nx, 0.8, steps=20, limiter=0, params=prm, subcycles=subcycles)
    with gpu.Solver(gpu.HPR, nx, ny, prm, precision=gpu.MIXED) as s:
        s.upload(W)
        s.run(1.0 / nx, 0.8, steps=20, limiter=0, subcycles=subcycles)
        out = s.download()
    l1, linf = _errors(out[0], ref[0])
    print(f"hpr mixed sub{subcycles}: L1(rho) {l1:.3e}  Linf(rho) {linf:.3e}  L1(all) {np.abs(out - ref).mean():.3e}")
    assert l1 <= L1_RHO
    assert linf <= 1e-4
    assert np.abs(out - ref).mean() <= 1e-6


@pytest.mark.parametrize("precision", [0, 1])
def test_hpr_conservation_periodic(gpu, oracle_lib, precision):
    """Mass, momentum and total energy of HPR change by round-off only (the relaxation source moves only A and J)."""
    nx, ny = 40, 36
    W = wl.hpr_smooth_2d(nx, ny, seed=41)
    prm = wl.hpr_params(tau1=1e-2, tau2=1e-2)
    before = _totals(O.HPR, W, prm)
    with gpu.Solver(gpu.HPR, nx, ny, prm, precision=precision, boundary=gpu.PERIODIC) as s:
        s.upload(W)
        s.run(1.0 / nx, 0.8, steps=12, limiter=0, subcycles=1)
        out = s.download()
    after = _totals(O.HPR, out, prm)
    idx = [0, 1, 11, 12]
    scale = np.abs(before[idx]).max()
    drift = np.abs(after[idx] - before[idx]) / scale
    print(f"hpr precision {precision}: relative drift {drift}")
    assert drift.max() <= 1e-12


@pytest.mark.parametrize("shape", [(131, 37), (300, 2), (257, 1)])
@pytest.mark.parametrize("periodic", [False, True])
def test_tma_x_sweep_matches_plain_two_row_kernel(gpu, shape, periodic):
    """The TMA-staged X sweep (launch shapes 1 and 2 of the Euler mixed form) against the plain two-row kernel
    (shape 0), bit for bit, on grids whose edges cut tiles (odd rows, a partial last tile, 1D) for both boundary
    kinds: the ghost cells it patches after the zero-filled copy and the rows it computes but never stores."""
    nx, ny = shape
    W = wl.euler_quadrants_2d(nx, ny, seed=71) if ny > 1 else wl.sod_1d(nx)
    bc = gpu.PERIODIC if periodic else gpu.TRANSMISSIVE
    outs = []
    with gpu.Solver(gpu.EULER, nx, ny, wl.euler_params(1.4), precision=gpu.MIXED, boundary=bc) as s:
        for xc in (0, 1, 2):
            s.set_launch_config(xc, 0)
            assert (s.launch_config()[2].startswith("TMA")) == (xc > 0)
            s.upload(W)
            s.run(1.0 / nx, 0.8, steps=7, limiter=0)
            outs.append(s.download())
    assert np.isfinite(outs[0]).all()
    assert np.array_equal(outs[1], outs[0]) and np.array_equal(outs[2], outs[0])

