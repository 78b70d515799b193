"""The one-launch 1D loop (solve1d_kernels.cuh): a plain second-order exact-FP64 Euler run of a row of 16 .. 2032
cells runs entirely inside one thread-block cluster.  Bit for bit against the oracle (and so against the graph-driven
loop, which the row of 2033 cells still takes) for both boundary kinds, every limiter, a bias, time- and step-driven
runs, rows that leave the last blocks of the cluster short or empty, and a stiffened gas; one launch per run."""
import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _device(gpu, W, prm, dx, boundary, **run):
    with gpu.Solver(gpu.EULER, W.shape[1], 1, prm, boundary=boundary) as s:
        s.upload(W)
        t, n = s.run(dx, 0.8, **run)
        return s.download(), t, n, s.last_launch_count()


def _bitwise(a, b):
    assert np.array_equal(a, b), f"max diff {np.nanmax(np.abs(a - b)):.3e}"


@pytest.mark.parametrize("nx", [16, 17, 23, 100, 1000, 2031, 2032, 2033])
@pytest.mark.parametrize("periodic", [False, True])
def test_sod_time_driven_matches_oracle(gpu, oracle_lib, nx, periodic):
    W = wl.sod_1d(nx)
    prm = wl.euler_params(1.4)
    bc = gpu.PERIODIC if periodic else gpu.TRANSMISSIVE
    ref = W.copy()
    t_ref, n_ref = O.run(O.EULER, ref, 1.0 / nx, 0.8, t_end=0.1, limiter=O.MINBEE, params=prm,
                         bc=O.PERIODIC if periodic else O.TRANSMISSIVE)
    out, t, n, launches = _device(gpu, W, prm, 1.0 / nx, bc, t_end=0.1, limiter=O.MINBEE)
    assert (t, n) == (t_ref, n_ref)
    _bitwise(out, ref)
    if nx <= 2032:
        assert launches == 1
    else:
        assert launches > n  # the graph-driven loop: at least one kernel per step plus the first maximum


@pytest.mark.parametrize("limiter", [O.SUPERBEE, O.VANLEER, O.MINBEE])
@pytest.mark.parametrize("bias", [0.0, 0.4, -0.7])
def test_seeded_riemann_step_driven_matches_oracle(gpu, oracle_lib, limiter, bias):
    rng = np.random.default_rng(int(10 * bias) + limiter + 7)
    nx = 777
    W = wl.sod_1d(nx)
    left = np.arange(nx) <= nx / 2
    W[0] = np.where(left, rng.uniform(0.1, 2.0), rng.uniform(0.1, 2.0))
    W[1] = np.where(left, rng.uniform(-1, 1), rng.uniform(-1, 1))
    W[4] = np.where(left, rng.uniform(0.1, 10.0), rng.uniform(0.1, 10.0))
    prm = wl.euler_params(1.3, 0.4)  # stiffened gas
    ref = W.copy()
    O.run(O.EULER, ref, 1.0 / nx, 0.8, steps=150, limiter=limiter, bias=bias, params=prm)
    out, t, n, launches = _device(gpu, W, prm, 1.0 / nx, gpu.TRANSMISSIVE, steps=150, limiter=limiter, bias=bias)
    assert n == 150 and launches == 1
    _bitwise(out, ref)


def test_runs_continue_where_they_stopped(gpu, oracle_lib):
    # two calls of 40 and 60 steps: the second starts from the first's state with the dt schedule restarted, as the
    # reference's solve does when called twice
    nx = 1000
    W = wl.sod_1d(nx)
    prm = wl.euler_params(1.4)
    ref = W.copy()
    O.run(O.EULER, ref, 1e-3, 0.9, steps=40, limiter=O.MINBEE, params=prm)
    O.run(O.EULER, ref, 1e-3, 0.9, steps=60, limiter=O.MINBEE, params=prm)
    with gpu.Solver(gpu.EULER, nx, 1, prm) as s:
        s.upload(W)
        s.run(1e-3, 0.9, steps=40, limiter=O.MINBEE)
        s.run(1e-3, 0.9, steps=60, limiter=O.MINBEE)
        out = s.download()
    _bitwise(out, ref)


def _same_with_nan(a, b):
    assert np.array_equal(np.isnan(a), np.isnan(b))
    assert np.array_equal(np.nan_to_num(a, nan=0.0), np.nan_to_num(b, nan=0.0))


@pytest.mark.parametrize("nx", [600, 2033])
@pytest.mark.parametrize("poison", ["nan_density", "negative_pressure"])
def test_poisoned_row_reports_enan(gpu, oracle_lib, nx, poison):
    # the one-launch loop (600 cells) and the graph-driven one (2033) report VG_ENAN alike and leave the same state
    W = wl.sod_1d(nx)
    if poison == "nan_density":
        W[0, 200] = np.nan
    else:
        W[4, 150:170] = -0.5
    prm = wl.euler_params(1.4)
    ref = W.copy()
    O.run(O.EULER, ref, 1.0 / nx, 0.8, steps=4, limiter=O.MINBEE, params=prm)
    with gpu.Solver(gpu.EULER, nx, 1, prm) as s:
        s.upload(W)
        with pytest.raises(gpu.VgError) as e:
            s.run(1.0 / nx, 0.8, steps=4, limiter=O.MINBEE)
        assert e.value.status == gpu.VG_ENAN
        _same_with_nan(s.download(), ref)
        s.upload(wl.sod_1d(nx))  # the handle stays usable
        t, n = s.run(1.0 / nx, 0.8, steps=3, limiter=O.MINBEE)
        assert n == 3
