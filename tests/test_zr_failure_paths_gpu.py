"""Failure paths: states poisoned on the host, reported through the C ABI's status codes.

The reference has no error reporting: solve() and the per-sweep functions return whatever the arithmetic gives,
NaN and negative pressures included (Solvers/secondordersolver.cpp:288-314).  The device keeps those results bit
for bit, NaN where the reference has NaN (in the planes it does not carry too: a non-finite cell's w and lambda
are NaN in the reference), and, in addition, flags every update that leaves a non-finite value, a non-positive
density or a pressure at or below -p_inf: vg_run and vg_solve return VG_ENAN after the run, and vg_solve still
delivers the planes.  No device fault is involved: the poison is ordinary floating-point data.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _same_with_nan(a, b):
    """Bit-equal values, NaN where the oracle has NaN."""
    assert np.array_equal(np.isnan(a), np.isnan(b)), "NaN patterns differ"
    m = ~np.isnan(b)
    assert np.array_equal(a[m], b[m])


@pytest.mark.parametrize("poison", ["nan_density", "negative_pressure", "inf_velocity"])
def test_poisoned_cell_reports_enan(gpu, oracle_lib, poison):
    nx, ny = 64, 48
    W = wl.euler_quadrants_2d(nx, ny, seed=3)
    if poison == "nan_density":
        W[0, 20, 30] = np.nan
    elif poison == "negative_pressure":
        W[4, 18:26, 26:34] = -0.5   # a block: its inner cells stay uniform, so the first sweep keeps them negative
    else:
        W[1, 20, 30] = np.inf
    prm = wl.euler_params(1.4)
    ref = W.copy()
    O.run(O.EULER, ref, 1.0 / nx, 0.8, steps=3, limiter=O.SUPERBEE, params=prm)
    with gpu.Solver(gpu.EULER, nx, ny, prm) as s:
        s.upload(W)
        with pytest.raises(gpu.VgError) as e:
            s.run(1.0 / nx, 0.8, steps=3)
        assert e.value.status == gpu.VG_ENAN
        out = s.download()
        _same_with_nan(out, ref)
        # the handle stays usable: a clean state runs without error afterwards
        s.upload(wl.euler_quadrants_2d(nx, ny, seed=4))
        s.run(1.0 / nx, 0.8, steps=2)
    # vg_solve: the status is VG_ENAN and the planes are still downloaded
    c = gpu.RunConfig(1.0 / nx, 0.8, 0.0, 3, 0.0, 0, 0, 2, 0, 0)
    out = np.empty_like(W)
    with gpu.Solver(gpu.EULER, nx, ny, prm) as s:
        st = gpu.lib().vg_solve(s._h, W.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p),
                                ctypes.byref(c), None, None, None)
    assert st == gpu.VG_ENAN
    _same_with_nan(out, ref)


def test_poisoned_mhd_and_hpr_report_enan(gpu):
    """The same status from the MHD and HPR loops (NaN density in one interior cell)."""
    W = wl.mhd_vortex_2d(40, seed=1)
    W[0, 10, 12] = np.nan
    with gpu.Solver(gpu.MHD, 40, 40, wl.mhd_params(), boundary=gpu.PERIODIC) as s:
        s.upload(W)
        with pytest.raises(gpu.VgError) as e:
            s.run(1.0 / 40, 0.8, steps=2)
        assert e.value.status == gpu.VG_ENAN
    W = wl.hpr_smooth_2d(24, 20, seed=2)
    W[0, 5, 7] = np.nan
    with gpu.Solver(gpu.HPR, 24, 20, wl.hpr_params()) as s:
        s.upload(W)
        with pytest.raises(gpu.VgError) as e:
            s.run(1.0 / 24, 0.8, steps=2, subcycles=1)
        assert e.value.status == gpu.VG_ENAN


def test_poisoned_batch_instance_reports_enan(gpu):
    """A NaN in one instance of the ragged batch: the run reports VG_ENAN; the other instances are unaffected."""
    ncell = np.array([50, 80, 64])
    dx = 1.0 / ncell
    gamma = np.array([1.4, 1.3, 1.5])
    theta = np.tile([1.0, 0.0, 1.0, 0.125, 0.0, 0.1], (3, 1))
    W = wl.batch_planes(ncell, theta)
    with gpu.Batch(ncell, dx, gamma) as b:
        b.upload(W)
        clean = b.run(0.8, 5)
        ref = b.download()
        Wp = W.copy()
        Wp[0, 60] = np.nan          # instance 1
        b.upload(Wp)
        with pytest.raises(gpu.VgError) as e:
            b.run(0.8, 5)
        assert e.value.status == gpu.VG_ENAN
        out = b.download()
    assert np.array_equal(out[:, :50], ref[:, :50])
    assert np.array_equal(out[:, 130:], ref[:, 130:])
    assert np.isnan(out[:, 50:130]).any()
    assert np.isfinite(clean).all()
