"""First-order FORCE loops (FirstOrderSolver / MHDFirstOrderSolver / HPRFirstOrderSolver::solve{,2D}) on the device,
bit for bit with the oracle, which is pinned to the reference (tests/test_oracle_pin.py)."""
import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _cases():
    return [
        ("euler1d", O.EULER, wl.sod_1d(300), wl.euler_params(1.4), 0),
        ("euler2d", O.EULER, wl.euler_quadrants_2d(150, 130, seed=3), wl.euler_params(1.4), 0),
        ("euler2d_periodic", O.EULER, wl.euler_quadrants_2d(130, 129, seed=4), wl.euler_params(1.4), 1),
        ("mhd2d_periodic", O.MHD, wl.mhd_vortex_2d(72, 64, seed=2), wl.mhd_params(5 / 3, c_h=1.3), 1),
        ("mhd1d", O.MHD, wl.brio_wu_1d(200), wl.mhd_params(2.0, c_h=0.7), 0),
        ("hpr2d", O.HPR, wl.hpr_smooth_2d(40, 36, seed=5), wl.hpr_params(), 0),
        ("hpr1d_periodic", O.HPR, wl.hpr_heat_conduction_1d(90), wl.hpr_params(), 1),
    ]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_first_order_matches_oracle(gpu, oracle_lib, case):
    _, model, W, prm, bc = case
    nx = W.shape[-1]
    ny = W.shape[1] if W.ndim == 3 else 1
    ref = W.copy()
    t_ref, n_ref = O.run_first_order(model, ref, 1.0 / nx, 0.8, steps=25, params=prm, bc=bc)
    with gpu.Solver(model, nx, ny, prm, boundary=bc) as s:
        s.upload(W)
        t, n = s.run(1.0 / nx, 0.8, steps=25, order=1)
        out = s.download()
    assert (t, n) == (t_ref, n_ref)
    assert np.array_equal(out, ref)


def test_first_order_time_driven(gpu, oracle_lib):
    W = wl.sod_1d(400)
    prm = wl.euler_params(1.4)
    ref = W.copy()
    t_ref, n_ref = O.run_first_order(O.EULER, ref, 1.0 / 400, 0.9, t_end=0.2, params=prm)
    with gpu.Solver(gpu.EULER, 400, 1, prm) as s:
        s.upload(W)
        t, n = s.run(1.0 / 400, 0.9, t_end=0.2, order=1)
        out = s.download()
    assert (t, n) == (t_ref, n_ref) and t == 0.2
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_first_order_mixed_form(gpu, case):
    """The mixed form of the first-order loop against its FP64 form: L1(rho) <= 1e-6, and on periodic grids mass is
    conserved to round-off (the FP32 interface fluxes telescope in the FP64 update)."""
    _, model, W, prm, bc = case
    nx = W.shape[-1]
    ny = W.shape[1] if W.ndim == 3 else 1
    outs = []
    for prec in (gpu.FP64, gpu.MIXED):
        with gpu.Solver(model, nx, ny, prm, boundary=bc, precision=prec) as s:
            s.upload(W)
            s.run(1.0 / nx, 0.8, steps=25, order=1)
            outs.append(s.download())
    fp64, mixed = outs
    l1 = np.abs(mixed[0] - fp64[0]).mean()
    print(f"first-order mixed L1(rho) {l1:.2e}")
    assert np.isfinite(mixed).all() and l1 <= 1e-6
    if bc == 1:
        assert abs(mixed[0].sum() - W[0].sum()) <= 1e-12 * W[0].sum()


def test_first_order_rejects_bad_order(gpu):
    with gpu.Solver(gpu.EULER, 64, 64, wl.euler_params(1.4), precision=gpu.MIXED) as s:
        s.upload(wl.euler_quadrants_2d(64, 64, seed=1))
        with pytest.raises(gpu.VgError):
            s.run(1.0 / 64, 0.8, steps=3, order=3)
