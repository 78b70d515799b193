"""The MHD multiphysics two-material model in the oracle (oracle/slic_oracle.c, M_MMPH) against the reference
(MHD/Multiphysics/mhdmultiphysicsstatevector.cpp through MHDSecondOrderSolver::solve and its per-step functions,
compiled into oracle/_ref): bit for bit on the reference's Dumbser layouts (one material, gamma 2; two, 1.4 | 1.67) and
seeded perturbations of them, with every limiter, a bias and non-zero hyperbolic wave speeds.  The reference has this
model in 1D only, and its loop runs no source and no reinitialisation."""
import numpy as np
import pytest

import oracle as O
import vanguard_b200 as vg
from vanguard_b200 import workloads as wl

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference not built (oracle/_ref)")
PRMS = {"one": wl.mhd_multiphysics_params(2.0, 0.0, 2.0, 0.0),
        "two": wl.mhd_multiphysics_params(1.4, 0.0, 1.67, 0.0),
        "glm": wl.mhd_multiphysics_params(1.4, 0.1, 1.67, 0.0, 0.5, 0.7)}


def _pair(W, prm, **kw):
    nx = W.shape[-1]
    a, b = W.copy(), W.copy()
    ta = O.run_two_material(O.MHD_MULTIPHYSICS, a, 1 / nx, 0.8, params=prm, **kw)
    tb = O.run_two_material(O.MHD_MULTIPHYSICS, b, 1 / nx, 0.8, params=prm, reference=True, **kw)
    return a, b, ta, tb


@needs_ref
@pytest.mark.parametrize("materials", list(PRMS))
@pytest.mark.parametrize("noise", [0.0, 1e-2])
@pytest.mark.parametrize("kw", [dict(steps=5, limiter=O.SUPERBEE), dict(steps=20, limiter=O.MINBEE, bias=0.3),
                                dict(steps=12, limiter=O.VANLEER)], ids=["superbee", "minbee_bias", "vanleer"])
def test_oracle_matches_reference(oracle_lib, materials, noise, kw):
    a, b, ta, tb = _pair(wl.mhd_multiphysics_dumbser_1d(60, seed=3, noise=noise), PRMS[materials], **kw)
    assert np.isfinite(a).all()
    assert ta == tb
    assert np.array_equal(a, b), f"max diff {np.abs(a - b).max():.3e}"


@needs_ref
def test_oracle_matches_reference_solve_t_end(oracle_lib):
    # MHDMultiphysicsTests::solveDumbserMultimaterialTest1's setting through the reference's own solve
    # (Solvers/mhdsecondordersolver.cpp:362-385), to t = 0.05
    a, b, ta, _ = _pair(wl.mhd_multiphysics_dumbser_1d(80), PRMS["two"], t_end=0.05, limiter=O.SUPERBEE)
    assert ta[0] == 0.05 and ta[1] > 10
    assert np.array_equal(a, b)


def test_no_source_no_reinitialisation(oracle_lib):
    # sub-cycles and a reinitialisation frequency are accepted and change nothing, as in the reference's loop
    W = wl.mhd_multiphysics_dumbser_1d(40, seed=2, noise=1e-2)
    a, b = W.copy(), W.copy()
    O.run_two_material(O.MHD_MULTIPHYSICS, a, 1 / 40, 0.8, steps=6, params=PRMS["glm"])
    O.run_two_material(O.MHD_MULTIPHYSICS, b, 1 / 40, 0.8, steps=6, params=PRMS["glm"], subcycles=2, reinit=2)
    assert np.array_equal(a, b)


def test_layouts():
    assert vg.NVAR[vg.MHD_MULTIPHYSICS] == 16 and vg.MHD_MULTIPHYSICS == O.MHD_MULTIPHYSICS == 10
    W = wl.mhd_multiphysics_dumbser_1d(10)
    assert W.shape == (16, 10)
    assert list(W[:, 0]) == [0.999, 0, 0, 0, 1.0, 1.0, 0.75, 1.0, 0, 0, 0.125, 0.1, 0.75, -1.0, 0, 0]
    assert W[0, 9] == 0.001
