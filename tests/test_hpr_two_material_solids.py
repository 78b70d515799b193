"""The HPR two-material models (reduced, intermediate, multiphysics) with solid materials, the reference's own scenarios
for them (HPR/Multiphysics/hprreducedtests.cpp, hprintermediatetests.cpp, hprmultiphysicstests.cpp): the oracle
(oracle/slic_oracle.c) against the reference (compiled into oracle/_ref) bit for bit with ShockMieGruneisen solids,
elastic and plastic, thermal and cold, with the relaxation sub-cycles, a bias, the reinitialisation, and in 2D.

GodunovRomenski solids, the equation of state of the reference's Barton and Zhang scenarios, run in the oracle only:
the reference's acoustic tensors of these models (HPR/Multiphysics/hprreducedacoustictensor.cpp and its siblings) call
computeGruneisenCoefficientDerivative, which has no GodunovRomenski return (HPR/hprmiegruneisen.cpp:104-119), and
compiled with -O2 that call does not return.  The oracle takes that branch's derivative as 0 (its Grueneisen
coefficient is the constant gamma); the single-material functions it builds on are pinned to the reference in
test_hpr_solids.py.

Cases are chosen to stay finite (a run that goes non-finite before a 1D reinitialisation corrupts the reference's
heap)."""
import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference not built (oracle/_ref)")

ELASTIC1 = wl.hpr_shock_mg_params(tau1=0.05)
ELASTIC2 = wl.hpr_shock_mg_params(tau1=0.5)
PLASTIC2 = wl.hpr_shock_mg_params(plastic=True, sigma0=0.3, n=2.0, tau1=1.0)
MILD_PLASTIC2 = wl.hpr_shock_mg_params(plastic=True, sigma0=1.0, n=1.0, tau1=1.0)
THERMAL1 = wl.hpr_shock_mg_params(tau1=0.05, thermal=True)
COLD2 = wl.hpr_shock_mg_params(tau1=1.0)
ZHANG_V = ((0.0, 0.2, 0.1), (0.0, -0.03, -0.01))
BARTON_V = ((0.0, 0.3, 0.5), (0.0, 0.0, 0.0))
MODELS = [O.HPR_REDUCED, O.HPR_INTERMEDIATE, O.HPR_MULTIPHYSICS]
MODEL_IDS = ["reduced", "intermediate", "multiphysics"]


def planes(model, W):
    """The HPR reduced planes W in `model`'s layout."""
    if model == O.HPR_INTERMEDIATE:
        return wl.hpr_intermediate_from_reduced(W)
    if model == O.HPR_MULTIPHYSICS:
        return wl.hpr_multiphysics_from_reduced(W)
    return W


def solids(model, m1, m2, F, v, nx, ny=1, heat=0.0):
    return planes(model, wl.hpr_two_solid_riemann(nx, m1, m2, *F, *v, ny=ny, heat=heat, seed=nx))


def _pair(model, W, nx, prm, **kw):
    a, b = W.copy(), W.copy()
    ta = O.run_two_material(model, a, 1 / nx, 0.8, params=prm, **kw)
    tb = O.run_two_material(model, b, 1 / nx, 0.8, params=prm, reference=True, **kw)
    return a, b, ta, tb


CASES_1D = {
    "elastic_minbee": (ELASTIC1, ELASTIC2, wl.ZHANG_F, ZHANG_V, 0.0, dict(steps=20, limiter=O.MINBEE)),
    "elastic_superbee_sub1": (ELASTIC1, ELASTIC2, wl.ZHANG_F, ZHANG_V, 0.0,
                              dict(steps=20, limiter=O.SUPERBEE, subcycles=1)),
    "elastic_sub1_reinit3": (ELASTIC1, ELASTIC2, wl.ZHANG_F, ZHANG_V, 0.0,
                             dict(steps=20, limiter=O.MINBEE, subcycles=1, reinit=3)),
    "plastic_bias_sub2_reinit3": (ELASTIC1, PLASTIC2, wl.ZHANG_F, ZHANG_V, 0.0,
                                  dict(steps=20, limiter=O.MINBEE, subcycles=2, reinit=3, bias=0.2)),
    "plastic_superbee_sub1": (ELASTIC1, PLASTIC2, wl.BARTON_F, BARTON_V, 0.0,
                              dict(steps=20, limiter=O.SUPERBEE, subcycles=1)),
    "thermal_vanleer_sub1": (THERMAL1, COLD2, wl.BARTON_F, BARTON_V, 0.05,
                             dict(steps=12, limiter=O.VANLEER, subcycles=1)),
}


@needs_ref
@pytest.mark.parametrize("case", list(CASES_1D))
@pytest.mark.parametrize("model", MODELS, ids=MODEL_IDS)
def test_solids_oracle_matches_reference_1d(oracle_lib, model, case):
    m1, m2, F, v, heat, kw = CASES_1D[case]
    a, b, ta, tb = _pair(model, solids(model, m1, m2, F, v, 60, heat=heat), 60, wl.hpr_two_params(m1, m2), **kw)
    assert np.isfinite(a).all()
    assert ta == tb
    assert np.array_equal(a, b), f"max diff {np.abs(a - b).max():.3e}"


@needs_ref
@pytest.mark.parametrize("model,kw", [
    (O.HPR_REDUCED, dict(t_end=0.02, limiter=O.MINBEE, subcycles=2, reinit=4)),
    (O.HPR_INTERMEDIATE, dict(t_end=0.03, limiter=O.MINBEE, reinit=3)),
    (O.HPR_MULTIPHYSICS, dict(t_end=0.03, limiter=O.MINBEE, subcycles=1, reinit=3)),
], ids=MODEL_IDS)
def test_solids_oracle_matches_reference_solve(oracle_lib, model, kw):
    # the reference's own HPRSecondOrderSolver::solve to t_end, the plastic pair of its Zhang layout
    a, b, ta, _ = _pair(model, solids(model, ELASTIC1, PLASTIC2, wl.ZHANG_F, ZHANG_V, 60), 60,
                        wl.hpr_two_params(ELASTIC1, PLASTIC2), **kw)
    assert ta[0] == kw["t_end"] and ta[1] > 5
    assert np.isfinite(a).all()
    assert np.array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("m2,kw", [
    (ELASTIC2, dict(steps=6, limiter=O.MINBEE, subcycles=1, reinit=2, bias=-0.2)),
    (MILD_PLASTIC2, dict(steps=6, limiter=O.SUPERBEE, subcycles=2)),
], ids=["elastic_sub1_reinit2", "plastic_sub2"])
@pytest.mark.parametrize("model", MODELS[:2], ids=MODEL_IDS[:2])
def test_solids_oracle_matches_reference_2d(oracle_lib, model, m2, kw):
    a, b, ta, tb = _pair(model, solids(model, ELASTIC1, m2, wl.BARTON_F, BARTON_V, 16, ny=12), 16,
                         wl.hpr_two_params(ELASTIC1, m2), **kw)
    assert np.isfinite(a).all()
    assert ta == tb
    assert np.array_equal(a, b)


@pytest.mark.parametrize("model", MODELS, ids=MODEL_IDS)
@pytest.mark.parametrize("scenario", ["barton", "zhang"])
def test_godunov_romenski_runs_in_the_oracle(oracle_lib, model, scenario):
    # the reference's Barton (copper | copper) and Zhang (plastic aluminium | copper) materials and layouts
    cu = wl.hpr_barton_params()
    m1, F, v = (cu, wl.BARTON_F, ((0.0, 0.5, 1.0), (0.0, 0.0, 0.0))) if scenario == "barton" else \
        (wl.hpr_zhang_params(), wl.ZHANG_F, ((2.0, 0.0, 0.1), (0.0, -0.03, -0.01)))
    W = solids(model, m1, cu, F, v, 60)
    W0 = W.copy()
    t, n = O.run_two_material(model, W, 1 / 60, 0.8, params=wl.hpr_two_params(m1, cu), steps=20, limiter=O.MINBEE,
                              subcycles=1)
    assert n == 20 and t > 0.0
    assert np.isfinite(W).all() and not np.array_equal(W, W0)


def test_solid_parameter_layout():
    prm = wl.hpr_two_params(wl.hpr_zhang_params(), wl.hpr_barton_params())
    assert prm.shape == (40,)
    assert prm[12] == prm[32] == wl.HPR_EOS["GodunovRomenski"]
    assert prm[17] == 1.0 and prm[37] == 0.0  # aluminium plastic, copper elastic
    assert prm[3] == 2.71 and prm[23] == 8.9
    with pytest.raises(AssertionError):
        wl.hpr_two_params(prm[:20], prm[:11])


def test_solid_riemann_layout():
    W = wl.hpr_two_solid_riemann(20, ELASTIC1, PLASTIC2, *wl.ZHANG_F, *ZHANG_V)
    left = np.arange(20) <= 10
    assert W.shape == (19, 20)
    assert (W[0][left] == 0.999).all() and (W[0][~left] == 0.001).all()
    A = np.linalg.inv(np.array(wl.ZHANG_F[0]))
    assert np.allclose(W[2:11, 0], A.reshape(9))
    assert np.isclose(W[17, 0], ELASTIC1[3] * np.linalg.det(A))
    assert np.isclose(W[1, 0], wl.smg_reference_pressure(W[17, 0], ELASTIC1))
    W2 = wl.hpr_two_solid_riemann(16, ELASTIC1, PLASTIC2, *wl.ZHANG_F, *ZHANG_V, ny=12)
    assert W2.shape == (19, 12, 16) and np.array_equal(W2[:, 5], wl.hpr_two_solid_riemann(16, ELASTIC1, PLASTIC2, *wl.ZHANG_F, *ZHANG_V))
