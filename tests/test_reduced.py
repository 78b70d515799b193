"""The Euler two-material models (EulerReducedStateVector and EulerMultiphysicsStateVector with
SecondOrderSolver::solve{,2D} and MultiphysicsSolvers::reinitialiseVolumeFraction) in the oracle against the
reference, bit for bit: the reference's own time-driven solve, step-driven runs through its per-step functions, both
material pairs of its scenarios (Euler/Multiphysics/eulerreducedtests.cpp, eulermultiphysicstests.cpp), 1D and 2D,
with and without reinitialisation."""
import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference not built (oracle/_ref)")


MODELS = [O.EULER_REDUCED, O.EULER_MULTIPHYSICS]


def _planes(model, W):
    return W if model == O.EULER_REDUCED else wl.multiphysics_from_reduced(W)


def _both(W, dx, model=O.EULER_REDUCED, **kw):
    W = _planes(model, W)
    ours, ref = W.copy(), W.copy()
    r1 = O.run_two_material(model, ours, dx, 0.8, **kw)
    r2 = O.run_two_material(model, ref, dx, 0.8, reference=True, **kw)
    return ours, ref, r1, r2


@needs_ref
@pytest.mark.parametrize("model", MODELS)
@pytest.mark.parametrize("gammas", [(1.4, 1.4), (1.4, 1.67)])
@pytest.mark.parametrize("limiter", [0, 1, 2])
def test_reduced_1d_time_driven(oracle_lib, model, gammas, limiter):
    W = wl.reduced_shock_tube(90)
    prm = wl.reduced_params(gammas[0], 0.0, gammas[1], 0.0)
    ours, ref, (t1, _), (t2, _) = _both(W, 1 / 90, model, t_end=0.04, limiter=limiter, params=prm)
    assert np.isfinite(ours).all() and np.array_equal(ours, ref)


@needs_ref
@pytest.mark.parametrize("model", MODELS)
@pytest.mark.parametrize("reinit", [0, 1, 4])
def test_reduced_1d_steps_and_reinitialisation(oracle_lib, model, reinit):
    W = wl.reduced_shock_tube(110, rho=(1.0, 0.1379), p=(2.0, 1.0))
    ours, ref, (_, n1), (_, n2) = _both(W, 1 / 110, model, steps=25, limiter=0,
                                        params=wl.reduced_params(1.4, 0.0, 1.67, 0.0), reinit=reinit)
    assert n1 == n2 == 25
    assert np.array_equal(ours, ref)


@needs_ref
@pytest.mark.parametrize("model", MODELS)
@pytest.mark.parametrize("reinit", [0, 2])
def test_reduced_2d(oracle_lib, model, reinit):
    W = wl.reduced_bubble_2d(26, 22)
    ours, ref, _, _ = _both(W, 1 / 26, model, steps=7, limiter=2, params=wl.reduced_params(1.4, 0.0, 1.67, 0.0),
                            reinit=reinit)
    assert np.array_equal(ours, ref)


def test_reduced_conserves_mass_per_material(oracle_lib):
    """Without reinitialisation the update is conservative in every conserved component: alpha_k rho_k summed over a
    periodic-free closed tube stays put while no wave has reached the ends."""
    W = wl.reduced_shock_tube(200)
    prm = wl.reduced_params(1.4, 0.0, 1.67, 0.0)
    m0 = (W[0] * W[4]).sum(), ((1 - W[0]) * W[5]).sum()
    O.run_reduced(W, 1 / 200, 0.8, steps=20, limiter=0, params=prm)
    m1 = (W[0] * W[4]).sum(), ((1 - W[0]) * W[5]).sum()
    assert np.allclose(m0, m1, rtol=1e-13)
