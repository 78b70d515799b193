"""The Euler reduced two-material model (EulerReducedStateVector with SecondOrderSolver::solve{,2D} and
MultiphysicsSolvers::reinitialiseVolumeFraction) in the oracle against the reference, bit for bit: the reference's
own time-driven solve, step-driven runs through its per-step functions, both material pairs of its scenarios
(Euler/Multiphysics/eulerreducedtests.cpp), 1D and 2D, with and without reinitialisation."""
import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference not built (oracle/_ref)")


def _both(W, dx, **kw):
    ours, ref = W.copy(), W.copy()
    r1 = O.run_reduced(ours, dx, 0.8, **kw)
    r2 = O.run_reduced(ref, dx, 0.8, reference=True, **kw)
    return ours, ref, r1, r2


@needs_ref
@pytest.mark.parametrize("gammas", [(1.4, 1.4), (1.4, 1.67)])
@pytest.mark.parametrize("limiter", [0, 1, 2])
def test_reduced_1d_time_driven(oracle_lib, gammas, limiter):
    W = wl.reduced_shock_tube(90)
    prm = wl.reduced_params(gammas[0], 0.0, gammas[1], 0.0)
    ours, ref, (t1, _), (t2, _) = _both(W, 1 / 90, t_end=0.04, limiter=limiter, params=prm)
    assert np.isfinite(ours).all() and np.array_equal(ours, ref)


@needs_ref
@pytest.mark.parametrize("reinit", [0, 1, 4])
def test_reduced_1d_steps_and_reinitialisation(oracle_lib, reinit):
    W = wl.reduced_shock_tube(110, rho=(1.0, 0.1379), p=(2.0, 1.0))
    ours, ref, (_, n1), (_, n2) = _both(W, 1 / 110, steps=25, limiter=0, params=wl.reduced_params(1.4, 0.0, 1.67, 0.0),
                                        reinit=reinit)
    assert n1 == n2 == 25
    assert np.array_equal(ours, ref)


@needs_ref
@pytest.mark.parametrize("reinit", [0, 2])
def test_reduced_2d(oracle_lib, reinit):
    W = wl.reduced_bubble_2d(26, 22)
    ours, ref, _, _ = _both(W, 1 / 26, steps=7, limiter=2, params=wl.reduced_params(1.4, 0.0, 1.67, 0.0),
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
