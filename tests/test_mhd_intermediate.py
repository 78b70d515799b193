"""The MHD intermediate two-material model in the oracle (oracle/slic_oracle.c, M_MINT) against the reference
(MHD/Multiphysics/mhdintermediatestatevector.cpp through MHDSecondOrderSolver::solve and its per-step functions,
compiled into oracle/_ref): bit for bit on seeded cases beyond the golden fixtures; the 2D cases over mirror ghosts built
by the harness, because the reference's insertBoundaryCells2D for this model fills the outermost bottom ghost row from
the padded grid instead of the cells (Solvers/mhdsolvers.cpp:213)."""
import numpy as np
import pytest

import oracle as O
import vanguard_b200 as vg
from vanguard_b200 import workloads as wl

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference not built (oracle/_ref)")
PRM = wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0)


def _swirled(W, seed):
    rng = np.random.default_rng(seed)
    x = np.linspace(0.0, 1.0, W.shape[-1])
    W = W.copy()
    for plane, amp in ((3, 0.1), (10, 0.2), (11, 0.05)):
        W[plane] = W[plane] + amp * np.sin(2 * np.pi * (x + rng.uniform()))
    return W


@needs_ref
@pytest.mark.parametrize("case", ["superbee", "glm_reinit", "swirl_bias", "solve_t_end"])
def test_oracle_matches_reference_1d(oracle_lib, case):
    W = wl.mhd_intermediate_from_reduced(wl.mhd_reduced_dumbser_1d(96))
    kw = {
        "superbee": dict(steps=20, limiter=O.SUPERBEE),
        "glm_reinit": dict(steps=25, limiter=O.MINBEE, subcycles=3, reinit=2),
        "swirl_bias": dict(steps=20, limiter=1, bias=0.4, subcycles=1, reinit=5),
        "solve_t_end": dict(t_end=0.04, limiter=O.MINBEE, subcycles=2, reinit=3),
    }[case]
    if case == "swirl_bias":
        W = _swirled(W, 3)
    a, b = W.copy(), W.copy()
    ta = O.run_two_material(O.MHD_INTERMEDIATE, a, 1 / 96, 0.8, params=PRM, **kw)
    O.run_two_material(O.MHD_INTERMEDIATE, b, 1 / 96, 0.8, params=PRM, reference=True, **kw)
    assert np.array_equal(a, b), f"max diff {np.abs(a - b).max():.3e}"
    assert ta[0] > 0.0


@needs_ref
@pytest.mark.parametrize("sub,reinit", [(0, 0), (2, 2)])
def test_oracle_matches_reference_2d(oracle_lib, sub, reinit):
    W = wl.mhd_intermediate_from_reduced(wl.mhd_reduced_dumbser_2d(22, 18))
    W = np.stack([_swirled(W[:, r], seed=r) for r in range(W.shape[1])], axis=1)
    a, b = W.copy(), W.copy()
    kw = dict(steps=5, limiter=O.MINBEE, subcycles=sub, reinit=reinit)
    O.run_two_material(O.MHD_INTERMEDIATE, a, 1 / 22, 0.8, params=PRM, **kw)
    O.run_two_material(O.MHD_INTERMEDIATE, b, 1 / 22, 0.8, params=PRM, reference=True, **kw)
    assert np.array_equal(a, b), f"max diff {np.abs(a - b).max():.3e}"


def test_reinitialisation_relaxes_density_and_pressure(oracle_lib):
    W = wl.mhd_intermediate_from_reduced(wl.mhd_reduced_dumbser_1d(100))
    O.run_two_material(O.MHD_INTERMEDIATE, W, 1 / 100, 0.8, steps=4, limiter=O.MINBEE, params=PRM, reinit=4)
    a = W[0]
    loc = max(i for i in range(1, 100) if a[i] < 0.5 <= a[i - 1])
    assert list(a[loc - 2:loc + 2]) == [0.999, 0.999, 0.001, 0.001]
    assert np.array_equal(W[4, loc - 2:loc + 2], W[6, loc - 2:loc + 2])
    assert np.array_equal(W[5, loc - 2:loc + 2], W[7, loc - 2:loc + 2])


def test_layouts():
    assert vg.NVAR[vg.MHD_INTERMEDIATE] == wl.MHD_INTERMEDIATE_NVAR == 12
    R = wl.mhd_reduced_dumbser_1d(10)
    W = wl.mhd_intermediate_from_reduced(R)
    assert np.array_equal(W[5], R[6]) and np.array_equal(W[7], R[6]) and np.array_equal(W[6], R[5])
    assert np.array_equal(W[8:], R[7:])
