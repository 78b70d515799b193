"""The MHD reduced two-material model in the oracle (oracle/slic_oracle.c, M_MRED) against the reference
(MHD/Multiphysics/mhdreducedstatevector.cpp through MHDSecondOrderSolver::solve{,2D} and its per-step functions,
compiled into oracle/_ref): bit for bit on seeded cases beyond the golden fixtures (every limiter, a bias, a stiffened
material, non-zero w / Bz / psi, GLM damping sub-cycles, reinitialisation); and the host-side layouts."""
import numpy as np
import pytest

import oracle as O
import vanguard_b200 as vg
from vanguard_b200 import workloads as wl

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference not built (oracle/_ref)")


def _swirled(W, seed):
    rng = np.random.default_rng(seed)
    x = np.linspace(0.0, 1.0, W.shape[-1])
    W = W.copy()
    for plane, amp in ((3, 0.1), (9, 0.2), (10, 0.05)):
        W[plane] = W[plane] + amp * np.sin(2 * np.pi * (x + rng.uniform()))
    return W


@needs_ref
@pytest.mark.parametrize("case", ["one_material", "two_materials_glm", "stiffened_swirl", "bias_vanleer"])
def test_oracle_matches_reference_1d(oracle_lib, case):
    prm, W, kw = {
        "one_material": (wl.mhd_reduced_params(), wl.mhd_reduced_dumbser_1d(110),
                         dict(steps=25, limiter=O.SUPERBEE)),
        "two_materials_glm": (wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0), wl.mhd_reduced_dumbser_1d(110),
                              dict(steps=25, limiter=O.MINBEE, subcycles=3, reinit=2)),
        "stiffened_swirl": (wl.mhd_reduced_params(2.0, 0.0, 1.67, 0.3), _swirled(wl.mhd_reduced_dumbser_1d(90), 1),
                            dict(steps=20, limiter=0, subcycles=1, reinit=4)),
        "bias_vanleer": (wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0), _swirled(wl.mhd_reduced_dumbser_1d(80), 2),
                         dict(steps=20, limiter=1, bias=0.4, subcycles=2)),
    }[case]
    a, b = W.copy(), W.copy()
    dx = 1.0 / W.shape[-1]
    ta = O.run_two_material(O.MHD_REDUCED, a, dx, 0.8, params=prm, **kw)
    tb = O.run_two_material(O.MHD_REDUCED, b, dx, 0.8, params=prm, reference=True, **kw)
    assert ta == tb
    assert np.array_equal(a, b), f"max diff {np.abs(a - b).max():.3e}"


@needs_ref
def test_oracle_matches_reference_2d(oracle_lib):
    prm = wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0)
    W = wl.mhd_reduced_dumbser_2d(22, 18)
    W = np.stack([_swirled(W[:, r], seed=r) for r in range(W.shape[1])], axis=1)
    a, b = W.copy(), W.copy()
    kw = dict(steps=5, limiter=O.MINBEE, subcycles=2, reinit=2)
    O.run_two_material(O.MHD_REDUCED, a, 1 / 22, 0.8, params=prm, **kw)
    O.run_two_material(O.MHD_REDUCED, b, 1 / 22, 0.8, params=prm, reference=True, **kw)
    assert np.array_equal(a, b), f"max diff {np.abs(a - b).max():.3e}"


def test_reinitialisation_resets_the_interface(oracle_lib):
    """After a reinitialisation step the four cells about the last descending crossing carry pure volume fractions
    and equal material densities (relaxTotalDensity)."""
    prm = wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0)
    W = wl.mhd_reduced_dumbser_1d(100)
    O.run_two_material(O.MHD_REDUCED, W, 1 / 100, 0.8, steps=4, limiter=O.MINBEE, params=prm, reinit=4)
    a = W[0]
    loc = max(i for i in range(1, 100) if a[i] < 0.5 <= a[i - 1])
    assert list(a[loc - 2:loc + 2]) == [0.999, 0.999, 0.001, 0.001]
    assert np.array_equal(W[4, loc - 2:loc + 2], W[5, loc - 2:loc + 2])


def test_layouts():
    assert vg.NVAR[vg.MHD_REDUCED] == wl.MHD_REDUCED_NVAR == 11
    W = wl.mhd_reduced_dumbser_1d(10)
    assert W.shape == (11, 10) and W[0, 5] == 0.999 and W[0, 6] == 0.001 and W[8, 6] == -1.0
    W2 = wl.mhd_reduced_dumbser_2d(20, 16)
    assert W2.shape == (11, 16, 20) and W2[0, 8, 10] == 0.999 and W2[0, 0, 0] == 0.001
