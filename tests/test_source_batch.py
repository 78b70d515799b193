"""The homogeneous HPR relaxation batch, CPU side: its tangent-linear reference (oracle/tangent_source.py) against
the oracle's forcing on uniform fields and against central finite differences of itself."""
import numpy as np
import pytest

import oracle as O
from oracle import tangent_source as TS
from vanguard_b200 import workloads as wl


def _forcing_uniform(W, tau, prm, h, steps):
    """The oracle's RK4 forcing sub-cycle (HPRForcingSolver on a grid) applied to each cell as a uniform 2-cell
    field, zero limiter bias: the reference's source step of a homogeneous state."""
    out = np.empty_like(W)
    for c in range(W.shape[1]):
        p = prm.copy()
        p[7], p[8] = tau[0, c], tau[1, c]
        g = np.repeat(W[:, c:c + 1], 2, axis=1).copy()
        for _ in range(steps):
            O.forcing(g, 0.1, h, bias=0.0, limiter=O.SUPERBEE, params=p)
        assert np.array_equal(g[:, 0], g[:, 1])
        out[:, c] = g[:, 0]
    return out


@pytest.mark.parametrize("thermal", [True, False])
def test_tangent_value_is_the_reference_forcing(oracle_lib, thermal):
    W, tau, prm = wl.hpr_relaxation_cells(12, seed=3, thermal=thermal)
    h, steps = 2e-4, 6
    ref = _forcing_uniform(W, tau, prm, h, steps)
    val, _ = TS.jvp(W, tau, prm, h, steps)
    rel = np.abs(val - ref) / np.maximum(np.abs(ref), 1e-300)
    assert rel.max() <= 1e-13, rel.max()


@pytest.mark.parametrize("thermal", [True, False])
def test_tangent_matches_central_differences(thermal):
    W, tau, prm = wl.hpr_relaxation_cells(8, seed=4, thermal=thermal)
    h, steps, eps = 3e-4, 10, 1e-6
    rng = np.random.default_rng(1)
    dW = rng.standard_normal(W.shape)
    if not thermal:
        dW[14:17] = 0.0
    dtau = tau * rng.standard_normal(tau.shape)
    _, tan = TS.jvp(W, tau, prm, h, steps, dW, dtau)
    plus, _ = TS.jvp(W + eps * dW, tau + eps * dtau, prm, h, steps)
    minus, _ = TS.jvp(W - eps * dW, tau - eps * dtau, prm, h, steps)
    fd = (plus - minus) / (2 * eps)
    err = np.abs(fd - tan).max() / np.abs(tan).max()
    assert err <= 1e-6, err
