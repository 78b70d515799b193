"""The FP64 tangent-linear reference used to check the adjoint: its value part is the oracle's forward bit for
bit, its full gradient agrees with its own directional derivatives, and both agree with central finite
differences along the Riemann-state and gamma directions (where no CFL-maximum ties make the loss kinked)."""
import numpy as np
import pytest

import oracle as O
from oracle import tangent
from vanguard_b200 import workloads as wl


@pytest.mark.parametrize("limiter", [0, 1, 2])
def test_value_part_is_oracle_forward(oracle_lib, limiter):
    ncell, dx, gamma, theta, W0 = wl.ragged_riemann_batch(ninst=3, seed=limiter, nmin=2, nmax=70)
    steps = 9
    _, _, rho_T = tangent.jvp(ncell, dx, gamma, W0, np.zeros(W0.shape[1]), 0.8, steps, 0.0, limiter)
    off = 0
    for k, n in enumerate(ncell):
        ref = np.ascontiguousarray(W0[:, off:off + n])
        O.run(O.EULER, ref, dx[k], 0.8, steps=steps, limiter=limiter, params=wl.euler_params(gamma[k]))
        assert np.array_equal(ref[0], rho_T[off:off + n])
        off += n


def test_full_gradient_consistent_with_jvp():
    ncell = np.array([2, 7, 30])
    rng = np.random.default_rng(0)
    gamma = rng.uniform(1.2, 1.67, 3)
    theta = np.stack([rng.uniform(0.1, 2, 3), rng.uniform(-1, 1, 3), rng.uniform(0.1, 10, 3),
                      rng.uniform(0.1, 2, 3), rng.uniform(-1, 1, 3), rng.uniform(0.1, 10, 3)], 1)
    W0 = wl.batch_planes(ncell, theta)
    target = rng.uniform(0.1, 2.0, W0.shape[1])
    L, G, gg = tangent.gradient(ncell, 1.0 / ncell, gamma, W0, target, 0.8, 8, 0.0, 0)
    d = np.zeros_like(W0)
    d[[0, 1, 4]] = rng.standard_normal((3, W0.shape[1]))
    dg = rng.standard_normal(3)
    L2, dL, _ = tangent.jvp(ncell, 1.0 / ncell, gamma, W0, target, 0.8, 8, 0.0, 0, d, dg)
    assert L == L2
    assert abs(dL - (np.sum(G * d) + gg @ dg)) <= 1e-12 * abs(dL)


def test_tangent_matches_central_fd_on_riemann_states():
    ncell, dx, gamma, theta, W0 = wl.ragged_riemann_batch(ninst=4, seed=3, nmin=20, nmax=60)
    rng = np.random.default_rng(1)
    target = rng.uniform(0.1, 2.0, W0.shape[1])
    steps, h = 12, 1e-6
    tl, fd = [], []
    for comp in range(7):
        dth = np.zeros_like(theta)
        dg = np.zeros(len(ncell))
        if comp == 6:
            dg = rng.standard_normal(len(ncell))
        else:
            dth[:, comp] = rng.standard_normal(len(ncell))
        d = wl.batch_planes(ncell, dth)
        d[5] = 0.0
        _, dL, _ = tangent.jvp(ncell, dx, gamma, W0, target, 0.8, steps, 0.0, 0, d, dg)
        Lp, _, _ = tangent.jvp(ncell, dx, gamma + h * dg, wl.batch_planes(ncell, theta + h * dth), target, 0.8,
                               steps, 0.0, 0)
        Lm, _, _ = tangent.jvp(ncell, dx, gamma - h * dg, wl.batch_planes(ncell, theta - h * dth), target, 0.8,
                               steps, 0.0, 0)
        tl.append(dL)
        fd.append((Lp - Lm) / (2 * h))
    tl, fd = np.array(tl), np.array(fd)
    assert np.linalg.norm(tl - fd) / np.linalg.norm(tl) <= 1e-6
