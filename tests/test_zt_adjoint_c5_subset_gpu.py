"""The discrete adjoint (vg_batch_gradient) on the first 64 instances of the C5 ragged batch -- 4096 Riemann problems of
200..4000 cells, seed 2024, superbee, CFL 0.8 -- at its full 500 steps with the binomial schedule's 32 checkpoints:
127,607 cells.

The adjoint's directional derivative along a seeded direction in (initial states, gamma) is checked against the
forward-mode FP64 tangent-linear run (oracle.tangent.jvp), which follows the same limiter branches, at 1e-9 relative;
and against central finite differences through the device forward.  At 500 steps the superbee limiter's kinks and the
1e-5 slope floor are crossed within +-h somewhere among the 127,607 cells, so central differences carry a
branch-crossing error that no step size removes: on this subset it is 1.1e-4 relative at h = 1e-5 and 3.6e-3 at
h = 1e-6 (the tangent-linear value is exact), so the finite-difference bound is 1e-3 at h = 1e-5.

Runs after the other GPU tests: the tangent-linear run takes about a minute of host CPU."""
import math

import numpy as np
import pytest

from oracle import tangent
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

NINST, STEPS, CFL, LIMITER, SEED, CHECKPOINTS = 64, 500, 0.8, 0, 2024, 32


def _subset():
    ncell, dx, gamma, theta, _ = wl.ragged_riemann_batch(4096, seed=SEED)
    target_all = np.random.default_rng(SEED + 1).uniform(0.1, 2.0, int(ncell.sum()))
    ncell, dx, gamma, theta = ncell[:NINST], dx[:NINST], gamma[:NINST], theta[:NINST]
    return ncell, dx, gamma, theta, target_all[:int(ncell.sum())]


def _theta_grad(ncell, G):
    out = np.zeros((len(ncell), 6))
    off = 0
    for k, n in enumerate(ncell):
        left = np.arange(n) <= 0.5 * n
        for j, plane in enumerate((0, 1, 4)):
            g = G[plane, off:off + n]
            out[k, j] = g[left].sum()
            out[k, 3 + j] = g[~left].sum()
        off += n
    return out


def _loss(gpu, ncell, dx, gamma, theta, target):
    with gpu.Batch(ncell, dx, gamma) as b:
        b.upload(wl.batch_planes(ncell, theta))
        b.run(CFL, STEPS, limiter=LIMITER)
        rho = b.download()[0]
    return math.fsum((rho - target) ** 2)


def test_c5_subset_adjoint_at_500_steps(gpu):
    ncell, dx, gamma, theta, target = _subset()
    assert int(ncell.sum()) == 127607
    rng = np.random.default_rng(7)
    v_theta, v_gamma = rng.standard_normal((NINST, 6)), 0.1 * rng.standard_normal(NINST)
    with gpu.Batch(ncell, dx, gamma) as b:
        b.upload(wl.batch_planes(ncell, theta))
        L, G, gg, fw, aw = b.gradient(target, CFL, STEPS, limiter=LIMITER, checkpoints=CHECKPOINTS)
    assert fw > STEPS and aw == STEPS
    ad = float(np.sum(_theta_grad(ncell, G) * v_theta) + np.sum(gg * v_gamma))

    dW0 = wl.batch_planes(ncell, v_theta)
    dW0[5] = 0.0
    Lt, dLt, _ = tangent.jvp(ncell, dx, gamma, wl.batch_planes(ncell, theta), target, CFL, STEPS, 0.0, LIMITER,
                             dW0=dW0, dgamma=v_gamma)
    assert abs(L - Lt) <= 1e-12 * Lt
    assert abs(ad - dLt) <= 1e-9 * abs(dLt), (ad, dLt)

    h = 1e-5
    fd = (_loss(gpu, ncell, dx, gamma + h * v_gamma, theta + h * v_theta, target) -
          _loss(gpu, ncell, dx, gamma - h * v_gamma, theta - h * v_theta, target)) / (2 * h)
    assert abs(fd - ad) <= 1e-3 * abs(ad), (fd, ad)
