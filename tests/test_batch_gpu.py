"""Ragged batch of independent 1D Euler problems: every instance bit-equal to its own solve() loop."""
import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("limiter", [0, 2])
def test_batch_matches_per_instance_oracle(gpu, oracle_lib, limiter):
    ncell, dx, gamma, theta, W = wl.ragged_riemann_batch(ninst=37, seed=5 + limiter, nmin=20, nmax=400)
    steps = 60
    with gpu.Batch(ncell, dx, gamma) as b:
        b.upload(W)
        dts = b.run(0.8, steps, limiter=limiter)
        out = b.download()
        assert b.last_launch_count() == steps + 1
    off = 0
    for k, n in enumerate(ncell):
        ref = W[:, off:off + n].copy()
        _, st, dtl = O.run(O.EULER, ref, dx[k], 0.8, steps=steps, limiter=limiter,
                           params=wl.euler_params(gamma[k]), dt_log=True)
        assert st == steps
        assert np.array_equal(out[:, off:off + n], ref), k
        assert dts[k] == dtl[-1]
        off += n


def test_batch_repeated_runs_and_tiny_instances(gpu, oracle_lib):
    ncell = np.array([2, 3, 127, 126, 128, 300])
    dx = 1.0 / ncell
    gamma = np.array([1.4, 1.3, 1.5, 1.67, 1.2, 1.4])
    theta = np.tile([1.0, 0.2, 1.0, 0.3, -0.1, 0.2], (6, 1))
    W = wl.batch_planes(ncell, theta)
    with gpu.Batch(ncell, dx, gamma) as b:
        for steps in (7, 8):
            b.upload(W)
            b.run(0.8, steps)
            out = b.download()
            off = 0
            for k, n in enumerate(ncell):
                ref = W[:, off:off + n].copy()
                O.run(O.EULER, ref, dx[k], 0.8, steps=steps, limiter=0, params=wl.euler_params(gamma[k]))
                assert np.array_equal(out[:, off:off + n], ref), (steps, k)
                off += n
