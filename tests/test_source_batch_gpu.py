"""The homogeneous HPR relaxation batch on the GPU: its forward against the oracle's forcing on uniform fields, and
its hand-written discrete adjoint against the tangent-linear reference (oracle/tangent_source.py), against central
finite differences of the device forward (h = 1e-6), across checkpoint schedules, and through a test-only
torch.autograd.Function wrapper."""
import numpy as np
import pytest

import oracle as O
from oracle import tangent_source as TS
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

REL = 1e-12   # pow(det A, 5/3): CUDA's and glibc's may differ in the last place


def _forcing_uniform(W, tau, prm, h, steps):
    out = np.empty_like(W)
    for c in range(W.shape[1]):
        p = prm.copy()
        p[7], p[8] = tau[0, c], tau[1, c]
        g = np.repeat(W[:, c:c + 1], 2, axis=1).copy()
        for _ in range(steps):
            O.forcing(g, 0.1, h, bias=0.0, limiter=O.SUPERBEE, params=p)
        out[:, c] = g[:, 0]
    return out


def _rel(a, b):
    return float((np.where(a == b, 0.0, np.abs(a - b) / np.maximum(np.abs(b), 1e-300))).max())


@pytest.mark.parametrize("thermal", [True, False])
def test_forward_is_the_reference_forcing(gpu, oracle_lib, thermal):
    W, tau, prm = wl.hpr_relaxation_cells(300, seed=5, thermal=thermal)
    h, steps = 2e-4, 7
    ref = _forcing_uniform(W, tau, prm, h, steps)
    with gpu.SourceBatch(300, prm) as b:
        b.upload(W, tau)
        b.run(h, steps)
        out = b.download()
    assert _rel(out, ref) <= REL
    if not thermal:
        assert np.array_equal(out[14:17], W[14:17])


def _adjoint(gpu, W, tau, prm, h, steps, lam, checkpoints=None):
    with gpu.SourceBatch(W.shape[1], prm) as b:
        b.upload(W, tau)
        g, gt, fw, aw = b.gradient(lam, h, steps, checkpoints=checkpoints)
        assert np.array_equal(b.download(), W)  # the batch keeps its state
    return g, gt, fw, aw


@pytest.mark.parametrize("thermal", [True, False])
def test_adjoint_matches_tangent_linear(gpu, thermal):
    """Every component of dL/dW0 and dL/dtau of every cell against the forward-mode reference (19 directions)."""
    n, h, steps = 40, 3e-4, 12
    W, tau, prm = wl.hpr_relaxation_cells(n, seed=6, thermal=thermal)
    lam = np.random.default_rng(2).standard_normal((17, n))
    g, gt, fw, aw = _adjoint(gpu, W, tau, prm, h, steps, lam)
    assert aw == steps
    ref = np.zeros((19, n))
    for k in range(19):
        dW, dtau = np.zeros_like(W), np.zeros_like(tau)
        if k < 17:
            dW[k] = 1.0
        else:
            dtau[k - 17] = 1.0
        _, tan = TS.jvp(W, tau, prm, h, steps, dW, dtau)
        ref[k] = (lam * tan).sum(axis=0)
    got = np.concatenate([g, gt])
    scale = np.abs(ref).max(axis=1, keepdims=True) + 1e-300
    err = (np.abs(got - ref) / scale).max()
    assert err <= 1e-9, err


def test_adjoint_matches_central_differences(gpu):
    """<dL/dtheta, d> against (L(theta + h d) - L(theta - h d)) / 2h of the device forward, h = 1e-6, for random
    directions of the initial primitives and (relative) relaxation times; L = <lambda, W(T)>."""
    n, h, steps, eps = 64, 3e-4, 20, 1e-6
    W, tau, prm = wl.hpr_relaxation_cells(n, seed=7)
    rng = np.random.default_rng(3)
    lam = rng.standard_normal((17, n))
    g, gt, _, _ = _adjoint(gpu, W, tau, prm, h, steps, lam)

    def loss(Wx, taux):
        with gpu.SourceBatch(n, prm) as b:
            b.upload(Wx, taux)
            b.run(h, steps)
            return float((lam * b.download()).sum())

    for trial in range(4):
        dW = rng.standard_normal(W.shape)
        dtau = tau * rng.standard_normal(tau.shape)
        fd = (loss(W + eps * dW, tau + eps * dtau) - loss(W - eps * dW, tau - eps * dtau)) / (2 * eps)
        ad = float((g * dW).sum() + (gt * dtau).sum())
        assert abs(fd - ad) <= 1e-6 * abs(ad), (trial, fd, ad)


def test_checkpoint_schedules_are_bit_identical(gpu):
    n, h, steps = 50, 2e-4, 37
    W, tau, prm = wl.hpr_relaxation_cells(n, seed=8)
    lam = np.random.default_rng(4).standard_normal((17, n))
    base = _adjoint(gpu, W, tau, prm, h, steps, lam)
    for ck in (1, 2, 3, 5, 36):
        g, gt, fw, aw = _adjoint(gpu, W, tau, prm, h, steps, lam, checkpoints=ck)
        assert np.array_equal(g, base[0]) and np.array_equal(gt, base[1]), ck
        assert aw == steps and fw >= base[2]
    # every state stored: one advance per checkpoint and the step's own recomputation inside each reverse step
    assert base[2] == 2 * steps - 1


def test_autograd_wrapper_gradcheck(gpu):
    """A test-only torch.autograd.Function over the C ABI: forward = run, backward = the adjoint."""
    import torch

    n, h, steps = 6, 3e-4, 5
    W, tau, prm = wl.hpr_relaxation_cells(n, seed=9)

    class SourceRun(torch.autograd.Function):
        """W(T) from W(0) and log(tau): the relaxation times enter through their logarithm, so one finite-difference
        step size suits both inputs."""

        @staticmethod
        def forward(ctx, w0, logtau):
            ctx.save_for_backward(w0, logtau)
            with gpu.SourceBatch(n, prm) as b:
                b.upload(w0.detach().numpy(), np.exp(logtau.detach().numpy()))
                b.run(h, steps)
                return torch.from_numpy(b.download())

        @staticmethod
        def backward(ctx, grad_out):
            w0, logtau = ctx.saved_tensors
            tau_ = np.exp(logtau.detach().numpy())
            g, gt, _, _ = _adjoint(gpu, w0.detach().numpy(), tau_, prm, h, steps, grad_out.contiguous().numpy())
            return torch.from_numpy(g), torch.from_numpy(gt * tau_)

    w0 = torch.tensor(W, dtype=torch.float64, requires_grad=True)
    lt = torch.tensor(np.log(tau), dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(SourceRun.apply, (w0, lt), eps=1e-6, atol=1e-7, rtol=1e-6)
