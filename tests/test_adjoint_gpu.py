"""Discrete adjoint of the ragged 1D Euler batch (vg_batch_gradient).

Checks: (1) every component of dL/dW0 and dL/dgamma against the forward-mode FP64 tangent-linear reference
(oracle.tangent), which follows the same branches; (2) dL/dtheta (the six Riemann states) and dL/dgamma against
central finite differences with h = 1e-6 through the device forward; (3) every checkpoint schedule gives the
same gradient bit for bit, with the forward-step counts of the binomial schedule; (4) a torch.autograd.Function
wrapper (test harness only) passes gradcheck.
"""
import math

import numpy as np
import pytest

from oracle import tangent
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

CFL = 0.8


def _theta_batch(ncell, seed):
    rng = np.random.default_rng(seed)
    k = len(ncell)
    gamma = rng.uniform(1.2, 1.67, k)
    theta = np.stack([rng.uniform(0.1, 2.0, k), rng.uniform(-1.0, 1.0, k), rng.uniform(0.1, 10.0, k),
                      rng.uniform(0.1, 2.0, k), rng.uniform(-1.0, 1.0, k), rng.uniform(0.1, 10.0, k)], 1)
    return gamma, theta


def _final_rho(gpu, ncell, gamma, theta, steps, limiter):
    with gpu.Batch(ncell, 1.0 / ncell, gamma) as b:
        b.upload(wl.batch_planes(ncell, theta))
        b.run(CFL, steps, limiter=limiter)
        return b.download()[0]


def _instance_losses(ncell, rho, target):
    out, off = [], 0
    for n in ncell:
        out.append(math.fsum((rho[off:off + n] - target[off:off + n]) ** 2))
        off += n
    return np.array(out)


def _theta_grad(ncell, G):
    """dL/dtheta from the per-cell gradient: sums over each instance's left (i <= n/2) and right cells."""
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


@pytest.mark.parametrize("limiter", [0, 1, 2])
def test_adjoint_matches_tangent_linear(gpu, limiter):
    # sizes around the 118-cell adjoint tile and the 126-cell forward tile, plus the 2- and 3-cell minimum cases
    ncell = np.array([2, 3, 17, 118, 119, 237])
    gamma, theta = _theta_batch(ncell, 10 + limiter)
    W0 = wl.batch_planes(ncell, theta)
    # perturb every cell so no two cells tie and the slopes are not all floored
    rng = np.random.default_rng(limiter)
    W0[[0, 4]] *= 1.0 + 0.01 * rng.standard_normal((2, W0.shape[1]))
    W0[1] += 0.01 * rng.standard_normal(W0.shape[1])
    target = rng.uniform(0.1, 2.0, W0.shape[1])
    steps = 14
    with gpu.Batch(ncell, 1.0 / ncell, gamma) as b:
        b.upload(W0)
        L, G, gg, fw, aw = b.gradient(target, CFL, steps, limiter=limiter, checkpoints=4)
        assert aw == steps
        assert np.array_equal(b.download(), W0)  # the batch keeps its initial state
    Lt, Gt, ggt = tangent.gradient(ncell, 1.0 / ncell, gamma, W0, target, CFL, steps, 0.0, limiter)
    assert abs(L - Lt) <= 1e-12 * Lt
    scale = np.abs(Gt).max()
    assert np.abs(G - Gt).max() <= 1e-9 * scale
    assert np.all(G[[2, 3, 5]] == 0.0)
    assert np.allclose(gg, ggt, rtol=1e-9, atol=1e-12 * scale)


def test_adjoint_matches_central_fd(gpu):
    ncell = np.array([40, 97, 130, 300, 513])
    gamma, theta = _theta_batch(ncell, 3)
    steps, limiter = 40, 0
    W0 = wl.batch_planes(ncell, theta)
    rho_T = _final_rho(gpu, ncell, gamma, theta, steps, limiter)
    target = rho_T + 0.05 * np.random.default_rng(4).standard_normal(rho_T.shape)
    with gpu.Batch(ncell, 1.0 / ncell, gamma) as b:
        b.upload(W0)
        L, G, gg, _, _ = b.gradient(target, CFL, steps, limiter=limiter, checkpoints=6)
    assert L == pytest.approx(_instance_losses(ncell, rho_T, target).sum(), rel=1e-12)
    ad = np.concatenate([_theta_grad(ncell, G), gg[:, None]], 1)  # (ninst, 7)
    h = 1e-6
    fd = np.zeros_like(ad)
    for j in range(7):  # perturb component j of every instance at once; instances are independent
        Lpm = []
        for sgn in (1.0, -1.0):
            th, ga = theta.copy(), gamma.copy()
            if j < 6:
                th[:, j] += sgn * h
            else:
                ga += sgn * h
            Lpm.append(_instance_losses(ncell, _final_rho(gpu, ncell, ga, th, steps, limiter), target))
        fd[:, j] = (Lpm[0] - Lpm[1]) / (2 * h)
    err = np.linalg.norm(fd - ad) / np.linalg.norm(ad)
    assert err <= 1e-6, (err, ad, fd)


def test_checkpoint_schedules_bitwise(gpu):
    ncell = np.array([5, 130, 64])
    gamma, theta = _theta_batch(ncell, 7)
    W0 = wl.batch_planes(ncell, theta)
    target = np.random.default_rng(1).uniform(0.1, 2.0, W0.shape[1])
    steps = 23
    results = {}
    with gpu.Batch(ncell, 1.0 / ncell, gamma) as b:
        b.upload(W0)
        for c in (1, 2, 3, 5, 8, steps, steps + 4):
            results[c] = b.gradient(target, CFL, steps, checkpoints=c)
    base = results[steps]
    assert base[3] == steps  # every state stored: each step advanced once
    assert results[steps + 4][3] == steps
    assert results[1][3] == steps * (steps - 1) // 2 + 1  # only W0 stored: recompute from it
    fws = [results[c][3] for c in (1, 2, 3, 5, 8, steps)]
    assert all(a >= b for a, b in zip(fws, fws[1:]))
    assert results[3][3] <= 3 * steps  # binomial: 3 slots reverse 23 steps with <= 3 advances per step
    for c, r in results.items():
        assert r[0] == base[0] and np.array_equal(r[1], base[1]) and np.array_equal(r[2], base[2]), c
        assert r[4] == steps


def test_single_step_and_argument_errors(gpu):
    ncell = np.array([2, 9])
    gamma, theta = _theta_batch(ncell, 2)
    W0 = wl.batch_planes(ncell, theta)
    target = np.ones(W0.shape[1])
    with gpu.Batch(ncell, 1.0 / ncell, gamma) as b:
        b.upload(W0)
        L, G, gg, fw, aw = b.gradient(target, CFL, 1, checkpoints=1)
        assert (fw, aw) == (1, 1)
        Lt, Gt, ggt = tangent.gradient(ncell, 1.0 / ncell, gamma, W0, target, CFL, 1, 0.0, 0)
        assert np.abs(G - Gt).max() <= 1e-10 * np.abs(Gt).max()
        with pytest.raises(gpu.VgError):
            b.gradient(target, CFL, 5, checkpoints=0)
        with pytest.raises(gpu.VgError):
            b.gradient(target, CFL, 0)
        with pytest.raises(ValueError):
            b.gradient(target[:-1], CFL, 3)


def test_torch_autograd_wrapper_gradcheck(gpu):
    torch = pytest.importorskip("torch")
    ncell = np.array([12, 30])
    steps = 10
    target = np.random.default_rng(2).uniform(0.1, 2.0, int(ncell.sum()))

    class BatchLoss(torch.autograd.Function):
        """Loss of the device batch as a function of (theta, gamma), backward by vg_batch_gradient."""

        @staticmethod
        def forward(ctx, theta, gamma):
            th, ga = theta.detach().numpy(), gamma.detach().numpy()
            with gpu.Batch(ncell, 1.0 / ncell, ga) as b:
                b.upload(wl.batch_planes(ncell, th))
                L, G, gg, _, _ = b.gradient(target, CFL, steps, checkpoints=3)
            ctx.save_for_backward(torch.from_numpy(_theta_grad(ncell, G)), torch.from_numpy(gg))
            return torch.tensor(L, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            gth, ggam = ctx.saved_tensors
            return gout * gth, gout * ggam

    gamma, theta = _theta_batch(ncell, 8)
    th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    ga = torch.tensor(gamma, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(BatchLoss.apply, (th, ga), eps=1e-6, atol=1e-6, rtol=1e-5)


def test_device_buffers_match_host_buffers(gpu):
    torch = pytest.importorskip("torch")
    ncell = np.array([7, 140])
    gamma, theta = _theta_batch(ncell, 5)
    W0 = wl.batch_planes(ncell, theta)
    target = np.random.default_rng(3).uniform(0.1, 2.0, W0.shape[1])
    with gpu.Batch(ncell, 1.0 / ncell, gamma) as b:
        b.upload(W0)
        L, G, gg, fw, aw = b.gradient(target, CFL, 12, checkpoints=3)
        td = torch.from_numpy(target).cuda()
        g = torch.full((6, W0.shape[1]), 7.0, dtype=torch.float64, device="cuda")
        ggd = torch.empty(len(ncell), dtype=torch.float64, device="cuda")
        L2, _, _, fw2, aw2 = b.gradient(td, CFL, 12, checkpoints=3, out=(g, ggd))
    assert L == L2 and (fw, aw) == (fw2, aw2)
    assert np.array_equal(g.cpu().numpy(), G) and np.array_equal(ggd.cpu().numpy(), gg)


def test_adjoint_matches_tangent_linear_long_horizon(gpu):
    # 300 steps: far past the horizon where central differences stay smooth for superbee (limiter kinks and the
    # 1e-5 floor are crossed within +-h); the tangent-linear run follows the same branches and stays exact
    ncell = np.array([60, 131])
    gamma, theta = _theta_batch(ncell, 21)
    W0 = wl.batch_planes(ncell, theta)
    target = np.random.default_rng(9).uniform(0.1, 2.0, W0.shape[1])
    steps = 300
    with gpu.Batch(ncell, 1.0 / ncell, gamma) as b:
        b.upload(W0)
        L, G, gg, fw, aw = b.gradient(target, CFL, steps, checkpoints=20)
    Lt, Gt, ggt = tangent.gradient(ncell, 1.0 / ncell, gamma, W0, target, CFL, steps, 0.0, 0)
    assert abs(L - Lt) <= 1e-12 * Lt
    scale = np.abs(Gt).max()
    assert np.abs(G - Gt).max() <= 1e-8 * scale
    assert np.allclose(gg, ggt, rtol=1e-8, atol=1e-12 * scale)
