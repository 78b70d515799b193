"""Seeded synthetic initial data for the five benchmark workloads.

All arrays are float64 primitive planes in the reference's primitive order, shape (nvar, ny, nx) for
2D grids (row index = y, column index = x) and (nvar, n) for 1D lines.  Cell centres sit at
((j + 0.5) dx, (i + 0.5) dx) on [0, 1]^2.  The same arrays are fed to the CUDA path and to the CPU
oracle, so the oracle and the device always see identical inputs.
"""
from __future__ import annotations

import numpy as np

# Euler primitive order (Euler/eulerstatevector.cpp:36-45): rho, u, v, w, p, lambda
EULER_NVAR = 6
# MHD primitive order (MHD/mhdstatevector.cpp:35-47): rho, u, v, w, p, Bx, By, Bz, psi
MHD_NVAR = 9


def euler_params(gamma=1.4, p_inf=0.0):
    """EulerMaterialParameters(gamma, p_inf) with the reference's defaults for the reaction fields
    (Euler/eulermaterialparameters.cpp:25-34): c_v = 25, E0 = 0, T_ign = 0.25, rate = 250."""
    return np.array([gamma, p_inf, 25.0, 0.0, 0.25, 250.0])


def mhd_params(gamma=5.0 / 3.0, p_inf=0.0, c_h=0.0):
    """MHDMaterialParameters(gamma) (MHD/mhdmaterialparameters.cpp:12-19); c_h is reset every step."""
    return np.array([gamma, p_inf, c_h])


def sod_1d(n=1000, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1)):
    """1D shock tube, (rho, u, p) left/right.  Cell i is on the left when i <= 0.5 n, the convention of
    EulerTests::solveToroTest1 (Euler/eulertests.cpp:16), so cell n/2 starts with the left state."""
    W = np.zeros((EULER_NVAR, n))
    W[5] = 1.0
    is_left = np.arange(n) <= 0.5 * n
    W[0] = np.where(is_left, left[0], right[0])
    W[1] = np.where(is_left, left[1], right[1])
    W[4] = np.where(is_left, left[2], right[2])
    return W


def quadrant_states(seed):
    """Four (rho, u, v, p) states: rho ~ U[0.1, 2], u, v ~ U[-1, 1], p ~ U[0.1, 2]; quadrant q = 2*top + right."""
    rng = np.random.default_rng(seed)
    rho = rng.uniform(0.1, 2.0, 4)
    u = rng.uniform(-1.0, 1.0, 4)
    v = rng.uniform(-1.0, 1.0, 4)
    p = rng.uniform(0.1, 2.0, 4)
    return rho, u, v, p


def euler_quadrants_2d(nx=4096, ny=None, seed=0):
    """Four-quadrant 2D Riemann problem on [0,1]^2, split at the centre; quadrant states from `seed`."""
    ny = nx if ny is None else ny
    rho, u, v, p = quadrant_states(seed)
    top = (np.arange(ny) >= ny // 2)[:, None]
    right = (np.arange(nx) >= nx // 2)[None, :]
    q = (2 * top + right).astype(np.int64)
    W = np.zeros((EULER_NVAR, ny, nx))
    W[0] = rho[q]
    W[1] = u[q]
    W[2] = v[q]
    W[4] = p[q]
    W[5] = 1.0
    return W


def mhd_vortex_2d(nx=2048, ny=None, seed=0, gamma=5.0 / 3.0, amplitude=1e-3):
    """Orszag-Tang-type smooth vortex: rho = gamma^2, p = gamma, v = (-sin 2 pi y, sin 2 pi x, 0),
    B = (-sin 2 pi y, sin 4 pi x, 0) / sqrt(4 pi), psi = 0, plus i.i.d. N(0, 1) * amplitude added to rho
    and p from `seed`."""
    ny = nx if ny is None else ny
    dx = 1.0 / nx
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * (1.0 / ny)
    X, Y = np.meshgrid(x, y)
    rng = np.random.default_rng(seed)
    W = np.zeros((MHD_NVAR, ny, nx))
    W[0] = gamma * gamma + amplitude * rng.standard_normal((ny, nx))
    W[1] = -np.sin(2 * np.pi * Y)
    W[2] = np.sin(2 * np.pi * X)
    W[4] = gamma + amplitude * rng.standard_normal((ny, nx))
    s = 1.0 / np.sqrt(4 * np.pi)
    W[5] = -np.sin(2 * np.pi * Y) * s
    W[6] = np.sin(4 * np.pi * X) * s
    return W


HPR_NVAR = 17  # rho, p, A(9 row-major), u, v, w, Jx, Jy, Jz


def hpr_params(gamma=1.4, p_inf=0.0, c_v=2.5, rho0=1.0, T0=1.0, c_s=1.0, alpha=1.0, tau1=1e-2, tau2=1e-2,
               T_ref=0.0, p_ref=1.0, thermal=True):
    """HPRMaterialParameters for the StiffenedGas equation of state (ideal gas when p_inf = 0), non-plastic:
    {gamma, p_inf, c_v, rho0, T0, c_s, alpha, tau1, tau2, T_ref, p_ref, is_thermal}.  Defaults follow the
    reference's heat-conduction scenario (HPR/hprtests.cpp:33-57): rho0 = 1, p_ref = 1, T_ref = 0, T0 = 1,
    c_v = 2.5."""
    return np.array([gamma, p_inf, c_v, rho0, T0, c_s, alpha, tau1, tau2, T_ref, p_ref, 1.0 if thermal else 0.0])


def hpr_relaxation_times(seed):
    """tau1, tau2 log-uniform on [1e-6, 1e-2] from `seed`."""
    rng = np.random.default_rng(seed)
    return 10.0 ** rng.uniform(-6.0, -2.0, 2)


def hpr_smooth_2d(nx=1024, ny=None, seed=0):
    """Seeded smooth field: rho = 1 + 0.2 sin(2 pi (k.x) + phi), velocity of magnitude <= 0.1 from seeded
    Fourier phases, p = 1, A = I, J = 0 (A = I with rho != rho0 is not rho0 det A; the reference does not
    enforce that relation)."""
    ny = nx if ny is None else ny
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y)
    rng = np.random.default_rng(seed)
    kx, ky = rng.integers(1, 4, 2)
    phi = rng.uniform(0, 2 * np.pi, 5)
    W = np.zeros((HPR_NVAR, ny, nx))
    W[0] = 1.0 + 0.2 * np.sin(2 * np.pi * (kx * X + ky * Y) + phi[0])
    W[1] = 1.0
    W[2] = W[6] = W[10] = 1.0
    W[11] = 0.05 * (np.sin(2 * np.pi * Y + phi[1]) + np.cos(2 * np.pi * X + phi[2]))
    W[12] = 0.05 * (np.sin(2 * np.pi * X + phi[3]) + np.cos(2 * np.pi * Y + phi[4]))
    return W


def hpr_heat_conduction_1d(n=200):
    """HPRTests::solveHeatConductionProblem initial data (HPR/hprtests.cpp:42-53): rho = 2 | 0.5, p = 1,
    A = rho^(1/3) I, split at i <= n/2."""
    W = np.zeros((HPR_NVAR, n))
    left = np.arange(n) <= 0.5 * n
    W[0] = np.where(left, 2.0, 0.5)
    W[1] = 1.0
    a = np.where(left, 2.0 ** (1.0 / 3.0), 0.5 ** (1.0 / 3.0))
    W[2] = W[6] = W[10] = a
    return W


def brio_wu_1d(n=400, gamma=2.0):
    """Brio-Wu-type MHD shock tube (MHDTests' first Dumbser test family): left (1, 0, 0, 0, 1, 0.75, 1, 0),
    right (0.125, 0, 0, 0, 0.1, 0.75, -1, 0), split at i <= n/2."""
    W = np.zeros((MHD_NVAR, n))
    is_left = np.arange(n) <= 0.5 * n
    W[0] = np.where(is_left, 1.0, 0.125)
    W[4] = np.where(is_left, 1.0, 0.1)
    W[5] = 0.75
    W[6] = np.where(is_left, 1.0, -1.0)
    return W


def ragged_riemann_batch(ninst=4096, seed=0, nmin=200, nmax=4000):
    """Independent 1D Riemann problems on [0, 1]: cells ~ U{nmin..nmax}, gamma ~ U[1.2, 1.67], left/right
    rho ~ U[0.1, 2], u ~ U[-1, 1], p ~ U[0.1, 10], interface at the middle (cell i is left when i <= n/2).
    Returns (ncell, dx, gamma, theta, planes) with theta the (ninst, 6) initial states
    (rho_L, u_L, p_L, rho_R, u_R, p_R) and planes the (6, total) concatenated Euler primitives."""
    rng = np.random.default_rng(seed)
    ncell = rng.integers(nmin, nmax + 1, ninst)
    gamma = rng.uniform(1.2, 1.67, ninst)
    theta = np.stack([rng.uniform(0.1, 2.0, ninst), rng.uniform(-1.0, 1.0, ninst), rng.uniform(0.1, 10.0, ninst),
                      rng.uniform(0.1, 2.0, ninst), rng.uniform(-1.0, 1.0, ninst), rng.uniform(0.1, 10.0, ninst)], 1)
    return ncell, 1.0 / ncell, gamma, theta, batch_planes(ncell, theta)


def batch_planes(ncell, theta):
    """Concatenated (6, total) Euler primitive planes of Riemann problems with states theta (ninst, 6)."""
    total = int(np.sum(ncell))
    W = np.zeros((EULER_NVAR, total))
    W[5] = 1.0
    off = 0
    for k, n in enumerate(ncell):
        left = np.arange(n) <= 0.5 * n
        W[0, off:off + n] = np.where(left, theta[k, 0], theta[k, 3])
        W[1, off:off + n] = np.where(left, theta[k, 1], theta[k, 4])
        W[4, off:off + n] = np.where(left, theta[k, 2], theta[k, 5])
        off += n
    return W
