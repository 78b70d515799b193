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


HPR_EOS = {"StiffenedGas": 0, "ShockMieGruneisen": 1, "GodunovRomenski": 2}


def hpr_params(gamma=1.4, p_inf=0.0, c_v=2.5, rho0=1.0, T0=1.0, c_s=1.0, alpha=1.0, tau1=1e-2, tau2=1e-2,
               T_ref=0.0, p_ref=1.0, thermal=True, eos="StiffenedGas", Gamma0=0.0, c0=0.0, s=0.0, alpha_eos=0.0,
               plastic=False, sigma0=0.0, n=0.0):
    """HPRMaterialParameters (HPR/hprmaterialparameters.cpp:34-69) as the 20-value block
    {gamma, p_inf, c_v, rho0, T0, c_s, alpha, tau1, tau2, T_ref, p_ref, is_thermal,
     eos, Gamma0, c0, s, alpha_eos, is_plastic, sigma0, n}.
    eos: StiffenedGas (gamma, p_inf; an ideal gas when p_inf = 0), ShockMieGruneisen (Gamma0, c0, Hugoniot slope
    s, reference pressure p_ref) or GodunovRomenski (c0, exponent alpha_eos, Grueneisen coefficient gamma).
    plastic: the plastic strain relaxation theta1 * (min(|sigma|, 1e8) / sigma0)^n (HPR/hprsourceterms.cpp:12-23).
    Defaults follow the reference's heat-conduction scenario (HPR/hprtests.cpp:33-57): a non-plastic ideal gas,
    rho0 = 1, p_ref = 1, T_ref = 0, T0 = 1, c_v = 2.5."""
    return np.array([gamma, p_inf, c_v, rho0, T0, c_s, alpha, tau1, tau2, T_ref, p_ref, 1.0 if thermal else 0.0,
                     float(HPR_EOS[eos]), Gamma0, c0, s, alpha_eos, 1.0 if plastic else 0.0, sigma0, n])


def hpr_barton_params():
    """The copper of the reference's Barton test (HPR/hprtests.cpp:59-66): GodunovRomenski, rho0 8.9, c0 3.909,
    exponent 1, Grueneisen coefficient gamma 1 (its adiabatic index), c_s 2.1, c_v 3.94e-4, T_ref = T0 = 300,
    tau1 1e8 (elastic), tau2 4e-8, not thermal, not plastic."""
    return hpr_params(gamma=1.0, p_inf=0.0, c_v=3.94e-4, rho0=8.9, T0=300.0, c_s=2.1,
                      alpha=8.9 * 3.909 * np.sqrt(4.0e-4 / 300.0), tau1=1e8, tau2=4.0e-8, T_ref=300.0, p_ref=0.0,
                      thermal=False, eos="GodunovRomenski", c0=3.909, alpha_eos=1.0)


def hpr_zhang_params():
    """The aluminium of the reference's Zhang elastic-plastic test (HPR/hprtests.cpp:109-115): GodunovRomenski,
    rho0 2.71, c0 5.037, exponent 1, gamma 1, c_s 3.16, c_v 9e-4, p_ref 73, T_ref = T0 = 300, tau1 1e-9, plastic
    with sigma0 0.2976e9 and n 1.338, not thermal."""
    return hpr_params(gamma=1.0, p_inf=0.0, c_v=9.0e-4, rho0=2.71, T0=300.0, c_s=3.16, alpha=2.0, tau1=1e-9,
                      tau2=0.0, T_ref=300.0, p_ref=73.0, thermal=False, eos="GodunovRomenski", Gamma0=1.0, c0=5.037,
                      s=1.338, alpha_eos=1.0, plastic=True, sigma0=0.2976e9, n=1.338)


def hpr_shock_mg_params(thermal=False, plastic=False, sigma0=0.05, n=2.0, tau1=1e-3):
    """A ShockMieGruneisen solid (copper-like: rho0 8.93, c0 3.94, Gamma0 2.0, Hugoniot slope 1.49, p_ref 1e-4,
    c_s 2.2, c_v 3.9e-4, T_ref = T0 = 300)."""
    return hpr_params(gamma=2.0, p_inf=0.0, c_v=3.9e-4, rho0=8.93, T0=300.0, c_s=2.2, alpha=1.0, tau1=tau1,
                      tau2=1e-3, T_ref=300.0, p_ref=1e-4, thermal=thermal, eos="ShockMieGruneisen", Gamma0=2.0,
                      c0=3.94, s=1.49, plastic=plastic, sigma0=sigma0, n=n)


def gr_reference_pressure(rho, prm):
    """GodunovRomenski cold pressure c0^2 (rho / alpha) (c - 1) c, c = (rho / rho0)^alpha
    (HPR/hprmiegruneisen.cpp:55-63)."""
    c = (rho / prm[3]) ** prm[16]
    return prm[14] ** 2 * (rho / prm[16]) * (c - 1.0) * c


def hpr_solid_riemann_1d(n, prm, F_left, F_right, v_left, v_right, p_offset=0.0):
    """A 1D solid Riemann problem in the shape of the reference's Barton and Zhang tests (HPR/hprtests.cpp:68-104,
    :119-131): A = F^-1 on each side of i <= n/2, rho = rho0 det A, velocities v_left / v_right, and the cold state
    p = p_ref(rho) + p_offset of a GodunovRomenski solid.  The reference's own set-up takes p from the hyperelastic
    equation of state of its Elasticity module, which this package does not carry."""
    W = np.zeros((HPR_NVAR, n))
    left = np.arange(n) <= 0.5 * n
    for side, F, v in ((left, F_left, v_left), (~left, F_right, v_right)):
        A = np.linalg.inv(np.asarray(F, dtype=np.float64))
        rho = prm[3] * np.linalg.det(A)
        W[0, side] = rho
        W[1, side] = gr_reference_pressure(rho, prm) + p_offset
        W[2:11, side] = A.reshape(9)[:, None]
        W[11:14, side] = np.asarray(v, dtype=np.float64)[:, None]
    return W


def smg_reference_pressure(rho, prm):
    """ShockMieGruneisen cold pressure (HPR/hprmiegruneisen.cpp:41-54): compressed c0^2 (1/rho0 - 1/rho) /
    (1/rho0 - s (1/rho0 - 1/rho))^2, expanded c0^2 (rho - rho0)."""
    rho = np.asarray(rho, dtype=np.float64)
    v0, c0sq, s = 1.0 / prm[3], prm[14] ** 2, prm[15]
    comp = c0sq * ((v0 - 1.0 / rho) / (v0 - s * (v0 - 1.0 / rho)) ** 2)
    return np.where(rho > prm[3], comp, c0sq * (rho - prm[3]))


def hpr_shock_riemann(nx, ny, prm, seed=0):
    """A ShockMieGruneisen solid with a compressed left state (rho 9.4 | 8.93 for the copper-like set) on the cold
    curve plus a small thermal pressure, A = (rho / rho0)^(1/3) I, and a seeded shear velocity jump; ny == 1 gives
    planes (17, nx), else (17, ny, nx) with the split along x."""
    rng = np.random.default_rng(seed)
    shape = (nx,) if ny == 1 else (ny, nx)
    W = np.zeros((HPR_NVAR,) + shape)
    x = np.arange(nx) if ny == 1 else np.meshgrid(np.arange(nx), np.arange(ny))[0]
    left = x <= 0.5 * nx
    rho = np.where(left, 1.0526 * prm[3], prm[3])
    W[0] = rho
    W[1] = smg_reference_pressure(rho, prm) + np.where(left, 0.02, 1e-3)
    a = (rho / prm[3]) ** (1.0 / 3.0)
    W[2] = W[6] = W[10] = a
    W[11] = np.where(left, 0.0, -0.1)
    W[12] = np.where(left, rng.uniform(0.02, 0.08), 0.0)
    return W


BARTON_F = ([[0.98, 0.0, 0.0], [0.02, 1.0, 0.1], [0.0, 0.0, 1.0]],
            [[1.0, 0.0, 0.0], [0.0, 1.0, 0.1], [0.0, 0.0, 1.0]])
# the left and right deformation gradients of the reference's Zhang scenarios of the two-material HPR models
# (HPR/Multiphysics/hprintermediatetests.cpp:64-84)
ZHANG_F = ([[1.0, 0.0, 0.0], [-0.01, 0.95, 0.02], [-0.015, 0.0, 0.9]],
           [[1.0, 0.0, 0.0], [0.015, 0.95, 0.0], [-0.01, 0.0, 0.9]])


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


REDUCED_NVAR = 7  # alpha1, u, v, w, rho1, rho2, p (EulerReducedStateVector, Euler/Multiphysics/eulerreducedstatevector.cpp:30-41)


def reduced_params(gamma1=1.4, p_inf1=0.0, gamma2=1.4, p_inf2=0.0):
    """The two EulerMaterialParameters of the reduced model: (gamma1, p_inf1, gamma2, p_inf2)."""
    return np.array([gamma1, p_inf1, gamma2, p_inf2])


def reduced_shock_tube(n, rho=(1.0, 0.125), p=(1.0, 0.1), u=(0.0, 0.0)):
    """EulerReducedTests::solveToroTest1's layout (Euler/Multiphysics/eulerreducedtests.cpp:7-26): material 1
    (alpha1 = 0.999) at i <= n/2, material 2 (0.001) to the right, rho1 = rho[0] and rho2 = rho[1] everywhere."""
    W = np.zeros((REDUCED_NVAR, n))
    left = np.arange(n) <= 0.5 * n
    W[0] = np.where(left, 0.999, 0.001)
    W[1] = np.where(left, u[0], u[1])
    W[4] = rho[0]
    W[5] = rho[1]
    W[6] = np.where(left, p[0], p[1])
    return W


def reduced_bubble_2d(nx, ny=None, rho=(1.0, 0.125), p=(1.0, 0.1), radius=0.2):
    """EulerReducedTests::solve2DToroTest1's layout (:58-80): material 1 inside the disc of radius 0.2 n about the
    grid centre (row index i, column j), material 2 outside."""
    ny = nx if ny is None else ny
    I, J = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    inside = np.sqrt((I - 0.5 * ny) ** 2 + (J - 0.5 * nx) ** 2) <= radius * nx
    W = np.zeros((REDUCED_NVAR, ny, nx))
    W[0] = np.where(inside, 0.999, 0.001)
    W[4] = rho[0]
    W[5] = rho[1]
    W[6] = np.where(inside, p[0], p[1])
    return W


MULTIPHYSICS_NVAR = 8  # alpha1, u, v, w, rho1, p1, rho2, p2 (Euler/Multiphysics/eulermultiphysicsstatevector.cpp:32-44)


def multiphysics_from_reduced(W):
    """The multiphysics model's planes of a reduced-model state: both materials at the interface pressure."""
    out = np.zeros((MULTIPHYSICS_NVAR,) + W.shape[1:])
    out[:5] = W[:5]
    out[5] = W[6]
    out[6] = W[5]
    out[7] = W[6]
    return out



MHD_REDUCED_NVAR = 11  # alpha1, u, v, w, rho1, rho2, p, Bx, By, Bz, psi (MHD/Multiphysics/mhdreducedstatevector.cpp:91-111)


def mhd_reduced_params(gamma1=2.0, p_inf1=0.0, gamma2=2.0, p_inf2=0.0):
    """The two MHDMaterialParameters of the MHD reduced model: (gamma1, p_inf1, gamma2, p_inf2).  Dumbser test 1
    uses gamma 2 for both materials, its multimaterial variant 1.4 and 1.67."""
    return np.array([gamma1, p_inf1, gamma2, p_inf2])


_DUMBSER_IN = (0.999, 0.0, 0.0, 0.0, 1.0, 0.125, 1.0, 0.75, 1.0, 0.0, 0.0)
_DUMBSER_OUT = (0.001, 0.0, 0.0, 0.0, 1.0, 0.125, 0.1, 0.75, -1.0, 0.0, 0.0)


def mhd_reduced_dumbser_1d(n):
    """MHDReducedTests::solveDumbserTest1's layout (MHD/Multiphysics/mhdreducedtests.cpp:7-27): the Brio-Wu states
    with material 1 (alpha1 = 0.999) at i <= n/2 and material 2 (0.001) to the right."""
    left = np.arange(n) <= 0.5 * n
    return np.stack([np.where(left, a, b) for a, b in zip(_DUMBSER_IN, _DUMBSER_OUT)]).astype(np.float64)


def mhd_reduced_dumbser_2d(nx, ny=None, radius=0.2):
    """MHDReducedTests::solve2DDumbserTest1's layout (:53-76): the left Brio-Wu state inside the disc of radius 0.2 n
    about the grid centre (row index i, column j), the right one outside."""
    ny = nx if ny is None else ny
    I, J = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    inside = np.sqrt((I - 0.5 * ny) ** 2 + (J - 0.5 * nx) ** 2) <= radius * nx
    return np.stack([np.where(inside, a, b) for a, b in zip(_DUMBSER_IN, _DUMBSER_OUT)]).astype(np.float64)


MHD_INTERMEDIATE_NVAR = 12  # alpha1, u, v, w, rho1, p1, rho2, p2, Bx, By, Bz, psi (mhdintermediatestatevector.cpp:108-130)


def mhd_intermediate_from_reduced(W):
    """The MHD intermediate model's planes of an MHD reduced state: both materials at the interface pressure."""
    out = np.zeros((MHD_INTERMEDIATE_NVAR,) + W.shape[1:])
    out[:5] = W[:5]
    out[5] = W[6]
    out[6] = W[5]
    out[7] = W[6]
    out[8:] = W[7:]
    return out


def hpr_relaxation_cells(n, seed=0, thermal=True, tau_range=(1e-3, 1e-2), distortion=0.05):
    """n homogeneous HPR cells for the source batch: distorted A (I + N(0, distortion^2) per entry), heat flux J,
    rho ~ U[0.8, 1.2], p ~ U[0.5, 1.5], |u| ~ 0.1; tau1, tau2 log-uniform on tau_range per cell.
    Returns (W (17, n), tau (2, n), params)."""
    rng = np.random.default_rng(seed)
    W = np.zeros((17, n))
    W[0] = rng.uniform(0.8, 1.2, n)
    W[1] = rng.uniform(0.5, 1.5, n)
    A = np.eye(3)[:, :, None] + distortion * rng.standard_normal((3, 3, n))
    W[2:11] = A.reshape(9, n)
    W[11:14] = 0.1 * rng.standard_normal((3, n))
    W[14:17] = 0.1 * rng.standard_normal((3, n))
    lo, hi = np.log10(tau_range[0]), np.log10(tau_range[1])
    tau = 10.0 ** rng.uniform(lo, hi, (2, n))
    return W, tau, hpr_params(tau1=tau[0, 0], tau2=tau[1, 0], thermal=thermal)


def hpr_two_params(m1, m2):
    """The parameter block of the HPR two-material models (reduced, intermediate, multiphysics): the two materials'
    20-value hpr_params blocks, material k at [20 k] -- any equation of state, elastic or plastic."""
    m1, m2 = np.asarray(m1, dtype=np.float64), np.asarray(m2, dtype=np.float64)
    assert m1.shape == (20,) and m2.shape == (20,)
    return np.concatenate([m1, m2])


def hpr_reduced_params(gamma1=1.4, p_inf1=0.0, gamma2=1.67, p_inf2=0.0, c_v=2.5, rho0=1.0, T0=1.0, c_s=1.0, alpha=1.0,
                       tau1=1e-2, tau2=1e-2, T_ref=0.0, thermal=(True, True)):
    """Two StiffenedGas HPR materials with elastic strain relaxation for the HPR two-material models, as
    hpr_two_params' 40 values (p_ref 0, which the StiffenedGas branch does not read)."""
    def one(g, pinf, th):
        return hpr_params(gamma=g, p_inf=pinf, c_v=c_v, rho0=rho0, T0=T0, c_s=c_s, alpha=alpha, tau1=tau1, tau2=tau2,
                          T_ref=T_ref, p_ref=0.0, thermal=th)
    return hpr_two_params(one(gamma1, p_inf1, thermal[0]), one(gamma2, p_inf2, thermal[1]))


def _cold_pressure(rho, prm):
    """The reference pressure p_ref(rho) of a material's equation of state (HPR/hprmiegruneisen.cpp:30-66):
    ShockMieGruneisen and GodunovRomenski cold curves, -p_inf for StiffenedGas."""
    eos = int(prm[12])
    if eos == HPR_EOS["ShockMieGruneisen"]:
        return smg_reference_pressure(rho, prm)
    if eos == HPR_EOS["GodunovRomenski"]:
        return gr_reference_pressure(rho, prm)
    return -prm[1] + 0.0 * np.asarray(rho, dtype=np.float64)


def hpr_two_solid_riemann(nx, m1, m2, F_left, F_right, v_left, v_right, ny=1, p_offset=0.0, heat=0.0, seed=0):
    """A two-material solid Riemann problem in the shape of the reference's Barton and Zhang scenarios of the HPR
    two-material models (HPR/Multiphysics/hprreducedtests.cpp, hprintermediatetests.cpp:7-55): alpha1 0.999 at
    i <= nx/2 and 0.001 to the right, A = F^-1 and velocity v on each side, each material's density rho0_k det A, and
    the interface pressure the cold pressure of the side's dominant material plus p_offset (the reference takes it
    from its Elasticity module's hyperelastic equation of state, which this package does not carry); seeded heat flux
    of amplitude `heat`.  HPR reduced planes (19, nx) or (19, ny, nx), split along x."""
    m1, m2 = np.asarray(m1, dtype=np.float64), np.asarray(m2, dtype=np.float64)
    rng = np.random.default_rng(seed)
    shape = (ny, nx) if ny > 1 else (nx,)
    W = np.zeros((19,) + shape)
    left = np.broadcast_to(np.arange(nx) <= 0.5 * nx, shape)
    for side, F, v, dom, a1 in ((left, F_left, v_left, m1, 0.999), (~left, F_right, v_right, m2, 0.001)):
        A = np.linalg.inv(np.asarray(F, dtype=np.float64))
        d = np.linalg.det(A)
        W[0][side] = a1
        W[1][side] = _cold_pressure(dom[3] * d, dom) + p_offset
        for k in range(9):
            W[2 + k][side] = A.reshape(9)[k]
        for k in range(3):
            W[11 + k][side] = float(v[k])
        W[17][side] = m1[3] * d
        W[18][side] = m2[3] * d
    if heat:
        W[14:17] = heat * rng.standard_normal((3,) + shape)
    return W


def hpr_reduced_riemann(nx, ny=1, seed=0, distortion=0.02, heat=0.05, bubble=False):
    """A two-material HPR Riemann problem (material 1 in the left half, material 2 in the right; the reference's
    i <= n/2 convention; bubble=True in 2D: material 1 inside a disc of radius 0.3 about the centre), with a seeded
    distortion A = I + perturbation and heat flux J, as 19 primitive planes: alpha1, p, A(9), u, v, w, Jx, Jy, Jz,
    rho1, rho2; shape (19, n) or (19, ny, nx)."""
    rng = np.random.default_rng(seed)
    shape = (ny, nx) if ny > 1 else (nx,)
    W = np.zeros((19,) + shape)
    x = np.arange(nx)
    if bubble and ny > 1:
        yy, xx = np.meshgrid((np.arange(ny) + 0.5) / ny, (x + 0.5) / nx, indexing="ij")
        left = (xx - 0.5) ** 2 + (yy - 0.5) ** 2 <= 0.09
    else:
        left = (x <= 0.5 * nx) if ny == 1 else np.broadcast_to(x <= 0.5 * nx, shape)
    W[0] = np.where(left, 0.999, 0.001)
    W[1] = np.where(left, 1.0, 0.3)
    A = np.eye(3).reshape(9, *([1] * len(shape))) + distortion * rng.standard_normal((9,) + shape)
    W[2:11] = A
    W[11] = np.where(left, 0.2, -0.1)
    if ny > 1:
        W[12] = 0.05 * rng.standard_normal(shape)
    W[14:17] = heat * rng.standard_normal((3,) + shape)
    W[17] = np.where(left, 1.0, 0.8)
    W[18] = np.where(left, 0.5, 0.25)
    return W


HPR_INTERMEDIATE_NVAR = 20


def hpr_intermediate_from_reduced(W, p2_scale=1.0):
    """The HPR intermediate model's 20 planes (alpha1, A(9), u, v, w, Jx, Jy, Jz, rho1, p1, rho2, p2) of an HPR reduced
    state (alpha1, p, A(9), u, v, w, Jx, Jy, Jz, rho1, rho2): material 1 at the interface pressure, material 2 at
    p2_scale times it."""
    out = np.zeros((HPR_INTERMEDIATE_NVAR,) + W.shape[1:])
    out[0] = W[0]
    out[1:16] = W[2:17]
    out[16] = W[17]
    out[17] = W[1]
    out[18] = W[18]
    out[19] = p2_scale * W[1]
    return out


def hpr_intermediate_riemann(nx, ny=1, seed=0, distortion=0.02, heat=0.05, bubble=False, p2_scale=1.0):
    """hpr_reduced_riemann's two-material HPR Riemann problem in the intermediate model's planes, shape (20, n) or
    (20, ny, nx)."""
    return hpr_intermediate_from_reduced(hpr_reduced_riemann(nx, ny, seed, distortion, heat, bubble), p2_scale)


HPR_MULTIPHYSICS_NVAR = 32


def hpr_multiphysics_from_reduced(W, p2_scale=1.0, a2_scale=1.0):
    """The HPR multiphysics model's 32 planes (alpha1, u, v, w, rho1, p1, A1(9), J1(3), rho2, p2, A2(9), J2(3)) of a 1D
    HPR reduced state: material 1 at the interface pressure with the state's distortion and heat flux, material 2 at
    p2_scale times the pressure, with a2_scale times the distortion and half the heat flux."""
    assert W.ndim == 2, "the HPR multiphysics model is 1D only"
    out = np.zeros((HPR_MULTIPHYSICS_NVAR, W.shape[1]))
    out[0] = W[0]
    out[1:4] = W[11:14]
    out[4] = W[17]
    out[5] = W[1]
    out[6:15] = W[2:11]
    out[15:18] = W[14:17]
    out[18] = W[18]
    out[19] = p2_scale * W[1]
    out[20:29] = a2_scale * W[2:11]
    out[29:32] = 0.5 * W[14:17]
    return out


def hpr_multiphysics_riemann(nx, seed=0, distortion=0.02, heat=0.05, p2_scale=1.0, a2_scale=1.0):
    """hpr_reduced_riemann's 1D two-material HPR Riemann problem in the multiphysics model's planes, shape (32, nx)."""
    return hpr_multiphysics_from_reduced(hpr_reduced_riemann(nx, 1, seed, distortion, heat), p2_scale, a2_scale)


MHD_MULTIPHYSICS_NVAR = 16  # alpha1, u, v, w, rho1, p1, B1 (3), psi1, rho2, p2, B2 (3), psi2


def mhd_multiphysics_params(gamma1=2.0, p_inf1=0.0, gamma2=2.0, p_inf2=0.0, c_h1=0.0, c_h2=0.0):
    """The two MHDMaterialParameters of the MHD multiphysics model: (gamma1, p_inf1, gamma2, p_inf2, c_h1, c_h2).  The
    reference's solve leaves each material's hyperbolic wave speed as given (0 from MHDMaterialParameters(gamma))."""
    return np.array([gamma1, p_inf1, gamma2, p_inf2, c_h1, c_h2])


def mhd_multiphysics_dumbser_1d(n, seed=None, noise=0.0):
    """MHDMultiphysicsTests::solveDumbserTest1's layout (MHD/Multiphysics/mhdmultiphysicstests.cpp:7-26): material 1
    (rho 1, p 1, B (0.75, 1, 0)) and material 2 (rho 0.125, p 0.1, B (0.75, -1, 0)) in every cell, alpha1 0.999 at
    i <= n/2 and 0.001 to the right; optionally seeded noise of relative amplitude `noise` on the velocities, densities,
    pressures, fields and GLM scalars."""
    left = np.arange(n) <= 0.5 * n
    W = np.zeros((MHD_MULTIPHYSICS_NVAR, n))
    W[0] = np.where(left, 0.999, 0.001)
    W[4:10] = np.array([1.0, 1.0, 0.75, 1.0, 0.0, 0.0])[:, None]
    W[10:16] = np.array([0.125, 0.1, 0.75, -1.0, 0.0, 0.0])[:, None]
    if noise:
        rng = np.random.default_rng(seed)
        W[1:4] = noise * rng.standard_normal((3, n))
        for k in (4, 5, 6, 7, 8, 10, 11, 12, 13, 14):
            W[k] *= 1.0 + noise * rng.standard_normal(n)
        W[9] = noise * rng.standard_normal(n)
        W[15] = noise * rng.standard_normal(n)
    return W
