"""Tangent-linear (forward-mode) FP64 reference of the homogeneous HPR relaxation batch -- test infrastructure only.

It is the independent check of the hand-written adjoint of the source batch (vg_source_batch_gradient): jvp()
propagates dual numbers (value, tangent) through the same step as one sub-cycle of HPRForcingSolver's RK4 on a
spatially uniform field (Solvers/hprforcingsolver.cpp:332-357; the fractional flux predictor of such a field has
zero slopes and reduces to its primitive round trip), with
  * HPRStateVector::computeConservedVariableVector / setConservedVariableVector (HPR/hprstatevector.cpp:78-162),
  * the StiffenedGas branch of HPRMieGruneisen (HPR/hprmiegruneisen.cpp:7-102, :194-221) and the mesoscale
    energies of HPREquationOfState (HPR/hprequationofstate.cpp:7-81),
  * HPRStateVector::computeSourceTermVector (HPR/hprstatevector.cpp:312-366) with HPRSourceTerms' theta1 and
    theta2 (HPR/hprsourceterms.cpp:7-39, the elastic branch).
The value part follows the oracle's association order; the tangent part is the derivative of each operation.  It
shares no code with the device adjoint (which is reverse mode, written from the closed-form expressions).
Vectorised over the cells with numpy; tau1 and tau2 are per cell.
"""
from __future__ import annotations

import numpy as np

from oracle.tangent import Dual


def _pow(x: Dual, a: float) -> Dual:
    v = np.power(x.v, a)
    return Dual(v, a * np.power(x.v, a - 1.0) * x.d)


def _mat(a9):
    return [[a9[3 * i + j] for j in range(3)] for i in range(3)]


def _mul(a, b):
    return [[((0.0 + (a[i][0] * b[0][j])) + (a[i][1] * b[1][j])) + (a[i][2] * b[2][j]) for j in range(3)] for i in range(3)]


def _tmul(a, b):  # a^T b
    return [[((0.0 + (a[0][i] * b[0][j])) + (a[1][i] * b[1][j])) + (a[2][i] * b[2][j]) for j in range(3)] for i in range(3)]


def _dev(g):
    c = (((0.0 + g[0][0]) + g[1][1]) + g[2][2]) / 3.0
    return [[g[i][j] + (-1.0 * (c * (1.0 if i == j else 0.0))) for j in range(3)] for i in range(3)]


def _det(a):
    return ((a[0][0] * ((a[1][1] * a[2][2]) - (a[2][1] * a[1][2]))) -
            (a[0][1] * ((a[1][0] * a[2][2]) - (a[1][2] * a[2][0])))) + \
        (a[0][2] * ((a[1][0] * a[2][1]) - (a[1][1] * a[2][0])))


class Gas:
    """HPR material parameters of the StiffenedGas branch (the HPR block of vg_grid_desc)."""

    def __init__(self, params):
        p = list(params) + [0.0] * (24 - len(params))
        self.g, self.pinf, self.cv, self.rho0, self.T0, self.cs, self.alpha = p[0], p[1], p[2], p[3], p[4], p[5], p[6]
        self.Tref, self.thermal = p[9], p[11] != 0.0


def _meso(A, m: Gas):
    D = _dev(_tmul(A, A))
    s = 0.0
    for i in range(3):
        s = s + (((0.0 + (D[i][0] * D[i][0])) + (D[i][1] * D[i][1])) + (D[i][2] * D[i][2]))
    return (0.25 * (m.cs * m.cs)) * s


def _thermal_energy(j, m: Gas):
    return (0.5 * (m.alpha * m.alpha)) * (((j[0] * j[0]) + (j[1] * j[1])) + (j[2] * j[2]))


def cons(W, m: Gas):
    """17 primitive duals -> 17 conserved duals."""
    rho, p = W[0], W[1]
    A = _mat(W[2:11])
    u, j = W[11:14], W[14:17]
    e = (m.pinf / rho) + ((p - (-m.pinf)) / (rho * (m.g - 1.0)))
    E = (e + _meso(A, m)) + (0.5 * (((u[0] * u[0]) + (u[1] * u[1])) + (u[2] * u[2])))
    if m.thermal:
        E = E + _thermal_energy(j, m)
    zero = Dual(np.zeros_like(rho.v))
    U = [rho, rho * E] + list(W[2:11]) + [rho * u[0], rho * u[1], rho * u[2]]
    U += [rho * j[0], rho * j[1], rho * j[2]] if m.thermal else [zero, zero, zero]
    return U


def setcons(U, m: Gas, keep):
    """17 conserved duals -> 17 primitive duals; `keep` supplies J when the material is not thermal."""
    rho = U[0]
    A = _mat(U[2:11])
    u = [U[11] / rho, U[12] / rho, U[13] / rho]
    j = [U[14] / rho, U[15] / rho, U[16] / rho] if m.thermal else list(keep[14:17])
    e = (U[1] / rho) - ((0.5 * (((u[0] * u[0]) + (u[1] * u[1])) + (u[2] * u[2]))) + _meso(A, m))
    if m.thermal:
        e = e - _thermal_energy(j, m)
    p = (((e - (m.pinf / rho)) * rho) * (m.g - 1.0)) + (-m.pinf)
    return [rho, p] + list(U[2:11]) + u + j


def source(U, m: Gas, tau1, tau2):
    rho = U[0]
    A = _mat(U[2:11])
    cs2 = m.cs * m.cs
    AD = _mul(A, _dev(_tmul(A, A)))
    d = [[cs2 * AD[i][j] for j in range(3)] for i in range(3)]
    th1 = 3.0 * (_pow(_det(A), 5.0 / 3.0) / (cs2 * tau1))
    zero = Dual(np.zeros_like(rho.v))
    S = [zero, zero] + [(-d[i][j]) * th1 for i in range(3) for j in range(3)] + [zero] * 6
    if m.thermal:
        u = [U[11] / rho, U[12] / rho, U[13] / rho]
        j = [U[14] / rho, U[15] / rho, U[16] / rho]
        e = (U[1] / rho) - ((0.5 * (((u[0] * u[0]) + (u[1] * u[1])) + (u[2] * u[2]))) + _meso(A, m))
        e = e - _thermal_energy(j, m)
        p = (((e - (m.pinf / rho)) * rho) * (m.g - 1.0)) + (-m.pinf)
        T = m.Tref + ((p - (-m.pinf)) / ((rho * (m.g - 1.0)) * m.cv))
        a2 = m.alpha * m.alpha
        th2 = 1.0 / ((a2 * tau2) * ((rho / m.rho0) * (m.T0 / T)))
        for k in range(3):
            S[14 + k] = ((-rho) * th2) * (a2 * j[k])
    return S


def _roundtrip(U, m, default):
    return cons(setcons(U, m, default), m)


def step(W, m: Gas, tau1, tau2, h):
    """One source step of length h from primitive duals W (the uniform-field forcing sub-cycle)."""
    n = W[0].v.shape
    default = [Dual(np.zeros(n)) for _ in range(17)]
    default[0] = Dual(np.ones(n))
    default[1] = Dual(np.ones(n))
    for i in (2, 6, 10):
        default[i] = Dual(np.ones(n))
    U = cons(W, m)
    S = source(U, m, tau1, tau2)
    k = [[h * s for s in S]]
    for s in range(3):
        ut = [U[v] + ((0.5 * k[s][v]) if s < 2 else k[s][v]) for v in range(17)]
        ut = _roundtrip(ut, m, default)
        ut = [x + 0.0 for x in ut]
        ut = _roundtrip(ut, m, default)
        S = source(ut, m, tau1, tau2)
        k.append([h * x for x in S])
    Un = [U[v] + ((1.0 / 6.0) * (k[0][v] + ((2.0 * k[1][v]) + ((2.0 * k[2][v]) + k[3][v])))) for v in range(17)]
    return setcons(Un, m, W)


def jvp(W0, tau, params, h, steps, dW=None, dtau=None):
    """W(T) and its tangent along (dW, dtau) after `steps` steps; W0 (17, n), tau (2, n)."""
    m = Gas(params)
    n = W0.shape[1]
    dW = np.zeros_like(W0) if dW is None else dW
    dtau = np.zeros((2, n)) if dtau is None else dtau
    W = [Dual(W0[v], dW[v]) for v in range(17)]
    t1, t2 = Dual(tau[0], dtau[0]), Dual(tau[1], dtau[1])
    for _ in range(steps):
        W = step(W, m, t1, t2, h)
    return np.stack([w.v for w in W]), np.stack([w.d for w in W])
