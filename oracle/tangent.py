"""Tangent-linear (forward-mode) FP64 reference of the batched 1D Euler SLIC loop -- test infrastructure only.

It is the independent check of the hand-written discrete adjoint: for a direction d of the initial primitives
(rho, u, p of every cell) and of gamma, jvp() returns L and dL[d] by propagating dual numbers (value, tangent)
through the same step as SecondOrderSolver::solve (Solvers/secondordersolver.cpp:288-314) on one instance:
  * dt = CFL dx / S with S = max_i (|u_i| + c_i) (Solvers/solvers.cpp:259-276, :437-452), x0.2 for steps 0..5;
  * two transmissive ghosts each side (Solvers/solvers.cpp:17-23);
  * slopes with the limiter of SlopeLimiters (Solvers/slopelimiters.cpp:7-74, :217-246);
  * half-step evolution of both cell edges with the primitive round trip (Solvers/solvers.cpp:454-466);
  * FORCE flux (Solvers/firstordersolver.cpp:173-200) and the conservative update with setcons.
The value part uses the operations, in the same association order, as the C oracle, so it equals the oracle's
and the device's forward bit for bit (the tests check that).  Non-smooth points take the derivative of the
branch the value part takes: the comparisons of the limiter and of std::min, zero for the floored ratio operand,
sign(u) for |u| (0 at 0), and the first cell attaining the CFL maximum.
Vectorised over the cells of one instance with numpy; instances are independent and summed.
"""
from __future__ import annotations

import numpy as np

FLOOR5 = 10.0 ** -5.0


class Dual:
    """value + eps * tangent, elementwise over numpy arrays (or scalars)."""

    __slots__ = ("v", "d")

    def __init__(self, v, d=0.0):
        self.v = np.asarray(v, dtype=np.float64)
        self.d = np.asarray(d, dtype=np.float64) + np.zeros_like(self.v)

    @staticmethod
    def lift(x):
        return x if isinstance(x, Dual) else Dual(x, 0.0)

    def __add__(self, o):
        o = Dual.lift(o)
        return Dual(self.v + o.v, self.d + o.d)

    __radd__ = __add__

    def __sub__(self, o):
        o = Dual.lift(o)
        return Dual(self.v - o.v, self.d - o.d)

    def __rsub__(self, o):
        return Dual.lift(o) - self

    def __mul__(self, o):
        o = Dual.lift(o)
        return Dual(self.v * o.v, self.d * o.v + self.v * o.d)

    __rmul__ = __mul__

    def __truediv__(self, o):
        o = Dual.lift(o)
        q = self.v / o.v
        return Dual(q, (self.d - q * o.d) / o.v)

    def __rtruediv__(self, o):
        return Dual.lift(o) / self

    def __neg__(self):
        return Dual(-self.v, -self.d)

    def __getitem__(self, idx):
        return Dual(self.v[idx], self.d[..., idx])


def sqrt(x: Dual) -> Dual:
    r = np.sqrt(x.v)
    return Dual(r, x.d / (2.0 * r))


def fabs(x: Dual) -> Dual:
    return Dual(np.abs(x.v), np.sign(x.v) * x.d)


def where(c, a, b) -> Dual:
    a, b = Dual.lift(a), Dual.lift(b)
    return Dual(np.where(c, a.v, b.v), np.where(c, a.d, b.d))


def std_min(a, b) -> Dual:
    """std::min(a, b) = b < a ? b : a"""
    a, b = Dual.lift(a), Dual.lift(b)
    return where(b.v < a.v, b, a)


def limiter(r: Dual, w: float, lim: int) -> Dual:
    """SlopeLimiters::computeSlopeLimiter (Solvers/slopelimiters.cpp:7-74): 0 superbee, 1 van Leer, 2 minbee."""
    with np.errstate(divide="ignore", invalid="ignore"):
        xr = 2.0 / ((1.0 - w) + ((1.0 + w) * r))
        zero = Dual(np.zeros_like(r.v))
        if lim == 0:
            big = std_min(std_min(r, xr), 2.0)
            out = where(r.v < 1.0, Dual(np.ones_like(r.v)), big)
            out = where(r.v < 0.5, 2.0 * r, out)
        elif lim == 1:
            out = std_min((2.0 * r) / (1.0 + r), xr)
        else:
            out = where(r.v < 1.0, r, std_min(1.0, xr))
        return where(r.v < 0.0, zero, out)


def slope(uL: Dual, u: Dual, uR: Dual, bias: float, lim: int) -> Dual:
    """One component of SlopeLimiters::computeSlopeVector (Solvers/slopelimiters.cpp:217-246)."""
    dm = u - uL
    dp = uR - u
    s = ((0.5 * (1.0 + bias)) * dm) + ((0.5 * (1.0 - bias)) * dp)
    num = where(np.abs(dm.v) < FLOOR5, FLOOR5, dm)
    den = where(np.abs(dp.v) < FLOOR5, FLOOR5, dp)
    return s * limiter(num / den, bias, lim)


def cons(W, g, pinf):
    """EulerStateVector::computeConservedVariableVector (Euler/eulerstatevector.cpp:78-91)."""
    rho, u, p = W
    e = (p + (g * pinf)) / ((g - 1.0) * rho)
    return [rho, rho * u, rho * ((0.5 * (u * u)) + e)]


def setcons(U, g, pinf):
    """EulerStateVector::setConservedVariableVector (Euler/eulerstatevector.cpp:47-61)."""
    rho = U[0]
    u = U[1] / rho
    e = (U[2] / rho) - (0.5 * (u * u))
    return [rho, u, ((e * (g - 1.0)) * rho) - (g * pinf)]


def flux(U, g, pinf):
    """EulerStateVector::computeXFluxVector (Euler/eulerstatevector.cpp:93-120)."""
    rho = U[0]
    u = U[1] / rho
    E = U[2] / rho
    e = E - (0.5 * (u * u))
    p = ((e * (g - 1.0)) * rho) - (g * pinf)
    return [rho * u, (rho * (u * u)) + p, (rho * (u * E)) + (u * p)]


def max_wave(W, g, pinf) -> Dual:
    """Solvers::computeMaximumWaveSpeed (Solvers/solvers.cpp:259-276): the tangent of the first maximum."""
    rho, u, p = W
    s = fabs(u) + sqrt((g * (p + pinf)) / rho)
    i = int(np.argmax(s.v))  # first index attaining the maximum
    return Dual(s.v[i], s.d[..., i:i + 1])


def step(W, g, pinf, dx, cfl, s, bias, lim):
    """One SLIC step of one instance; W = [rho, u, p] Duals over its n cells."""
    S = max_wave(W, g, pinf)
    dt = cfl * (dx / S)
    if s <= 5:
        dt = dt * 0.2
    r = dt / dx
    rinv = dx / dt
    half_r = 0.5 * (dt / dx)
    n = W[0].v.shape[0]
    U = cons(W, g, pinf)
    gi = np.concatenate([[1, 0], np.arange(n), [n - 1, n - 2]])  # ghosts -2, -1, cells, n, n + 1
    Ug = [u[gi] for u in U]
    # evolved edges of positions 1 .. n + 2 (ghost -1 .. ghost n)
    xl, xr = [], []
    for v in range(3):
        sl = slope(Ug[v][0:n + 2], Ug[v][1:n + 3], Ug[v][2:n + 4], bias, lim)
        xl.append(Ug[v][1:n + 3] - (0.5 * sl))
        xr.append(Ug[v][1:n + 3] + (0.5 * sl))
    fl, fr = flux(xl, g, pinf), flux(xr, g, pinf)
    ev = [half_r * (fl[v] - fr[v]) for v in range(3)]
    a = cons(setcons([xl[v] + ev[v] for v in range(3)], g, pinf), g, pinf)  # left edges
    b = cons(setcons([xr[v] + ev[v] for v in range(3)], g, pinf), g, pinf)  # right edges
    # FORCE at the n + 1 interfaces between positions j and j + 1 (j = ghost -1 .. cell n - 1)
    ua = [b[v][0:n + 1] for v in range(3)]
    ub = [a[v][1:n + 2] for v in range(3)]
    fa, fb = flux(ua, g, pinf), flux(ub, g, pinf)
    uri = [0.5 * ((ua[v] + ub[v]) + (r * (fa[v] - fb[v]))) for v in range(3)]
    fri = flux(uri, g, pinf)
    F = [0.5 * ((0.5 * ((fa[v] + fb[v]) + (rinv * (ua[v] - ub[v])))) + fri[v]) for v in range(3)]
    Un = [U[v] + (r * (F[v][0:n] - F[v][1:n + 1])) for v in range(3)]
    return setcons(Un, g, pinf)


def _instance(W, g, pinf, dx, target, cfl, steps, bias, lim):
    for s in range(steps):
        W = step(W, g, pinf, dx, cfl, s, bias, lim)
    diff = W[0] - target
    sq = diff * diff
    return float(np.sum(sq.v)), np.sum(sq.d, axis=-1), W[0].v


def jvp(ncell, dx, gamma, W0, target_rho, cfl, steps, bias, lim, dW0=None, dgamma=None, p_inf=None):
    """L = sum (rho(T) - target)^2 and its directional derivative along (dW0, dgamma).

    W0, dW0: (6, total) Euler primitive planes (rho, u, v, w, p, lambda), only rho, u, p used; dgamma (ninst,).
    Returns (L, dL, final rho plane)."""
    total = int(np.sum(ncell))
    dW0 = np.zeros((6, total)) if dW0 is None else dW0
    dgamma = np.zeros(len(ncell)) if dgamma is None else dgamma
    L = dL = 0.0
    rho_T = np.empty(total)
    off = 0
    for k, n in enumerate(ncell):
        sl = slice(off, off + n)
        g = Dual(gamma[k], dgamma[k])
        pinf = 0.0 if p_inf is None else float(p_inf[k])
        W = [Dual(W0[i, sl], dW0[i, sl]) for i in (0, 1, 4)]
        Lk, dLk, rho_T[sl] = _instance(W, g, pinf, float(dx[k]), target_rho[sl], cfl, steps, bias, lim)
        L += Lk
        dL += float(dLk)
        off += n
    return L, dL, rho_T


def gradient(ncell, dx, gamma, W0, target_rho, cfl, steps, bias, lim, p_inf=None):
    """Full gradient by forward mode: per instance, one tangent direction per initial (rho, u, p) value of each
    of its cells and one for gamma, propagated together.  Returns (L, dL/dW0 as (6, total), dL/dgamma)."""
    total = int(np.sum(ncell))
    G = np.zeros((6, total))
    gg = np.zeros(len(ncell))
    L = 0.0
    off = 0
    for k, n in enumerate(ncell):
        sl = slice(off, off + n)
        nd = 3 * n + 1
        seeds = np.eye(nd)
        W = [Dual(W0[i, sl], seeds[:, j * n:(j + 1) * n]) for j, i in enumerate((0, 1, 4))]
        g = Dual(gamma[k], seeds[:, 3 * n:3 * n + 1])
        pinf = 0.0 if p_inf is None else float(p_inf[k])
        Lk, dLk, _ = _instance(W, g, pinf, float(dx[k]), target_rho[sl], cfl, steps, bias, lim)
        L += Lk
        for j, i in enumerate((0, 1, 4)):
            G[i, sl] = dLk[j * n:(j + 1) * n]
        gg[k] = dLk[3 * n]
        off += n
    return L, G, gg
