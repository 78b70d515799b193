"""Solution writers in the reference scenarios' `.dat` format, for side-by-side plots with Vanguard's own output.

Each file holds one row per cell, `x value` in 1D and `x_i x_j value` in 2D (row index first), with the cell
coordinate `spacing * index`, spacing = 1 / (number of cells, or of rows in 2D), and every number rendered as C++'s
default stream output renders a double (printf %g, 6 significant digits), as the reference's writers do:
  Euler 1D  density, xVelocity, yVelocity, zVelocity, pressure         (Euler/eulertests.cpp:54-80)
  MHD 1D    density, yMagneticField                                    (MHD/mhdtests.cpp:123-139)
  MHD 2D    density, yMagneticField                                    (MHD/mhdtests.cpp:141-161)
  HPR 1D    density, xVelocity, yVelocity, temperature, heatFlux       (HPR/hprtests.cpp:219-246)
  HPR 2D    density, xVelocity                                         (HPR/hprtests.cpp:248-269)
The planes are the primitive planes the solvers upload and download (Solver.download()).
"""
from __future__ import annotations

import os

import numpy as np


def _g(v: float) -> str:
    # C++ operator<<(double) with the default flags is printf("%g"); Python's "g" follows the same rules
    return format(float(v), "g")


def _write_1d(path: str, values) -> None:
    n = len(values)
    dx = 1.0 / n
    with open(path, "w") as f:
        for i, v in enumerate(values):
            f.write(f"{_g(dx * i)} {_g(v)}\n")


def _write_2d(path: str, values) -> None:
    rows, cols = values.shape
    d = 1.0 / rows
    with open(path, "w") as f:
        for i in range(rows):
            for j in range(cols):
                f.write(f"{_g(d * i)} {_g(d * j)} {_g(values[i, j])}\n")


def write_euler(planes, directory: str = ".") -> list[str]:
    """EulerTests::outputSolution of 1D Euler primitive planes (rho, u, v, w, p, lambda) x n."""
    planes = np.asarray(planes)
    if planes.ndim != 2:
        raise ValueError("the reference writes Euler solutions in 1D only")
    names = {"density": 0, "xVelocity": 1, "yVelocity": 2, "zVelocity": 3, "pressure": 4}
    out = []
    for name, k in names.items():
        out.append(os.path.join(directory, name + ".dat"))
        _write_1d(out[-1], planes[k])
    return out


def write_mhd(planes, directory: str = ".") -> list[str]:
    """MHDTests::outputSolution{,2D} of MHD primitive planes (rho, u, v, w, p, Bx, By, Bz, psi)."""
    planes = np.asarray(planes)
    write = _write_1d if planes.ndim == 2 else _write_2d
    out = []
    for name, k in (("density", 0), ("yMagneticField", 6)):
        out.append(os.path.join(directory, name + ".dat"))
        write(out[-1], planes[k])
    return out


def hpr_temperature(planes, params):
    """HPRStateVector::computeTemperature (HPR/hprmiegruneisen.cpp:212-221) of HPR primitive planes, every equation
    of state of the parameter block (params[12])."""
    prm = np.zeros(24)
    prm[:len(params)] = params
    rho, p = np.asarray(planes[0], dtype=np.float64), np.asarray(planes[1], dtype=np.float64)
    eos, rho0 = int(prm[12]), prm[3]
    if eos == 1:
        G = prm[13] * (rho0 / rho)
        v0 = 1.0 / rho0
        pref = np.where(rho > rho0, prm[14] ** 2 * ((v0 - 1.0 / rho) / (v0 - prm[15] * (v0 - 1.0 / rho)) ** 2),
                        prm[14] ** 2 * (rho - rho0))
    elif eos == 2:
        G = np.full_like(rho, prm[0])
        c = (rho / rho0) ** prm[16]
        pref = prm[14] ** 2 * (rho / prm[16]) * (c - 1.0) * c
    else:
        G = np.full_like(rho, prm[0] - 1.0)
        pref = np.full_like(rho, -prm[1])
    return prm[9] + (p - pref) / (rho * G * prm[2])


def write_hpr(planes, params, directory: str = ".") -> list[str]:
    """HPRTests::outputSolution{,2D} of HPR primitive planes (rho, p, A(9), u, v, w, Jx, Jy, Jz); the 1D files add
    the temperature and the x heat flux T alpha^2 Jx (HPREquationOfState::computeHeatFluxVector)."""
    planes = np.asarray(planes)
    out = []
    if planes.ndim == 3:
        for name, k in (("density", 0), ("xVelocity", 11)):
            out.append(os.path.join(directory, name + ".dat"))
            _write_2d(out[-1], planes[k])
        return out
    T = hpr_temperature(planes, params)
    series = {"density": planes[0], "xVelocity": planes[11], "yVelocity": planes[12], "temperature": T,
              "heatFlux": T * (params[6] * params[6] * planes[14])}
    for name, v in series.items():
        out.append(os.path.join(directory, name + ".dat"))
        _write_1d(out[-1], v)
    return out
