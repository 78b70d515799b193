"""The drop-in C++ surface (vanguard_b200/shim: the reference's class names over the C ABI) driven by a
Vanguard-style caller (tests/shim/shim_driver.cpp), compared with the oracle on the same inputs."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(HERE, "shim", "shim_driver")


def _rel(a, b):
    r = np.where(a == b, 0.0, np.abs(a - b) / np.maximum(np.abs(b), 1e-300))
    return float(r.max())


def test_shim_driver_matches_oracle(gpu, oracle_lib, tmp_path):
    if not os.path.exists(DRIVER):
        pytest.fail("tests/shim/shim_driver was not built (python -m vanguard_b200.build)")
    out = tmp_path / "shim.bin"
    subprocess.run([DRIVER, str(out)], check=True, timeout=300)
    data = np.fromfile(out, dtype=np.float64)
    off = 0

    def take(shape):
        nonlocal off
        n = int(np.prod(shape))
        a = data[off:off + n].reshape(shape)
        off += n
        return a

    # 1) SecondOrderSolver::solve, shock tube 200 cells, minbee, CFL 0.9, t = 0.1
    got = take((6, 200))
    ref = wl.sod_1d(200)
    O.run(O.EULER, ref, 1 / 200, 0.9, t_end=0.1, limiter=O.MINBEE, params=wl.euler_params(1.4))
    assert np.array_equal(got, ref)

    # 2) the per-step loop built from insertBoundaryCells2D / computeStableTimeStep2D / X, Y sweeps
    got = take((6, 20, 24))
    W = np.zeros((6, 20, 24))
    W[5] = 1.0
    same = (np.arange(20)[:, None] < 10) == (np.arange(24)[None, :] < 12)
    W[0] = np.where(same, 1.0, 0.3)
    W[1] = np.where(same, 0.1, -0.1)
    W[2] = np.where(same, -0.2, 0.3)
    W[4] = np.where(same, 1.0, 0.4)
    O.run(O.EULER, W, 1 / 24, 0.8, t_end=1.0, steps=6, limiter=0, params=wl.euler_params(1.4))
    assert np.array_equal(got, W)

    # 3) MHDSecondOrderSolver::solve2D, 16^2 vortex, to t = 0.02
    got = take((9, 16, 16))
    # the driver builds this field with libm's sin; math.sin is the same libm call, numpy's may differ in an ulp
    import math
    g, s, n = 5 / 3, 1 / math.sqrt(4 * math.pi), 16
    ref = np.zeros((9, n, n))
    for i in range(n):
        for j in range(n):
            x, y = (j + 0.5) / n, (i + 0.5) / n
            ref[:, i, j] = [g * g, -math.sin(2 * math.pi * y), math.sin(2 * math.pi * x), 0.0, g,
                            -math.sin(2 * math.pi * y) * s, math.sin(4 * math.pi * x) * s, 0.0, 0.0]
    O.run(O.MHD, ref, 1 / 16, 0.8, t_end=0.02, limiter=0, params=wl.mhd_params(5 / 3))
    assert np.array_equal(got, ref)

    # 4) HPRSecondOrderSolver::solve, heat-conduction material, one RK4 sub-cycle, to t = 0.02
    got = take((17, 50))
    mu, cs, pref, kappa, rho0, T0, alpha = 1e-2, 1.0, 1.0, 1e-2, 1.0, 1.0, 2.0
    prm = wl.hpr_params(c_v=2.5, alpha=alpha, tau1=6.0 * (mu / (pref * (cs * cs))),
                        tau2=kappa * (rho0 / (T0 * (alpha * alpha))))
    ref = wl.hpr_heat_conduction_1d(50)
    O.run(O.HPR, ref, 1 / 50, 0.8, t_end=0.02, limiter=0, params=prm, subcycles=1)
    assert _rel(got, ref) <= 1e-12

    # 5) the step-count overload solve(..., maxSteps = 37) with no end time
    got = take((6, 150))
    ref = wl.sod_1d(150)
    O.run(O.EULER, ref, 1 / 150, 0.8, steps=37, limiter=0, params=wl.euler_params(1.4))
    assert np.array_equal(got, ref)

    # 6) FirstOrderSolver::solve, to t = 0.05
    got = take((6, 150))
    ref = wl.sod_1d(150)
    O.run_first_order(O.EULER, ref, 1 / 150, 0.8, t_end=0.05, params=wl.euler_params(1.4))
    assert np.array_equal(got, ref)

    # 7) HPRSecondOrderSolver::solve(..., maxSteps = 20), the Zhang GodunovRomenski plastic material, 2 sub-cycles;
    #    a solid equation of state calls pow in every pressure recovery: per-plane normwise bound (test_hpr_solids_gpu)
    got = take((17, 60))
    zp = wl.hpr_zhang_params()
    ref = wl.hpr_solid_riemann_1d(60, zp, np.eye(3), np.eye(3), (0.75, 0.0, 0.0), (-0.75, 0.0, 0.0))
    O.run(O.HPR, ref, 10.0 / 60, 0.8, steps=20, limiter=0, params=zp, subcycles=2)
    d = np.abs(got - ref).max(axis=1) / np.maximum(np.abs(ref).max(axis=1), 1e-300)
    assert np.isfinite(got).all() and d.max() <= 1e-10

    # 8) SecondOrderSolver::solve of the reduced two-material model, reinitialisation every 5 steps, t = 0.05
    got = take((7, 120))
    ref = wl.reduced_shock_tube(120)
    O.run_reduced(ref, 1 / 120, 0.8, t_end=0.05, limiter=0, params=wl.reduced_params(1.4, 0.0, 1.67, 0.0), reinit=5)
    assert np.array_equal(got, ref)

    # 9) SecondOrderSolver::solve of the multiphysics two-material model, reinitialisation every 4 steps, t = 0.04
    got = take((8, 100))
    ref = wl.multiphysics_from_reduced(wl.reduced_shock_tube(100, rho=(1.0, 0.1379), p=(2.0, 1.0)))
    O.run_two_material(O.EULER_MULTIPHYSICS, ref, 1 / 100, 0.8, t_end=0.04, limiter=0,
                       params=wl.reduced_params(1.4, 0.0, 1.67, 0.0), reinit=4)
    assert np.array_equal(got, ref)

    # 10) MHDSecondOrderSolver::solve2D of the MHD reduced two-material model, one GLM sub-cycle, reinit every 3 steps
    got = take((11, 24, 24))
    ref = wl.mhd_reduced_dumbser_2d(24)
    O.run_two_material(O.MHD_REDUCED, ref, 1 / 24, 0.8, steps=6, limiter=0, params=wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0),
                       reinit=3, subcycles=1)
    assert np.array_equal(got, ref)

    # 11) MHDSecondOrderSolver::solve of the MHD intermediate two-material model to t = 0.05
    got = take((12, 80))
    ref = wl.mhd_intermediate_from_reduced(wl.mhd_reduced_dumbser_1d(80))
    O.run_two_material(O.MHD_INTERMEDIATE, ref, 1 / 80, 0.8, t_end=0.05, limiter=2,
                       params=wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0), reinit=5, subcycles=1)
    assert np.array_equal(got, ref)

    # 12) computeMaximumWaveSpeed2D over exactly the cells given (interior only: no default-state corners), and
    #     solve2D on a single row refused with std::invalid_argument
    smax = take((1,))[0]
    j, i = np.meshgrid(np.arange(8), np.arange(6))
    rho, u, v, p = 1.0 + 0.01 * j, 0.01 * i, -0.02 * j, 0.01 + 0.001 * i
    expect = (np.maximum(np.abs(u), np.abs(v)) + np.sqrt((1.4 * (p + 0.0)) / rho)).max()
    assert smax == expect
    assert smax < np.sqrt(1.4)  # below the default state's speed, which the padded-grid maximum would add
    assert take((1,))[0] == 1.0

    # 13) HPRSecondOrderSolver::solve2D of the HPR reduced two-material model, one sub-cycle (pow in the source: 1e-12
    #     per cell), reinitialisation every 2 steps, 4 steps
    import math as m
    hprm = wl.hpr_reduced_params(gamma2=2.0, p_inf2=0.5)
    got = take((19, 16, 16))
    n = 16
    ref = np.zeros((19, n, n))
    for i in range(n):
        for j in range(n):
            r = m.sqrt(((i - 0.5 * n) * (i - 0.5 * n)) + ((j - 0.5 * n) * (j - 0.5 * n)))
            A = [1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0]
            ref[:, i, j] = ([0.999, 1.0, *A, 0.2, 0.0, 0.0, 0.02, 0.0, 0.0, 1.0, 0.5] if r <= 0.3 * n
                            else [0.001, 0.3, *A, -0.1, 0.0, 0.0, 0.0, 0.01, 0.0, 0.8, 0.25])
    O.run_two_material(O.HPR_REDUCED, ref, 1 / n, 0.8, t_end=1.0, steps=4, limiter=2, params=hprm, subcycles=1,
                       reinit=2)
    assert _rel(got, ref) <= 1e-12

    # 14) HPRSecondOrderSolver::solve of the HPR intermediate two-material model to t = 0.02, one sub-cycle
    got = take((20, 60))
    n = 60
    ref = np.zeros((20, n))
    for i in range(n):
        A = [1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0]
        ref[:, i] = ([0.999, *A, 0.2, 0.0, 0.0, 0.02, 0.0, 0.0, 1.0, 1.0, 0.5, 1.0] if i <= 0.5 * n
                     else [0.001, *A, -0.1, 0.0, 0.0, 0.0, 0.01, 0.0, 0.8, 0.3, 0.25, 0.36])
    O.run_two_material(O.HPR_INTERMEDIATE, ref, 1 / n, 0.8, t_end=0.02, limiter=2, params=hprm, subcycles=1, reinit=4)
    assert _rel(got, ref) <= 1e-12

    # 15) HPRSecondOrderSolver::solve of the HPR multiphysics two-material model to t = 0.015 (pow(alpha, 1/3) in the
    #     conserved distortion: 1e-12 of each plane's largest magnitude)
    got = take((32, 60))
    n = 60
    ref = np.zeros((32, n))
    I3 = [1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0]
    A2 = [1.01, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.99]
    for i in range(n):
        ref[:, i] = ([0.999, 0.2, 0.0, 0.0, 1.0, 1.0, *I3, 0.02, 0.0, 0.0, 0.5, 1.1, *A2, 0.01, 0.0, 0.0] if i <= 0.5 * n
                     else [0.001, -0.1, 0.0, 0.0, 0.8, 0.3, *I3, 0.0, 0.01, 0.0, 0.25, 0.33, *A2, 0.0, 0.005, 0.0])
    O.run_two_material(O.HPR_MULTIPHYSICS, ref, 1 / n, 0.8, t_end=0.015, limiter=2, params=hprm, subcycles=2)
    d = np.abs(got - ref).max(axis=1) / np.maximum(np.abs(ref).max(axis=1), 1e-300)
    assert np.isfinite(got).all() and d.max() <= 1e-12

    # 16) MHDSecondOrderSolver::solve of the MHD multiphysics two-material model to t = 0.05 (pow(alpha, 1/2) in the
    #     conserved fields: 1e-12 of each plane's largest magnitude)
    got = take((16, 80))
    ref = wl.mhd_multiphysics_dumbser_1d(80)
    O.run_two_material(O.MHD_MULTIPHYSICS, ref, 1 / 80, 0.8, t_end=0.05, limiter=0,
                       params=wl.mhd_multiphysics_params(1.4, 0.0, 1.67, 0.0))
    d = np.abs(got - ref).max(axis=1) / np.maximum(np.abs(ref).max(axis=1), 1e-300)
    assert np.isfinite(got).all() and d.max() <= 1e-12

    # 17) HPRSecondOrderSolver::solve of the HPR intermediate two-material model with the GodunovRomenski aluminium |
    #     copper of HPRIntermediateTests::solveZhangTest to t = 0.01 (pow in the equation of state: 1e-10 of each
    #     plane's largest magnitude).  The driver's literals are these states' shortest round-trip decimals.
    got = take((20, 60))
    al = wl.hpr_params(gamma=1.0, p_inf=0.0, c_v=9.0e-4, rho0=2.71, T0=300.0, c_s=3.16, alpha=2.0, tau1=1e8, tau2=0.0,
                       T_ref=300.0, p_ref=73.0, thermal=False, eos="GodunovRomenski", Gamma0=1.0, c0=5.037, s=1.338,
                       alpha_eos=1.0, n=1.338)
    cu = wl.hpr_params(gamma=1.0, p_inf=0.0, c_v=3.94e-4, rho0=8.9, T0=300.0, c_s=2.1,
                       alpha=8.9 * 3.909 * np.sqrt(4.0e-4 / 300.0), tau1=1e8, tau2=0.0, T_ref=300.0, p_ref=0.0,
                       thermal=False, eos="GodunovRomenski", c0=3.909, alpha_eos=1.0, n=1.0)
    ref = wl.hpr_intermediate_from_reduced(
        wl.hpr_two_solid_riemann(60, al, cu, *wl.ZHANG_F, (2.0, 0.0, 0.1), (0.0, -0.03, -0.01)))
    O.run_two_material(O.HPR_INTERMEDIATE, ref, 1 / 60, 0.8, t_end=0.01, limiter=2, params=wl.hpr_two_params(al, cu),
                       subcycles=1, reinit=3)
    d = np.abs(got - ref).max(axis=1) / np.maximum(np.abs(ref).max(axis=1), 1e-300)
    assert np.isfinite(got).all() and d.max() <= 1e-10

    assert take((1,))[0] == 6
    assert off == data.size
