"""Generate the golden fixtures in tests/golden/ by running the reference's own code.

The reference (Vanguard) ships no golden vectors or known-answer tests, so the fixtures are produced by
running its unmodified OpenMP C++ sources, compiled into oracle/_ref/libvgref.so by oracle/Makefile, on
one thread (its CFL maximum is an unsynchronised OpenMP update and is only reproducible on one thread).
Each fixture stores the input primitive planes, the run parameters and the reference's output planes.

Run from the repository root where the reference tree is present:
    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from vanguard_b200 import workloads as wl  # noqa: E402

# name -> (model, initial planes, run kwargs).  steps == 0: the reference's own time-driven solve().
CASES = {
    # the 1D Sod benchmark case exactly: 1000 cells, minbee, CFL 0.9, t = 0.25, transmissive
    "euler1d_sod1000_minbee_t025": (O.EULER, lambda: wl.sod_1d(1000),
                                     dict(dx=1e-3, cfl=0.9, t_end=0.25, steps=0, limiter=O.MINBEE,
                                          params=wl.euler_params(1.4))),
    "euler2d_quad64_superbee_50": (O.EULER, lambda: wl.euler_quadrants_2d(64, 64, seed=7),
                                   dict(dx=1 / 64, cfl=0.8, steps=50, limiter=O.SUPERBEE,
                                        params=wl.euler_params(1.4))),
    "euler2d_quad48x40_vanleer_20": (O.EULER, lambda: wl.euler_quadrants_2d(48, 40, seed=8),
                                     dict(dx=1 / 48, cfl=0.8, steps=20, limiter=O.VANLEER,
                                          params=wl.euler_params(1.4))),
    "euler2d_quad40_minbee_t005": (O.EULER, lambda: wl.euler_quadrants_2d(40, 40, seed=9),
                                   dict(dx=1 / 40, cfl=0.8, t_end=0.05, steps=0, limiter=O.MINBEE,
                                        params=wl.euler_params(1.4))),
    "mhd2d_vortex48_periodic_superbee_30": (O.MHD, lambda: wl.mhd_vortex_2d(48, 48, seed=1),
                                            dict(dx=1 / 48, cfl=0.8, steps=30, limiter=O.SUPERBEE,
                                                 params=wl.mhd_params(5 / 3), bc=O.PERIODIC)),
    "mhd1d_briowu200_superbee_t01": (O.MHD, lambda: wl.brio_wu_1d(200),
                                     dict(dx=1 / 200, cfl=0.8, t_end=0.1, steps=0, limiter=O.SUPERBEE,
                                          params=wl.mhd_params(2.0))),
    # HPR, thermal, StiffenedGas ideal gas: sweeps only, then with the RK4 relaxation source sub-cycled
    "hpr2d_smooth24x20_superbee_10": (O.HPR, lambda: wl.hpr_smooth_2d(24, 20, seed=3),
                                      dict(dx=1 / 24, cfl=0.8, steps=10, limiter=O.SUPERBEE,
                                           params=wl.hpr_params(tau1=1e-2, tau2=1e-2))),
    "hpr2d_smooth16_rk4sub1_4": (O.HPR, lambda: wl.hpr_smooth_2d(16, 16, seed=4),
                                 dict(dx=1 / 16, cfl=0.8, steps=4, limiter=O.SUPERBEE, subcycles=1,
                                      params=wl.hpr_params(tau1=1e-2, tau2=1e-2))),
    "hpr1d_heat100_rk4sub2_20": (O.HPR, lambda: wl.hpr_heat_conduction_1d(100),
                                 dict(dx=1 / 100, cfl=0.8, steps=20, limiter=O.SUPERBEE, subcycles=2,
                                      params=wl.hpr_params(tau1=1e-1, tau2=1e-1))),
    # HPR solids: the ShockMieGruneisen equation of state, thermal with the RK4 source, and 2D sweeps only
    "hpr1d_shockmg60_thermal_rk4sub2_12": (O.HPR, lambda: wl.hpr_shock_riemann(60, 1, wl.hpr_shock_mg_params(thermal=True, tau1=0.1)),
                                           dict(dx=1 / 60, cfl=0.8, steps=12, limiter=O.SUPERBEE, subcycles=2,
                                                params=wl.hpr_shock_mg_params(thermal=True, tau1=0.1))),
    "hpr2d_shockmg20x16_minbee_8": (O.HPR, lambda: wl.hpr_shock_riemann(20, 16, wl.hpr_shock_mg_params(), seed=2),
                                    dict(dx=1 / 20, cfl=0.8, steps=8, limiter=O.MINBEE,
                                         params=wl.hpr_shock_mg_params())),
    # HPR plastic strain relaxation (StiffenedGas gas, theta1 scaled by (|sigma| / sigma0)^n), RK4 source
    "hpr1d_heat80_plastic_rk4sub2_16": (O.HPR, lambda: wl.hpr_heat_conduction_1d(80),
                                        dict(dx=1 / 80, cfl=0.8, steps=16, limiter=O.SUPERBEE, subcycles=2,
                                             params=wl.hpr_params(tau1=1e-2, tau2=1e-1, plastic=True, sigma0=0.05,
                                                                  n=2.0))),
}


# The Euler reduced two-material model (model id O.EULER_REDUCED): run by oracle.run_reduced's reference arm.
REDUCED_CASES = {
    "reduced1d_toro100_superbee_30": (lambda: wl.reduced_shock_tube(100),
                                      dict(dx=1 / 100, cfl=0.8, steps=30, limiter=O.SUPERBEE, reinit=0,
                                           params=wl.reduced_params(1.4, 0.0, 1.4, 0.0))),
    "reduced1d_twogamma120_minbee_reinit4_40": (lambda: wl.reduced_shock_tube(120, rho=(1.0, 0.1379), p=(2.0, 1.0)),
                                                 dict(dx=1 / 120, cfl=0.8, steps=40, limiter=O.MINBEE, reinit=4,
                                                      params=wl.reduced_params(1.4, 0.0, 1.67, 0.0))),
    "reduced2d_bubble32_superbee_reinit3_9": (lambda: wl.reduced_bubble_2d(32),
                                              dict(dx=1 / 32, cfl=0.8, steps=9, limiter=O.SUPERBEE, reinit=3,
                                                   params=wl.reduced_params(1.4, 0.0, 1.67, 0.0))),
}
# The Euler multiphysics two-material model (model id O.EULER_MULTIPHYSICS), same layouts, per-material pressures.
MULTIPHYSICS_CASES = {
    "multiphysics1d_twogamma120_superbee_reinit4_40": (
        lambda: wl.multiphysics_from_reduced(wl.reduced_shock_tube(120, rho=(1.0, 0.1379), p=(2.0, 1.0))),
        dict(dx=1 / 120, cfl=0.8, steps=40, limiter=O.SUPERBEE, reinit=4,
             params=wl.reduced_params(1.4, 0.0, 1.67, 0.0))),
    "multiphysics2d_bubble30x26_minbee_reinit3_9": (
        lambda: wl.multiphysics_from_reduced(wl.reduced_bubble_2d(30, 26)),
        dict(dx=1 / 30, cfl=0.8, steps=9, limiter=O.MINBEE, reinit=3, params=wl.reduced_params(1.4, 0.0, 1.67, 0.0))),
}
# The MHD reduced two-material model (model id O.MHD_REDUCED) on MHDReducedTests' Dumbser layouts: one material
# (gamma 2) and two (1.4, 1.67), RK4 GLM damping sub-cycles, reinitialisation, and one run of the reference's own
# MHDSecondOrderSolver::solve to t_end (steps = 0).
MHD_REDUCED_CASES = {
    "mhdreduced1d_dumbser100_superbee_30": (lambda: wl.mhd_reduced_dumbser_1d(100),
                                            dict(dx=1 / 100, cfl=0.8, steps=30, limiter=O.SUPERBEE, reinit=0,
                                                 subcycles=0, params=wl.mhd_reduced_params())),
    "mhdreduced1d_dumbsermm100_minbee_glm2_reinit4_30": (lambda: wl.mhd_reduced_dumbser_1d(100),
                                                         dict(dx=1 / 100, cfl=0.8, steps=30, limiter=O.MINBEE,
                                                              reinit=4, subcycles=2,
                                                              params=wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0))),
    "mhdreduced1d_dumbser60_solve_t01_glm1_reinit5": (lambda: wl.mhd_reduced_dumbser_1d(60),
                                                      dict(dx=1 / 60, cfl=0.8, t_end=0.1, steps=0, limiter=0,
                                                           reinit=5, subcycles=1, params=wl.mhd_reduced_params())),
    "mhdreduced2d_dumbsermm24x20_superbee_glm1_reinit3_6": (lambda: wl.mhd_reduced_dumbser_2d(24, 20),
                                                            dict(dx=1 / 24, cfl=0.8, steps=6, limiter=O.SUPERBEE,
                                                                 reinit=3, subcycles=1,
                                                                 params=wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0))),
}
# The MHD intermediate two-material model (model id O.MHD_INTERMEDIATE) on the same layouts, both materials at the
# interface pressure.  In 2D the reference's own solve2D pads the grid with a defective insertBoundaryCells2D
# (Solvers/mhdsolvers.cpp:213), so the 2D fixture comes from its per-step functions over mirror ghosts.
MHD_INTERMEDIATE_CASES = {
    "mhdintermediate1d_dumbsermm100_minbee_glm2_reinit4_30": (
        lambda: wl.mhd_intermediate_from_reduced(wl.mhd_reduced_dumbser_1d(100)),
        dict(dx=1 / 100, cfl=0.8, steps=30, limiter=O.MINBEE, reinit=4, subcycles=2,
             params=wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0))),
    "mhdintermediate1d_dumbsermm80_solve_t005_glm1_reinit5": (
        lambda: wl.mhd_intermediate_from_reduced(wl.mhd_reduced_dumbser_1d(80)),
        dict(dx=1 / 80, cfl=0.8, t_end=0.05, steps=0, limiter=O.MINBEE, reinit=5, subcycles=1,
             params=wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0))),
    "mhdintermediate2d_dumbsermm24x20_superbee_glm1_reinit3_6": (
        lambda: wl.mhd_intermediate_from_reduced(wl.mhd_reduced_dumbser_2d(24, 20)),
        dict(dx=1 / 24, cfl=0.8, steps=6, limiter=O.SUPERBEE, reinit=3, subcycles=1,
             params=wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0))),
}
# The HPR reduced two-material model (model id O.HPR_REDUCED): a seeded Riemann problem with distortion and heat flux
# (material 1 left, the stiffened material 2 right) in 1D, to t_end through the reference's own solve and per step with
# neither material thermal (the reference then drops the input J), and a 2D bubble with the reinitialisation.
HPR_REDUCED_PRM = wl.hpr_reduced_params(gamma2=2.0, p_inf2=0.5)
HPR_REDUCED_CASES = {
    "hprreduced1d_riemann80_solve_t002_sub1_reinit4": (
        lambda: wl.hpr_reduced_riemann(80, 1, seed=80),
        dict(dx=1 / 80, cfl=0.8, t_end=0.02, steps=0, limiter=O.MINBEE, reinit=4, subcycles=1,
             params=HPR_REDUCED_PRM)),
    "hprreduced1d_riemann60_minbee_cold_sub1_reinit2_12": (
        lambda: wl.hpr_reduced_riemann(60, 1, seed=60),
        dict(dx=1 / 60, cfl=0.8, steps=12, limiter=O.MINBEE, reinit=2, subcycles=1,
             params=wl.hpr_reduced_params(gamma2=2.0, p_inf2=0.5, thermal=(False, False)))),
    "hprreduced2d_bubble20_minbee_reinit2_6": (
        lambda: wl.hpr_reduced_riemann(20, 20, seed=20, bubble=True),
        dict(dx=1 / 20, cfl=0.8, steps=6, limiter=O.MINBEE, reinit=2, subcycles=0, params=HPR_REDUCED_PRM)),
}
# The HPR intermediate two-material model (model id O.HPR_INTERMEDIATE): the reduced model's problems in its planes,
# material 2 at 1.2 times the interface pressure, through the reference's own solve and solve2D to t_end and per step
# with cold materials.
HPR_INTERMEDIATE_CASES = {
    "hprintermediate1d_riemann80_solve_t002_sub1_reinit4": (
        lambda: wl.hpr_intermediate_riemann(80, 1, seed=80, p2_scale=1.2),
        dict(dx=1 / 80, cfl=0.8, t_end=0.02, steps=0, limiter=O.MINBEE, reinit=4, subcycles=1,
             params=HPR_REDUCED_PRM)),
    "hprintermediate1d_riemann60_superbee_cold_sub1_reinit2_12": (
        lambda: wl.hpr_intermediate_riemann(60, 1, seed=60),
        dict(dx=1 / 60, cfl=0.8, steps=12, limiter=O.SUPERBEE, reinit=2, subcycles=1,
             params=wl.hpr_reduced_params(gamma2=2.0, p_inf2=0.5, thermal=(False, False)))),
    "hprintermediate2d_bubble16_solve_t002_sub1_reinit4": (
        lambda: wl.hpr_intermediate_riemann(16, 16, seed=16, bubble=True, p2_scale=1.2),
        dict(dx=1 / 16, cfl=0.8, t_end=0.02, steps=0, limiter=O.MINBEE, reinit=4, subcycles=1,
             params=HPR_REDUCED_PRM)),
    "hprintermediate2d_bubble20_vanleer_reinit2_6": (
        lambda: wl.hpr_intermediate_riemann(20, 20, seed=20, bubble=True),
        dict(dx=1 / 20, cfl=0.8, steps=6, limiter=O.VANLEER, reinit=2, subcycles=0, params=HPR_REDUCED_PRM)),
}
# The HPR multiphysics two-material model (model id O.HPR_MULTIPHYSICS, 1D only): the reduced model's problem with a
# distortion and heat flux per material, through the reference's own solve to t_end, and per step up to its
# reinitialisation with material 2 cold.
HPR_MULTIPHYSICS_CASES = {
    "hprmultiphysics1d_riemann80_solve_t0015_sub2": (
        lambda: wl.hpr_multiphysics_riemann(80, seed=80, p2_scale=1.2),
        dict(dx=1 / 80, cfl=0.8, t_end=0.015, steps=0, limiter=O.MINBEE, reinit=0, subcycles=2,
             params=HPR_REDUCED_PRM)),
    "hprmultiphysics1d_riemann50_vanleer_cold2_reinit1_2": (
        lambda: wl.hpr_multiphysics_riemann(50, seed=5, p2_scale=1.1, a2_scale=1.01),
        dict(dx=1 / 50, cfl=0.8, steps=2, limiter=O.VANLEER, reinit=1, subcycles=0,
             params=wl.hpr_reduced_params(gamma2=2.0, p_inf2=0.5, thermal=(True, False)))),
}
# The HPR two-material models with solid materials, the reference's own scenarios for them (HPR/Multiphysics/
# hprintermediatetests.cpp): an elastic ShockMieGruneisen solid against a plastic one, in the layout of the reference's
# Zhang test (its deformation gradients and velocities), through the reference's own solve to t_end, and in 2D with the
# Barton deformation gradients.  GodunovRomenski solids cannot be run here: the reference's acoustic tensors of these
# models call computeGruneisenCoefficientDerivative, which has no GodunovRomenski return (HPR/hprmiegruneisen.cpp:
# 104-119) and compiled with -O2 does not return.
HPR_SOLID1 = wl.hpr_shock_mg_params(tau1=0.05)
HPR_SOLID2 = wl.hpr_shock_mg_params(plastic=True, sigma0=0.3, n=2.0, tau1=1.0)
HPR_SOLID_PRM = wl.hpr_two_params(HPR_SOLID1, HPR_SOLID2)
HPR_SOLID2_MILD = wl.hpr_shock_mg_params(plastic=True, sigma0=1.0, n=1.0, tau1=1.0)


def _zhang_solids(nx, ny=1):
    return wl.hpr_two_solid_riemann(nx, HPR_SOLID1, HPR_SOLID2, *wl.ZHANG_F, (0.0, 0.2, 0.1), (0.0, -0.03, -0.01),
                                    ny=ny)


HPR_REDUCED_CASES["hprreduced1d_smgplastic60_solve_t002_sub2_reinit4"] = (
    lambda: _zhang_solids(60),
    dict(dx=1 / 60, cfl=0.8, t_end=0.02, steps=0, limiter=O.MINBEE, reinit=4, subcycles=2, params=HPR_SOLID_PRM))
HPR_INTERMEDIATE_CASES["hprintermediate2d_smgplastic16x12_minbee_sub2_6"] = (
    lambda: wl.hpr_intermediate_from_reduced(wl.hpr_two_solid_riemann(16, HPR_SOLID1, HPR_SOLID2_MILD, *wl.BARTON_F,
                                                                      (0.0, 0.3, 0.5), (0.0, 0.0, 0.0), ny=12)),
    dict(dx=1 / 16, cfl=0.8, steps=6, limiter=O.MINBEE, reinit=0, subcycles=2,
         params=wl.hpr_two_params(HPR_SOLID1, HPR_SOLID2_MILD)))
HPR_MULTIPHYSICS_CASES["hprmultiphysics1d_smgplastic60_solve_t003_sub1_reinit3"] = (
    lambda: wl.hpr_multiphysics_from_reduced(_zhang_solids(60)),
    dict(dx=1 / 60, cfl=0.8, t_end=0.03, steps=0, limiter=O.MINBEE, reinit=3, subcycles=1, params=HPR_SOLID_PRM))
# The MHD multiphysics two-material model (model id O.MHD_MULTIPHYSICS, 1D only): MHDMultiphysicsTests'
# solveDumbserMultimaterialTest1 setting through the reference's own solve, and a perturbed layout per step with
# non-zero hyperbolic wave speeds.
MHD_MULTIPHYSICS_CASES = {
    "mhdmultiphysics1d_dumbsermm80_solve_t005": (
        lambda: wl.mhd_multiphysics_dumbser_1d(80),
        dict(dx=1 / 80, cfl=0.8, t_end=0.05, steps=0, limiter=O.SUPERBEE, reinit=0, subcycles=0,
             params=wl.mhd_multiphysics_params(1.4, 0.0, 1.67, 0.0))),
    "mhdmultiphysics1d_dumbser60_noise_glm_minbee_20": (
        lambda: wl.mhd_multiphysics_dumbser_1d(60, seed=6, noise=1e-2),
        dict(dx=1 / 60, cfl=0.8, steps=20, limiter=O.MINBEE, reinit=0, subcycles=0,
             params=wl.mhd_multiphysics_params(1.4, 0.1, 1.67, 0.0, 0.5, 0.7))),
}
TWO_MATERIAL = {O.EULER_REDUCED: REDUCED_CASES, O.EULER_MULTIPHYSICS: MULTIPHYSICS_CASES,
                O.MHD_REDUCED: MHD_REDUCED_CASES, O.MHD_INTERMEDIATE: MHD_INTERMEDIATE_CASES,
                O.HPR_REDUCED: HPR_REDUCED_CASES, O.HPR_INTERMEDIATE: HPR_INTERMEDIATE_CASES,
                O.HPR_MULTIPHYSICS: HPR_MULTIPHYSICS_CASES, O.MHD_MULTIPHYSICS: MHD_MULTIPHYSICS_CASES}


def make_two_material(name):
    model = next(m for m, cases in TWO_MATERIAL.items() if name in cases)
    init, kw = TWO_MATERIAL[model][name]
    w0 = np.ascontiguousarray(init())
    out = w0.copy()
    kw2 = dict(kw)
    O.run_two_material(model, out, kw2.pop("dx"), kw2.pop("cfl"), reference=True, **kw2)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), model=model, w0=w0, out=out,
                        **{k: np.asarray(v) for k, v in kw.items()})
    print("wrote", name)


def make(name):
    if any(name in cases for cases in TWO_MATERIAL.values()):
        return make_two_material(name)
    model, init, kw = CASES[name]
    w0 = np.ascontiguousarray(init())
    out = w0.copy()
    kw = dict(kw)
    O.ref_run(model, out, kw.pop("dx"), kw.pop("cfl"), threads=1, **kw)
    _, _, kw2 = CASES[name]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), model=model, w0=w0, out=out,
                        **{k: np.asarray(v) for k, v in kw2.items()})
    print("wrote", name)


if __name__ == "__main__":
    for n in (sys.argv[1:] or list(CASES) + [n for cases in TWO_MATERIAL.values() for n in cases]):
        make(n)
