"""ctypes bindings for the CPU oracle (test infrastructure only).

Two libraries sit behind this module:

* ``liboracle.so`` -- our plain-C restatement of the reference's SLIC/FORCE path (slic_oracle.c),
  built by ``make -C oracle oracle``.  It is the checker the CUDA path is compared against.
* ``_ref/libvgref.so`` -- the reference's own unmodified C++ sources plus an extern "C" harness
  (ref_harness.cpp), built by ``make -C oracle ref`` where the reference tree exists.  It pins the
  restatement and is the timed CPU baseline.

Only tests/, bench.py's CPU legs and __graft_entry__.smoke() import this module.  Arrays are numpy
float64 primitive planes of shape (nvar, ny, nx) (or (nvar, n) in 1D), C-contiguous, in the
reference's primitive order.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libvgref.so")

(EULER, MHD, HPR, EULER_REDUCED, EULER_MULTIPHYSICS, MHD_REDUCED, MHD_INTERMEDIATE, HPR_REDUCED, HPR_INTERMEDIATE,
 HPR_MULTIPHYSICS, MHD_MULTIPHYSICS) = 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10
NVAR = {EULER: 6, MHD: 9, HPR: 17}
TRANSMISSIVE, PERIODIC = 0, 1
SUPERBEE, VANLEER, MINBEE = 0, 1, 2

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_c_int, _c_double = ctypes.c_int, ctypes.c_double

_lib = None
_ref = None


def _ptr(a):
    return a.ctypes.data_as(_D) if a is not None else None


def _check(planes, nvar):
    if not (isinstance(planes, np.ndarray) and planes.dtype == np.float64 and planes.flags.c_contiguous):
        raise TypeError("planes must be a C-contiguous float64 numpy array")
    if planes.shape[0] != nvar:
        raise ValueError(f"expected {nvar} primitive planes, got {planes.shape[0]}")


def lib():
    """Load liboracle.so (our C restatement), building it on first use if missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            import subprocess
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        L = ctypes.CDLL(ORACLE_SO)
        L.vo_run1d.restype = _c_double
        L.vo_run1d.argtypes = [_c_int, _D, _c_int, _c_double, _c_double, _c_double, _c_int, _c_double,
                               _c_int, _D, _c_int, _c_int, _I, _D]
        L.vo_run2d.restype = _c_double
        L.vo_run2d.argtypes = [_c_int, _D, _c_int, _c_int, _c_double, _c_double, _c_double, _c_int,
                               _c_double, _c_int, _D, _c_int, _c_int, _I, _D]
        L.vo_sweep1d.argtypes = [_c_int, _D, _c_int, _c_double, _c_double, _c_double, _c_int, _D, _c_int]
        L.vo_sweep2d.argtypes = [_c_int, _D, _c_int, _c_int, _c_int, _c_double, _c_double, _c_double,
                                 _c_int, _D, _c_int]
        L.vo_max_wave1d.restype = _c_double
        L.vo_max_wave1d.argtypes = [_c_int, _D, _c_int, _D]
        L.vo_max_wave2d.restype = _c_double
        L.vo_max_wave2d.argtypes = [_c_int, _D, _c_int, _c_int, _D]
        L.vo_slope_limiter.restype = _c_double
        L.vo_slope_limiter.argtypes = [_c_double, _c_double, _c_int]
        for name in ("vo_prim_to_cons", "vo_cons_to_prim"):
            getattr(L, name).argtypes = [_c_int, _D, _D, _D]
        L.vo_flux.argtypes = [_c_int, _D, _c_int, _D, _D]
        L.vo_slic_flux.argtypes = [_c_int, _D, _D, _D, _D, _c_int, _c_double, _c_double, _c_double,
                                   _c_int, _D, _D]
        L.vo_nvar.restype = _c_int
        L.vo_nparams.restype = _c_int
        L.vo_forcing.argtypes = [_c_int, _D, _c_int, _c_int, _c_double, _c_double, _c_double, _c_int, _D, _c_int]
        L.vo_hpr_cell.argtypes = [_D, _D, _D, _D, _D, _D, _D]
        L.vo_run_first_order.restype = _c_double
        L.vo_run_first_order.argtypes = [_c_int, _D, _c_int, _c_int, _c_double, _c_double, _c_double, _c_int, _D,
                                         _c_int, ctypes.POINTER(_c_int)]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    """Load the compiled reference harness (oracle/_ref/libvgref.so)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_SO} not built (make -C oracle ref needs the reference tree)")
        R = ctypes.CDLL(REF_SO)
        R.vgref_first_order_run.restype = _c_double
        R.vgref_first_order_run.argtypes = [_c_int, _D, _c_int, _c_int, _c_double, _c_double, _c_double, _c_int, _D,
                                            _c_int, ctypes.POINTER(_c_int)]
        R.vgref_set_threads.restype = _c_int
        R.vgref_euler1d_batch_run.argtypes = [_D, _c_int, _I, _D, _D, _c_double, _c_int, _c_double, _c_int]
        R.vgref_set_threads.argtypes = [_c_int]
        R.vgref_euler1d_run.restype = _c_double
        R.vgref_euler1d_run.argtypes = [_D, _c_int, _c_double, _c_double, _c_double, _c_int, _c_double,
                                        _c_int, _D, _I]
        R.vgref_euler2d_run.restype = _c_double
        R.vgref_euler2d_run.argtypes = [_D, _c_int, _c_int, _c_double, _c_double, _c_double, _c_int,
                                        _c_double, _c_int, _D, _c_int, _I]
        R.vgref_euler2d_sweep.argtypes = [_D, _c_int, _c_int, _c_int, _c_double, _c_double, _c_double,
                                          _c_int, _D, _c_int]
        R.vgref_euler2d_max_wave_speed.restype = _c_double
        R.vgref_euler2d_max_wave_speed.argtypes = [_D, _c_int, _c_int, _D, _c_int]
        for name in ("vgref_mhd1d_run",):
            getattr(R, name).restype = _c_double
            getattr(R, name).argtypes = [_D, _c_int, _c_double, _c_double, _c_double, _c_int, _c_double,
                                         _c_int, _D, _c_int, _c_int, _I]
        R.vgref_mhd2d_run.restype = _c_double
        R.vgref_mhd2d_run.argtypes = [_D, _c_int, _c_int, _c_double, _c_double, _c_double, _c_int,
                                      _c_double, _c_int, _D, _c_int, _c_int, _I]
        if hasattr(R, "vgref_hpr_cell"):
            R.vgref_hpr_cell.argtypes = [_D, _D, _D, _D, _D, _D, _D]
        if hasattr(R, "vgref_hpr2d_run"):
            R.vgref_hpr2d_run.restype = _c_double
            R.vgref_hpr2d_run.argtypes = [_D, _c_int, _c_int, _c_double, _c_double, _c_double, _c_int,
                                          _c_double, _c_int, _D, _c_int, _c_int, _I]
            R.vgref_hpr1d_run.restype = _c_double
            R.vgref_hpr1d_run.argtypes = [_D, _c_int, _c_double, _c_double, _c_double, _c_int, _c_double,
                                          _c_int, _D, _c_int, _c_int, _I]
        _ref = R
    return _ref


# ------------------------------------------------------------------------------------ restatement

NPARAMS = 48  # size of every parameter block handed to the C libraries (VG_MAX_PARAMS)


def _params(params):
    """The model's parameter block zero-padded to NPARAMS (zero = StiffenedGas, non-plastic for HPR)."""
    p = np.zeros(NPARAMS)
    v = np.asarray(params, dtype=np.float64).ravel()
    p[:len(v)] = v
    return p


def _ref_runnable(model, prm):
    """The compiled reference cannot run a GodunovRomenski HPR material: its computeGruneisenCoefficientDerivative
    (HPR/hprmiegruneisen.cpp:104-119) has no return for that branch and, compiled with -O2, does not return."""
    if model == HPR and int(prm[12]) == 2:
        raise ValueError("the reference's GodunovRomenski wave speed does not return; use the oracle (run)")


def run(model, planes, dx, cfl, t_end=0.0, steps=0, bias=0.0, limiter=SUPERBEE, params=None,
        bc=TRANSMISSIVE, subcycles=0, dt_log=False):
    """Run solve()/solve2D()'s loop in the C restatement, in place.  Returns (t, steps[, dts])."""
    _check(planes, NVAR[model])
    prm = _params(params)
    st = ctypes.c_int()
    dts = np.zeros(max(steps, 1), dtype=np.float64) if dt_log else None
    if planes.ndim == 2:
        t = lib().vo_run1d(model, _ptr(planes), planes.shape[1], dx, cfl, t_end, steps, bias, limiter,
                           _ptr(prm), bc, subcycles, ctypes.byref(st), _ptr(dts))
    else:
        t = lib().vo_run2d(model, _ptr(planes), planes.shape[2], planes.shape[1], dx, cfl, t_end, steps,
                           bias, limiter, _ptr(prm), bc, subcycles, ctypes.byref(st), _ptr(dts))
    return (t, st.value, dts) if dt_log else (t, st.value)


def run_first_order(model, planes, dx, cfl, t_end=0.0, steps=0, params=None, bc=TRANSMISSIVE):
    """FirstOrderSolver::solve/solve2D's loop (and the MHD / HPR twins) in the C restatement, in place.
    Returns (t, steps)."""
    prm = _params(params)
    st = ctypes.c_int()
    nx, ny = (planes.shape[2], planes.shape[1]) if planes.ndim == 3 else (planes.shape[1], 1)
    if model in _TWO_MATERIAL_NW:  # the restatement carries one unused plane
        nw = _TWO_MATERIAL_NW[model]
        assert planes.shape[0] == nw and planes.dtype == np.float64 and planes.flags.c_contiguous
        padded = np.zeros((nw + 1,) + planes.shape[1:])
        padded[:nw] = planes
        t = lib().vo_run_first_order(model, _ptr(padded), nx, ny, dx, cfl, t_end, steps, _ptr(prm), bc,
                                     ctypes.byref(st))
        planes[:] = padded[:nw]
        return t, st.value
    _check(planes, NVAR[model])
    t = lib().vo_run_first_order(model, _ptr(planes), nx, ny, dx, cfl, t_end, steps, _ptr(prm), bc, ctypes.byref(st))
    return t, st.value


def ref_run_first_order(model, planes, dx, cfl, t_end=0.0, steps=0, params=None, bc=TRANSMISSIVE, threads=1):
    """The reference's first-order loop from its own per-step functions, in place.  Returns (t, steps)."""
    _check(planes, NVAR[model])
    R = ref()
    R.vgref_set_threads(threads)
    prm = _params(params)
    _ref_runnable(model, prm)
    st = ctypes.c_int()
    nx, ny = (planes.shape[2], planes.shape[1]) if planes.ndim == 3 else (planes.shape[1], 1)
    t = R.vgref_first_order_run(model, _ptr(planes), nx, ny, dx, cfl, t_end, steps, _ptr(prm), bc, ctypes.byref(st))
    return t, st.value


def sweep(model, planes, axis, dx, dt, bias=0.0, limiter=SUPERBEE, params=None, bc=TRANSMISSIVE):
    _check(planes, NVAR[model])
    prm = _params(params)
    if planes.ndim == 2:
        lib().vo_sweep1d(model, _ptr(planes), planes.shape[1], dx, dt, bias, limiter, _ptr(prm), bc)
    else:
        lib().vo_sweep2d(model, _ptr(planes), planes.shape[2], planes.shape[1], axis, dx, dt, bias, limiter,
                         _ptr(prm), bc)


def max_wave(model, planes, params):
    """The CFL maximum wave speed of the grid (with the default-state corner ghosts in 2D)."""
    if model in _TWO_MATERIAL_NW:  # the restatement carries one unused plane
        nw = _TWO_MATERIAL_NW[model]
        assert planes.shape[0] == nw and planes.dtype == np.float64
        padded = np.zeros((nw + 1,) + planes.shape[1:])
        padded[:nw] = planes
        planes = padded
    else:
        _check(planes, NVAR[model])
    prm = _params(params)
    if planes.ndim == 2:
        return lib().vo_max_wave1d(model, _ptr(planes), planes.shape[1], _ptr(prm))
    return lib().vo_max_wave2d(model, _ptr(planes), planes.shape[2], planes.shape[1], _ptr(prm))


def forcing(planes, dx, dt, bias=0.0, limiter=SUPERBEE, params=None, bc=TRANSMISSIVE):
    """One HPR RK4 relaxation-source sub-cycle over the grid (restatement), in place."""
    _check(planes, NVAR[HPR])
    prm = _params(params)
    nx, ny = (planes.shape[2], planes.shape[1]) if planes.ndim == 3 else (planes.shape[1], 1)
    lib().vo_forcing(HPR, _ptr(planes), nx, ny, dx, dt, bias, limiter, _ptr(prm), bc)


def hpr_cell(w, params, reference=False):
    """(U, F_x, F_y, S, (speed_x, speed_y)) of one HPR primitive state, from the restatement or the reference."""
    w = np.ascontiguousarray(w, dtype=np.float64)
    prm = _params(params)
    outs = [np.zeros(17) for _ in range(4)]
    sp = np.zeros(2)
    fn = ref().vgref_hpr_cell if reference else lib().vo_hpr_cell
    fn(_ptr(w), _ptr(prm), *[_ptr(o) for o in outs], _ptr(sp))
    return (*outs, sp)


_TWO_MATERIAL_NW = {EULER_REDUCED: 7, EULER_MULTIPHYSICS: 8, MHD_REDUCED: 11, MHD_INTERMEDIATE: 12, HPR_REDUCED: 19,
                    HPR_INTERMEDIATE: 20, HPR_MULTIPHYSICS: 32, MHD_MULTIPHYSICS: 16}
# the two-material models with a source (their loops take sub-cycles: MHD GLM damping, HPR relaxation)
_MHD_TWO_MATERIAL = (MHD_REDUCED, MHD_INTERMEDIATE, HPR_REDUCED, HPR_INTERMEDIATE, HPR_MULTIPHYSICS, MHD_MULTIPHYSICS)


def run_two_material(model, planes, dx, cfl, t_end=0.0, steps=0, bias=0.0, limiter=SUPERBEE, params=None, reinit=0,
                     reference=False, threads=1, bc=TRANSMISSIVE, subcycles=0):
    """(MHD)SecondOrderSolver::solve{,2D} of a two-material model on its primitive planes, in place: EULER_REDUCED
    (7 planes: alpha1, u, v, w, rho1, rho2, p), EULER_MULTIPHYSICS (8: alpha1, u, v, w, rho1, p1, rho2, p2) or
    MHD_REDUCED (11: alpha1, u, v, w, rho1, rho2, p, Bx, By, Bz, psi), MHD_INTERMEDIATE (12: alpha1, u, v, w, rho1,
    p1, rho2, p2, Bx, By, Bz, psi), HPR_REDUCED (19: alpha1, p, A(9), u, v, w, Jx, Jy, Jz, rho1, rho2) or
    HPR_INTERMEDIATE (20: alpha1, A(9), u, v, w, Jx, Jy, Jz, rho1, p1, rho2, p2) or HPR_MULTIPHYSICS (32, 1D only:
    alpha1, u, v, w, rho1, p1, A1(9), J1(3), rho2, p2, A2(9), J2(3)) or MHD_MULTIPHYSICS (16, 1D only: alpha1, u, v,
    w, rho1, p1, B1(3), psi1, rho2, p2, B2(3), psi2; params (gamma1, p_inf1, gamma2, p_inf2, c_h1, c_h2); its loop has
    no source and no reinitialisation), x (n) or (ny, nx); from the restatement or (reference=True) the reference.  params = (gamma1, p_inf1, gamma2, p_inf2); the HPR models: 11 per
    material, {gamma, p_inf, c_v, rho0, T0, c_s, alpha, tau1, tau2, T_ref, is_thermal} each; reinit > 0
    reinitialises the volume fraction every `reinit` steps; subcycles > 0 (the MHD models: GLM damping; the HPR
    models: the relaxation source) adds the RK4 forcing sub-cycles.
    Returns (t, steps)."""
    nw = _TWO_MATERIAL_NW[model]
    assert subcycles == 0 or model in _MHD_TWO_MATERIAL, "only the MHD and HPR two-material models have a source"
    assert planes.shape[0] == nw and planes.dtype == np.float64 and planes.flags.c_contiguous
    nx = planes.shape[-1]
    ny = 1 if planes.ndim == 2 else planes.shape[1]
    prm = _params(params)
    st = ctypes.c_int()
    if reference:
        assert bc == TRANSMISSIVE, "the reference's two-material models have transmissive boundaries only"
        R = ref()
        R.vgref_set_threads(threads)
        if model in _MHD_TWO_MATERIAL:
            # the intermediate model's own solve2D pads with its defective insertBoundaryCells2D
            # (Solvers/mhdsolvers.cpp:213); the harness's per-step loop builds mirror ghosts instead
            assert not (model == MHD_INTERMEDIATE and ny > 1 and steps <= 0), "2D intermediate: per-step runs only"
            if model == MHD_MULTIPHYSICS:
                assert ny == 1, "the reference's MHD multiphysics model is 1D only"
                fn = R.vgref_mhd_multiphysics_run
                fn.restype = _c_double
                t = fn(_ptr(planes), nx, _c_double(dx), _c_double(cfl), _c_double(t_end), steps, _c_double(bias),
                       limiter, _ptr(prm), ctypes.byref(st))
                return t, st.value
            if model == HPR_MULTIPHYSICS:
                assert ny == 1, "the reference's HPR multiphysics model is 1D only"
                fn = R.vgref_hpr_multiphysics_run
                fn.restype = _c_double
                t = fn(_ptr(planes), nx, _c_double(dx), _c_double(cfl), _c_double(t_end), steps, _c_double(bias),
                       limiter, _ptr(prm), subcycles, reinit, ctypes.byref(st))
                return t, st.value
            fn = {MHD_REDUCED: R.vgref_mhd_reduced_run, HPR_REDUCED: R.vgref_hpr_reduced_run,
                  HPR_INTERMEDIATE: R.vgref_hpr_intermediate_run}.get(model, R.vgref_mhd_intermediate_run)
            fn.restype = _c_double
            t = fn(_ptr(planes), nx, ny, _c_double(dx), _c_double(cfl), _c_double(t_end), steps, _c_double(bias),
                   limiter, _ptr(prm), subcycles, reinit, ctypes.byref(st))
            return t, st.value
        fn = R.vgref_reduced_run if model == EULER_REDUCED else R.vgref_multiphysics_run
        fn.restype = _c_double
        t = fn(_ptr(planes), nx, ny, _c_double(dx), _c_double(cfl), _c_double(t_end), steps, _c_double(bias), limiter,
               _ptr(prm), reinit, ctypes.byref(st))
        return t, st.value
    padded = np.zeros((nw + 1,) + planes.shape[1:])  # the restatement carries one unused plane
    padded[:nw] = planes
    L = lib()
    if model in _MHD_TWO_MATERIAL:
        L.vo_run_mhd_two_material.restype = _c_double
        t = L.vo_run_mhd_two_material(model, _ptr(padded), nx, ny, _c_double(dx), _c_double(cfl), _c_double(t_end),
                                      steps, _c_double(bias), limiter, _ptr(prm), bc, subcycles, reinit,
                                      ctypes.byref(st))
    else:
        L.vo_run_two_material.restype = _c_double
        t = L.vo_run_two_material(model, _ptr(padded), nx, ny, _c_double(dx), _c_double(cfl), _c_double(t_end),
                                  steps, _c_double(bias), limiter, _ptr(prm), bc, reinit, ctypes.byref(st))
    planes[:] = padded[:nw]
    return t, st.value


def run_reduced(planes, dx, cfl, **kw):
    """run_two_material of the reduced model (7 planes)."""
    return run_two_material(EULER_REDUCED, planes, dx, cfl, **kw)


def hpr_eos(params, rho, p, e, reference=False):
    """(n, 13) HPR Mie-Grueneisen values at densities rho (see vo_hpr_eos), from the restatement or the
    reference's own functions (NaN where the reference's GodunovRomenski derivative does not return)."""
    rho, p, e = (np.ascontiguousarray(x, dtype=np.float64) for x in (rho, p, e))
    out = np.zeros((len(rho), 13))
    fn = ref().vgref_hpr_eos if reference else lib().vo_hpr_eos
    fn(_ptr(_params(params)), _ptr(rho), _ptr(p), _ptr(e), len(rho), _ptr(out))
    return out


def hpr_theta1(params, rho, A, reference=False):
    """HPRSourceTerms::computeTheta1Reciprocal of densities rho (n,) and distortions A (n, 3, 3)."""
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    A = np.ascontiguousarray(A, dtype=np.float64)
    out = np.zeros(len(rho))
    fn = ref().vgref_hpr_theta1 if reference else lib().vo_hpr_theta1
    fn(_ptr(_params(params)), _ptr(rho), _ptr(A), len(rho), _ptr(out))
    return out


# ------------------------------------------------------------------------------------ reference

def ref_write(model, planes, directory, params=None):
    """The reference scenarios' own .dat writers (EulerTests / MHDTests / HPRTests::outputSolution{,2D}) on
    primitive planes, into `directory` (they write into the working directory, which is switched around the
    call)."""
    planes = np.ascontiguousarray(planes, dtype=np.float64)
    nx = planes.shape[-1]
    ny = 1 if planes.ndim == 2 else planes.shape[1]
    R = ref()
    cwd = os.getcwd()
    os.chdir(directory)
    try:
        if model == EULER:
            R.vgref_write_euler(_ptr(planes), nx)
        elif model == MHD:
            R.vgref_write_mhd(_ptr(planes), nx, ny)
        else:
            R.vgref_write_hpr(_ptr(planes), nx, ny, _ptr(_params(params)))
    finally:
        os.chdir(cwd)


def ref_batch_run(planes, ncell, dx, gamma, cfl, steps, bias=0.0, limiter=SUPERBEE, threads=0):
    """The reference's way of solving a ragged batch of 1D Euler problems: SecondOrderSolver::solve's per-step loop
    once per problem, `steps` steps each, the problems spread over `threads` OpenMP threads (0: all host cores), one
    thread per problem.  planes: (6, total) primitives of all problems concatenated, updated in place.  Returns the
    thread count used."""
    _check(planes, 6)
    R = ref()
    n = R.vgref_set_threads(threads)
    nc = np.ascontiguousarray(ncell, dtype=np.int32)
    dxa = np.ascontiguousarray(dx, dtype=np.float64)
    ga = np.ascontiguousarray(gamma, dtype=np.float64)
    if planes.shape[1] != int(nc.sum()):
        raise ValueError("planes must hold sum(ncell) cells")
    R.vgref_euler1d_batch_run(_ptr(planes), len(nc), nc.ctypes.data_as(_I), _ptr(dxa), _ptr(ga), cfl, steps, bias,
                              limiter)
    return n


def ref_run(model, planes, dx, cfl, t_end=0.0, steps=0, bias=0.0, limiter=SUPERBEE, params=None,
            bc=TRANSMISSIVE, subcycles=0, threads=1):
    """Run the reference's own code on the same planes, in place.  steps <= 0 calls solve()/solve2D()
    itself (time-driven, transmissive only).  Returns (t, steps); solve() reports neither (-1, -1)."""
    _check(planes, NVAR[model])
    R = ref()
    R.vgref_set_threads(threads)
    prm = _params(params)
    _ref_runnable(model, prm)
    st = ctypes.c_int()
    if model == EULER and planes.ndim == 2:
        t = R.vgref_euler1d_run(_ptr(planes), planes.shape[1], dx, cfl, t_end, steps, bias, limiter,
                                _ptr(prm), ctypes.byref(st))
    elif model == EULER:
        t = R.vgref_euler2d_run(_ptr(planes), planes.shape[2], planes.shape[1], dx, cfl, t_end, steps, bias,
                                limiter, _ptr(prm), bc, ctypes.byref(st))
    elif model == MHD and planes.ndim == 2:
        t = R.vgref_mhd1d_run(_ptr(planes), planes.shape[1], dx, cfl, t_end, steps, bias, limiter, _ptr(prm),
                              bc, subcycles, ctypes.byref(st))
    elif model == MHD:
        t = R.vgref_mhd2d_run(_ptr(planes), planes.shape[2], planes.shape[1], dx, cfl, t_end, steps, bias,
                              limiter, _ptr(prm), bc, subcycles, ctypes.byref(st))
    elif model == HPR and planes.ndim == 2:
        t = R.vgref_hpr1d_run(_ptr(planes), planes.shape[1], dx, cfl, t_end, steps, bias, limiter, _ptr(prm),
                              bc, subcycles, ctypes.byref(st))
    else:
        t = R.vgref_hpr2d_run(_ptr(planes), planes.shape[2], planes.shape[1], dx, cfl, t_end, steps, bias,
                              limiter, _ptr(prm), bc, subcycles, ctypes.byref(st))
    return t, st.value
