"""vanguard_b200 -- B200-native SLIC/FORCE finite-volume update (Euler, ideal MHD, HPR).

The product is the CUDA library ``libvanguard_slic.so`` behind the C ABI in include/vanguard_slic.h and
the C++ shim in vanguard_b200/shim (Vanguard's own class names).  This module is a thin ctypes binding
of that C ABI used by the tests and bench.py; it has no compute path of its own and raises if the
library is missing or no GPU is present.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvanguard_slic.so")

VG_OK, VG_EINVAL, VG_ENAN, VG_ETIMEOUT, VG_ECUDA, VG_ENOMEM, VG_EUNSUPPORTED = range(7)
(EULER, MHD, HPR, EULER_REDUCED, EULER_MULTIPHYSICS, MHD_REDUCED, MHD_INTERMEDIATE, HPR_REDUCED, HPR_INTERMEDIATE,
 HPR_MULTIPHYSICS, MHD_MULTIPHYSICS) = 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10
FP64, MIXED = 0, 1
TRANSMISSIVE, PERIODIC = 0, 1
SUPERBEE, VANLEER, MINBEE = 0, 1, 2
NVAR = {EULER: 6, MHD: 9, HPR: 17, EULER_REDUCED: 7, EULER_MULTIPHYSICS: 8, MHD_REDUCED: 11, MHD_INTERMEDIATE: 12,
        HPR_REDUCED: 19, HPR_INTERMEDIATE: 20, HPR_MULTIPHYSICS: 32, MHD_MULTIPHYSICS: 16}
MAX_PARAMS = 48


class VgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{_STATUS.get(status, status)}: {msg}")
        self.status = status


_STATUS = {0: "VG_OK", 1: "VG_EINVAL", 2: "VG_ENAN", 3: "VG_ETIMEOUT", 4: "VG_ECUDA", 5: "VG_ENOMEM",
           6: "VG_EUNSUPPORTED"}


class GridDesc(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("precision", ctypes.c_int), ("boundary", ctypes.c_int), ("device", ctypes.c_int),
                ("params", ctypes.c_double * MAX_PARAMS)]


class RunConfig(ctypes.Structure):
    _fields_ = [("dx", ctypes.c_double), ("cfl", ctypes.c_double), ("t_end", ctypes.c_double),
                ("max_steps", ctypes.c_int), ("bias", ctypes.c_double), ("limiter", ctypes.c_int),
                ("subcycles", ctypes.c_int), ("order", ctypes.c_int), ("stiff_source", ctypes.c_int),
                ("reinit_frequency", ctypes.c_int)]


# Every function the C ABI header declares (tests check the library exports them all).
EXPORTS = ["vg_create", "vg_destroy", "vg_model_nvar", "vg_upload_primitive", "vg_download_primitive", "vg_run",
           "vg_solve", "vg_sweep", "vg_max_wave_speed", "vg_max_wave_speed_cells", "vg_state_device",
           "vg_last_launch_count", "vg_last_error_string", "vg_status_string", "vg_max_wave_speed_noalloc",
           "vg_autotune", "vg_set_launch_config", "vg_get_launch_config", "vg_set_schedule", "vg_get_schedule",
           "vg_batch_create", "vg_batch_destroy", "vg_batch_total_cells", "vg_batch_upload", "vg_batch_download",
           "vg_batch_run", "vg_batch_last_launch_count", "vg_batch_gradient", "vg_source_batch_create",
           "vg_source_batch_destroy", "vg_source_batch_upload", "vg_source_batch_download", "vg_source_batch_run",
           "vg_source_batch_gradient"]
NUM_XCFG, NUM_YCFG, NUM_SCHED = 5, 6, 2

NOALLOC_MAX_ROWS = 65536


def max_wave_speed_noalloc(model, planes_ptr, plane_stride, row_stride, nx, ny, params, out_ptr, stream=None):
    """vg_max_wave_speed_noalloc on caller-owned device memory (raw device pointers); asynchronous."""
    prm = np.zeros(MAX_PARAMS)
    prm[:len(params)] = params
    return _check(lib().vg_max_wave_speed_noalloc(model, ctypes.c_void_p(planes_ptr), plane_stride, row_stride, nx,
                                                  ny, prm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                  ctypes.c_void_p(out_ptr), stream))

_lib = None


def lib():
    """Load libvanguard_slic.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m vanguard_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, D = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        L.vg_create.argtypes = [ctypes.POINTER(GridDesc), ctypes.POINTER(vp)]
        L.vg_destroy.argtypes = [vp]
        L.vg_model_nvar.argtypes = [ctypes.c_int]
        L.vg_upload_primitive.argtypes = [vp, vp, ctypes.c_int, vp]
        L.vg_download_primitive.argtypes = [vp, vp, ctypes.c_int, vp]
        L.vg_run.argtypes = [vp, ctypes.POINTER(RunConfig), ctypes.POINTER(ctypes.c_int), D, vp]
        L.vg_solve.argtypes = [vp, vp, vp, ctypes.POINTER(RunConfig), ctypes.POINTER(ctypes.c_int), D, vp]
        L.vg_sweep.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, vp]
        L.vg_max_wave_speed.argtypes = [vp, D, vp]
        L.vg_max_wave_speed_cells.argtypes = [vp, D, vp]
        L.vg_state_device.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_long),
                                      ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_int)]
        L.vg_max_wave_speed_noalloc.argtypes = [ctypes.c_int, vp, ctypes.c_long, ctypes.c_long, ctypes.c_int,
                                                ctypes.c_int, D, vp, vp]
        L.vg_autotune.argtypes = [vp, ctypes.POINTER(RunConfig), ctypes.c_int, ctypes.POINTER(ctypes.c_float), vp]
        L.vg_set_launch_config.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.vg_set_schedule.argtypes = [vp, ctypes.c_int]
        L.vg_get_schedule.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.vg_get_launch_config.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_char_p)]
        L.vg_last_launch_count.argtypes = [vp]
        L.vg_last_launch_count.restype = ctypes.c_long
        I = ctypes.POINTER(ctypes.c_int)
        L.vg_batch_create.argtypes = [ctypes.c_int, I, D, D, D, ctypes.c_int, ctypes.POINTER(vp)]
        L.vg_batch_destroy.argtypes = [vp]
        L.vg_batch_total_cells.argtypes = [vp]
        L.vg_batch_total_cells.restype = ctypes.c_long
        L.vg_batch_upload.argtypes = [vp, vp, ctypes.c_int, vp]
        L.vg_batch_download.argtypes = [vp, vp, ctypes.c_int, vp]
        L.vg_batch_run.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int, D, vp]
        L.vg_batch_last_launch_count.argtypes = [vp]
        L.vg_batch_last_launch_count.restype = ctypes.c_long
        Lp = ctypes.POINTER(ctypes.c_long)
        L.vg_batch_gradient.argtypes = [vp, vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                        ctypes.c_int, D, vp, vp, ctypes.c_int, Lp, Lp, vp]
        L.vg_source_batch_create.argtypes = [ctypes.c_int, D, ctypes.c_int, ctypes.POINTER(vp)]
        L.vg_source_batch_destroy.argtypes = [vp]
        L.vg_source_batch_upload.argtypes = [vp, vp, vp, ctypes.c_int, vp]
        L.vg_source_batch_download.argtypes = [vp, vp, ctypes.c_int, vp]
        L.vg_source_batch_run.argtypes = [vp, ctypes.c_double, ctypes.c_int, vp]
        L.vg_source_batch_gradient.argtypes = [vp, vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_int,
                                               Lp, Lp, vp]
        L.vg_last_error_string.restype = ctypes.c_char_p
        L.vg_status_string.restype = ctypes.c_char_p
        L.vg_status_string.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _check(st, allow=()):
    if st != VG_OK and st not in allow:
        raise VgError(st, lib().vg_last_error_string().decode())
    return st


class Solver:
    """One grid on one GPU: a thin handle over vg_create / vg_destroy."""

    def __init__(self, model, nx, ny=1, params=(), precision=FP64, boundary=TRANSMISSIVE, device=0):
        d = GridDesc()
        d.model, d.nx, d.ny, d.precision, d.boundary, d.device = model, nx, ny, precision, boundary, device
        for i, v in enumerate(params):
            d.params[i] = float(v)
        self.model, self.nx, self.ny = model, nx, ny
        self._h = ctypes.c_void_p()
        _check(lib().vg_create(ctypes.byref(d), ctypes.byref(self._h)))

    def close(self):
        if self._h:
            lib().vg_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _shape(self):
        return (NVAR[self.model], self.ny, self.nx) if self.ny > 1 else (NVAR[self.model], self.nx)

    def upload(self, planes, stream=None):
        """planes: host float64 array (nvar, ny, nx) / (nvar, n), or a torch CUDA tensor of that shape."""
        if hasattr(planes, "data_ptr"):
            t = planes.contiguous()
            return _check(lib().vg_upload_primitive(self._h, ctypes.c_void_p(t.data_ptr()), 1, stream))
        a = np.ascontiguousarray(planes, dtype=np.float64)
        if a.shape != self._shape():
            raise ValueError(f"expected planes of shape {self._shape()}, got {a.shape}")
        return _check(lib().vg_upload_primitive(self._h, a.ctypes.data_as(ctypes.c_void_p), 0, stream))

    def download(self, out=None, stream=None):
        if out is not None and hasattr(out, "data_ptr"):
            _check(lib().vg_download_primitive(self._h, ctypes.c_void_p(out.data_ptr()), 1, stream))
            return out
        a = np.empty(self._shape(), dtype=np.float64) if out is None else out
        _check(lib().vg_download_primitive(self._h, a.ctypes.data_as(ctypes.c_void_p), 0, stream))
        return a

    def run(self, dx, cfl, t_end=0.0, steps=0, bias=0.0, limiter=SUPERBEE, subcycles=0, stream=None,
            allow_nan=False, order=2, stiff=False, reinit=0):
        """The solve() time loop on the device; order=1 runs FirstOrderSolver's FORCE loop instead; stiff=True
        (HPR) relaxes the source over dt/2 before and after the sweeps instead of the RK4 forcing sub-cycles."""
        c = RunConfig(dx, cfl, t_end, steps, bias, limiter, subcycles, order, 1 if stiff else 0, reinit)
        it = ctypes.c_int()
        t = ctypes.c_double()
        _check(lib().vg_run(self._h, ctypes.byref(c), ctypes.byref(it), ctypes.byref(t), stream),
               allow=(VG_ENAN,) if allow_nan else ())
        return t.value, it.value

    def solve(self, planes_in, dx, cfl, t_end=0.0, steps=0, bias=0.0, limiter=SUPERBEE, subcycles=0,
              out=None, stream=None):
        """Host-buffer round trip through vg_solve (upload, run, download)."""
        a = np.ascontiguousarray(planes_in, dtype=np.float64)
        o = np.empty_like(a) if out is None else out
        c = RunConfig(dx, cfl, t_end, steps, bias, limiter, subcycles, 2)
        it = ctypes.c_int()
        t = ctypes.c_double()
        _check(lib().vg_solve(self._h, a.ctypes.data_as(ctypes.c_void_p), o.ctypes.data_as(ctypes.c_void_p),
                              ctypes.byref(c), ctypes.byref(it), ctypes.byref(t), stream))
        return o, t.value, it.value

    def sweep(self, axis, dx, dt, bias=0.0, limiter=SUPERBEE, stream=None):
        return _check(lib().vg_sweep(self._h, axis, dx, dt, bias, limiter, stream))

    def max_wave_speed(self, stream=None, corners=True):
        """The CFL maximum of the padded grid (vg_max_wave_speed); corners=False: over exactly the uploaded cells,
        without the default-state corner ghosts of a 2D grid (vg_max_wave_speed_cells)."""
        v = ctypes.c_double()
        f = lib().vg_max_wave_speed if corners else lib().vg_max_wave_speed_cells
        _check(f(self._h, ctypes.byref(v), stream))
        return v.value

    def state_device(self):
        p = ctypes.c_void_p()
        ps, rs, n = ctypes.c_long(), ctypes.c_long(), ctypes.c_int()
        _check(lib().vg_state_device(self._h, ctypes.byref(p), ctypes.byref(ps), ctypes.byref(rs), ctypes.byref(n)))
        return p.value, ps.value, rs.value, n.value

    def last_launch_count(self):
        return lib().vg_last_launch_count(self._h)

    def autotune(self, dx, cfl, bias=0.0, limiter=SUPERBEE, reps=3, measure=True, stream=None):
        """Pick the fastest sweep tile shapes on the uploaded state; returns (x_times, y_times) in ms."""
        c = RunConfig(dx, cfl, 0.0, 1, bias, limiter, 0, 2)
        times = (ctypes.c_float * (NUM_XCFG + NUM_YCFG + NUM_SCHED))() if measure else None
        _check(lib().vg_autotune(self._h, ctypes.byref(c), reps, times, stream))
        if times is None:
            return None
        self.schedule_times = list(times[NUM_XCFG + NUM_YCFG:])  # step tail: CFL maximum fused, separate
        return list(times[:NUM_XCFG]), list(times[NUM_XCFG:NUM_XCFG + NUM_YCFG])

    def schedule(self):
        """0: the next step's CFL maximum folded into the last X sweep; 1: a separate reduction pass."""
        v = ctypes.c_int()
        _check(lib().vg_get_schedule(self._h, ctypes.byref(v)))
        return v.value

    def set_schedule(self, cfl_separate):
        return _check(lib().vg_set_schedule(self._h, int(cfl_separate)))

    def launch_config(self):
        x, y = ctypes.c_int(), ctypes.c_int()
        xn, yn = ctypes.c_char_p(), ctypes.c_char_p()
        _check(lib().vg_get_launch_config(self._h, ctypes.byref(x), ctypes.byref(y), ctypes.byref(xn), ctypes.byref(yn)))
        return x.value, y.value, xn.value.decode(), yn.value.decode()

    def set_launch_config(self, xcfg, ycfg):
        return _check(lib().vg_set_launch_config(self._h, xcfg, ycfg))


class Batch:
    """Ragged batch of independent 1D Euler problems (vg_batch_*): one persistent kernel per step, the whole
    time loop replayed from one CUDA graph, per-instance dt on the device."""

    def __init__(self, ncell, dx, gamma, p_inf=None, device=0):
        self.ncell = np.ascontiguousarray(ncell, dtype=np.int32)
        self.dx = np.ascontiguousarray(dx, dtype=np.float64)
        self.gamma = np.ascontiguousarray(gamma, dtype=np.float64)
        self.p_inf = None if p_inf is None else np.ascontiguousarray(p_inf, dtype=np.float64)
        self.ninst = len(self.ncell)
        self.total = int(self.ncell.sum())
        self._h = ctypes.c_void_p()
        D = ctypes.POINTER(ctypes.c_double)
        _check(lib().vg_batch_create(self.ninst, self.ncell.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                     self.dx.ctypes.data_as(D), self.gamma.ctypes.data_as(D),
                                     None if self.p_inf is None else self.p_inf.ctypes.data_as(D), device,
                                     ctypes.byref(self._h)))

    def close(self):
        if self._h:
            lib().vg_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload(self, planes, stream=None):
        """planes: (6, total) float64 Euler primitives of all instances concatenated."""
        if hasattr(planes, "data_ptr"):
            return _check(lib().vg_batch_upload(self._h, ctypes.c_void_p(planes.data_ptr()), 1, stream))
        a = np.ascontiguousarray(planes, dtype=np.float64)
        return _check(lib().vg_batch_upload(self._h, a.ctypes.data_as(ctypes.c_void_p), 0, stream))

    def download(self, out=None, stream=None):
        a = np.empty((6, self.total)) if out is None else out
        if a.shape != (6, self.total) or a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float64 array of shape (6, {self.total})")
        _check(lib().vg_batch_download(self._h, a.ctypes.data_as(ctypes.c_void_p), 0, stream))
        return a

    def run(self, cfl, steps, bias=0.0, limiter=SUPERBEE, stream=None):
        dts = np.empty(self.ninst)
        _check(lib().vg_batch_run(self._h, cfl, steps, bias, limiter,
                                  dts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), stream))
        return dts

    def last_launch_count(self):
        return lib().vg_batch_last_launch_count(self._h)

    def gradient(self, target_rho, cfl, steps, bias=0.0, limiter=SUPERBEE, checkpoints=None, out=None, stream=None):
        """Discrete adjoint of run(cfl, steps) from the current state for L = sum (rho(T) - target_rho)^2.
        Returns (L, dL/dW0 as (6, total) planes, dL/dgamma (ninst,), forward steps, reversed steps).
        checkpoints defaults to every state (no recomputation).  With torch CUDA tensors for target_rho and
        out = (grad_planes (6, total), grad_gamma (ninst,)) everything stays on the device; with numpy arrays
        (pinned ones for full copy speed) out receives the host result."""
        fw, aw = ctypes.c_long(), ctypes.c_long()
        L = ctypes.c_double()
        ck = steps if checkpoints is None else checkpoints
        if hasattr(target_rho, "data_ptr"):
            g, gg = out
            for x, shape in ((target_rho, (self.total,)), (g, (6, self.total)), (gg, (self.ninst,))):
                if tuple(x.shape) != shape or not x.is_contiguous():
                    raise ValueError(f"expected a contiguous device tensor of shape {shape}")
            _check(lib().vg_batch_gradient(self._h, ctypes.c_void_p(target_rho.data_ptr()), cfl, steps, bias, limiter,
                                           ck, ctypes.byref(L), ctypes.c_void_p(g.data_ptr()),
                                           ctypes.c_void_p(gg.data_ptr()), 1, ctypes.byref(fw), ctypes.byref(aw),
                                           stream))
            return L.value, g, gg, fw.value, aw.value
        t = np.ascontiguousarray(target_rho, dtype=np.float64)
        if t.shape != (self.total,):
            raise ValueError(f"target_rho must have shape ({self.total},)")
        g, gg = (np.empty((6, self.total)), np.empty(self.ninst)) if out is None else out
        for x, shape in ((g, (6, self.total)), (gg, (self.ninst,))):
            if x.shape != shape or x.dtype != np.float64 or not x.flags.c_contiguous:
                raise ValueError(f"expected a C-contiguous float64 array of shape {shape}")
        _check(lib().vg_batch_gradient(self._h, t.ctypes.data_as(ctypes.c_void_p), cfl, steps, bias, limiter, ck,
                                       ctypes.byref(L), g.ctypes.data_as(ctypes.c_void_p),
                                       gg.ctypes.data_as(ctypes.c_void_p), 0, ctypes.byref(fw), ctypes.byref(aw),
                                       stream))
        return L.value, g, gg, fw.value, aw.value


class SourceBatch:
    """Homogeneous HPR relaxation cells (vg_source_batch_*): each cell advanced by the reference's source step on a
    uniform field, and the discrete adjoint of that evolution."""

    def __init__(self, ncell, params, device=0):
        self.n = int(ncell)
        prm = np.zeros(MAX_PARAMS)
        prm[:len(params)] = params
        self._h = ctypes.c_void_p()
        _check(lib().vg_source_batch_create(self.n, prm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), device,
                                            ctypes.byref(self._h)))

    def close(self):
        if self._h:
            lib().vg_source_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def _host(a, shape):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != shape:
            raise ValueError(f"expected shape {shape}, got {a.shape}")
        return a

    def upload(self, planes, tau=None, stream=None):
        """planes: (17, ncell) HPR primitives; tau: (2, ncell) relaxation times or None (the params')."""
        if hasattr(planes, "data_ptr"):
            tp = ctypes.c_void_p(tau.data_ptr()) if tau is not None else None
            return _check(lib().vg_source_batch_upload(self._h, ctypes.c_void_p(planes.data_ptr()), tp, 1, stream))
        p = self._host(planes, (17, self.n))
        t = None if tau is None else self._host(tau, (2, self.n))
        return _check(lib().vg_source_batch_upload(self._h, p.ctypes.data_as(ctypes.c_void_p),
                                                   None if t is None else t.ctypes.data_as(ctypes.c_void_p), 0, stream))

    def download(self, stream=None):
        a = np.empty((17, self.n))
        _check(lib().vg_source_batch_download(self._h, a.ctypes.data_as(ctypes.c_void_p), 0, stream))
        return a

    def run(self, h, steps, stream=None):
        return _check(lib().vg_source_batch_run(self._h, h, steps, stream))

    def gradient(self, cotangent, h, steps, checkpoints=None, out=None, stream=None):
        """Adjoint of run(h, steps) from the current state: returns (dL/dW0 (17, n), dL/dtau (2, n), forward steps,
        reversed steps) for the cotangent dL/dW(T) (17, n).  With a torch CUDA tensor for the cotangent and out =
        (grad_planes (17, n), grad_tau (2, n)) CUDA tensors everything stays on the device."""
        fw, aw = ctypes.c_long(), ctypes.c_long()
        ck = steps if checkpoints is None else checkpoints
        if hasattr(cotangent, "data_ptr"):
            g, gt = out
            _check(lib().vg_source_batch_gradient(self._h, ctypes.c_void_p(cotangent.data_ptr()), h, steps, ck,
                                                  ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(gt.data_ptr()), 1,
                                                  ctypes.byref(fw), ctypes.byref(aw), stream))
            return g, gt, fw.value, aw.value
        lam = self._host(cotangent, (17, self.n))
        g, gt = np.empty((17, self.n)), np.empty((2, self.n))
        _check(lib().vg_source_batch_gradient(self._h, lam.ctypes.data_as(ctypes.c_void_p), h, steps, ck,
                                              g.ctypes.data_as(ctypes.c_void_p), gt.ctypes.data_as(ctypes.c_void_p), 0,
                                              ctypes.byref(fw), ctypes.byref(aw), stream))
        return g, gt, fw.value, aw.value
