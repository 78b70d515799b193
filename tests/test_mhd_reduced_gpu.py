"""The MHD reduced two-material model on the device (VG_MODEL_MHD_REDUCED): the exact FP64 form against the golden
fixtures made by the reference's own MHDSecondOrderSolver::solve{,2D} and per-step functions (tests/golden/
make_golden.py) and against the oracle (pinned to the reference in test_mhd_reduced.py), bit for bit, with the GLM
damping sub-cycles and the volume-fraction reinitialisation; the first-order loop; argument checks."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "mhdreduced*.npz")))


def _bitwise(a, b):
    if not np.array_equal(a, b):
        d = np.abs(a - b)
        raise AssertionError(f"max |diff| {d.max():.3e}; {np.count_nonzero(d)} values differ")


def _device(gpu, W, prm, dx, boundary=None, **run):
    nx = W.shape[-1]
    ny = 1 if W.ndim == 2 else W.shape[1]
    kw = {} if boundary is None else {"boundary": boundary}
    with gpu.Solver(gpu.MHD_REDUCED, nx, ny, prm, **kw) as s:
        s.upload(W)
        t, n = s.run(dx, 0.8, **run)
        return s.download(), t, n


def _swirled(W, seed):
    """W with seeded smooth w, Bz and psi fields, so that every plane of the model carries data."""
    rng = np.random.default_rng(seed)
    x = np.linspace(0.0, 1.0, W.shape[-1])
    W = W.copy()
    for plane, amp in ((3, 0.1), (9, 0.2), (10, 0.05)):
        W[plane] = W[plane] + amp * np.sin(2 * np.pi * (x + rng.uniform()))
    return W


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_mhd_reduced_golden(gpu, path):
    z = np.load(path)
    steps = int(z["steps"])
    t_end = float(z["t_end"]) if "t_end" in z.files else 0.0
    out, _, n = _device(gpu, z["w0"], z["params"], float(z["dx"]), steps=steps, t_end=t_end,
                        limiter=int(z["limiter"]), reinit=int(z["reinit"]), subcycles=int(z["subcycles"]))
    if steps:
        assert n == steps
    _bitwise(out, z["out"])


@pytest.mark.parametrize("subcycles", [0, 2])
@pytest.mark.parametrize("reinit", [0, 3])
@pytest.mark.parametrize("limiter", [0, 2])
@pytest.mark.parametrize("ny", [1, 26])
def test_mhd_reduced_matches_oracle(gpu, oracle_lib, ny, limiter, reinit, subcycles):
    """8 steps in 2D: on this disc, which nearly reaches the grid's top and bottom, the reference scheme itself drives
    the pressure negative within 15 steps (the oracle and the reference agree on that), which the device reports as
    VG_ENAN."""
    prm = wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0)
    W = wl.mhd_reduced_dumbser_1d(130) if ny == 1 else wl.mhd_reduced_dumbser_2d(32, ny)
    steps = 15 if ny == 1 else 8
    dx = 1.0 / W.shape[-1]
    ref = W.copy()
    O.run_two_material(O.MHD_REDUCED, ref, dx, 0.8, steps=steps, limiter=limiter, params=prm, reinit=reinit,
                       subcycles=subcycles)
    assert min(ref[4].min(), ref[5].min(), ref[6].min()) > 0.0
    out, _, _ = _device(gpu, W, prm, dx, steps=steps, limiter=limiter, reinit=reinit, subcycles=subcycles)
    _bitwise(out, ref)


def test_mhd_reduced_every_plane_time_driven(gpu, oracle_lib):
    """Non-zero w, Bz and psi, a stiffened second material, a bias, and a run to t_end."""
    prm = wl.mhd_reduced_params(2.0, 0.0, 1.67, 0.3)
    W = _swirled(wl.mhd_reduced_dumbser_1d(140), seed=4)
    ref = W.copy()
    t_ref, n_ref = O.run_two_material(O.MHD_REDUCED, ref, 1 / 140, 0.8, t_end=0.04, bias=0.3, limiter=1, params=prm,
                                      reinit=4, subcycles=1)
    out, t, n = _device(gpu, W, prm, 1 / 140, t_end=0.04, bias=0.3, limiter=1, reinit=4, subcycles=1)
    assert (t, n) == (t_ref, n_ref)
    _bitwise(out, ref)


def test_mhd_reduced_periodic_2d(gpu, oracle_lib):
    prm = wl.mhd_reduced_params()
    W = wl.mhd_reduced_dumbser_2d(26, 22)
    W = np.stack([_swirled(W[:, r], seed=r) for r in range(W.shape[1])], axis=1)
    ref = W.copy()
    O.run_two_material(O.MHD_REDUCED, ref, 1 / 26, 0.8, steps=7, limiter=0, params=prm, subcycles=1, bc=O.PERIODIC)
    out, _, _ = _device(gpu, W, prm, 1 / 26, boundary=gpu.PERIODIC, steps=7, limiter=0, subcycles=1)
    _bitwise(out, ref)


@pytest.mark.parametrize("ny", [1, 20])
def test_mhd_reduced_first_order(gpu, oracle_lib, ny):
    """The first-order loop keeps c_h at params[4] (both materials)."""
    prm = np.concatenate([wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0), [1.5]])
    W = wl.mhd_reduced_dumbser_1d(90) if ny == 1 else wl.mhd_reduced_dumbser_2d(24, ny)
    dx = 1.0 / W.shape[-1]
    ref = W.copy()
    O.run_first_order(O.MHD_REDUCED, ref, dx, 0.8, steps=12, params=prm)
    out, _, _ = _device(gpu, W, prm, dx, steps=12, order=1)
    _bitwise(out, ref)


def test_mhd_reduced_argument_checks(gpu):
    prm = wl.mhd_reduced_params()
    with pytest.raises(gpu.VgError):
        gpu.Solver(gpu.MHD_REDUCED, 16, 1, prm, precision=gpu.MIXED)
    with gpu.Solver(gpu.MHD_REDUCED, 32, 1, prm) as s:
        s.upload(wl.mhd_reduced_dumbser_1d(32))
        with pytest.raises(gpu.VgError):
            s.run(1 / 32, 0.8, steps=3, order=1, reinit=2)
        with pytest.raises(gpu.VgError):
            s.run(1 / 32, 0.8, steps=3, reinit=-1)
        t, n = s.run(1 / 32, 0.8, steps=3, subcycles=1, reinit=2)
        assert n == 3 and np.isfinite(s.download()).all()
