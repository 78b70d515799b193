"""The MHD intermediate two-material model on the device (VG_MODEL_MHD_INTERMEDIATE): the exact FP64 form against the
golden fixtures made by the reference (its own MHDSecondOrderSolver::solve in 1D; its per-step functions over mirror
ghosts in 2D, where its solve2D pads the grid with a defective insertBoundaryCells2D) and against the oracle (pinned in
test_mhd_intermediate.py), bit for bit, with the GLM damping sub-cycles and the volume-fraction reinitialisation (both
densities and both pressures relaxed); the first-order loop; argument checks."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "mhdintermediate*.npz")))
PRM = wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0)


def _bitwise(a, b):
    if not np.array_equal(a, b):
        d = np.abs(a - b)
        raise AssertionError(f"max |diff| {d.max():.3e}; {np.count_nonzero(d)} values differ")


def _device(gpu, W, prm, dx, boundary=None, **run):
    nx = W.shape[-1]
    ny = 1 if W.ndim == 2 else W.shape[1]
    kw = {} if boundary is None else {"boundary": boundary}
    with gpu.Solver(gpu.MHD_INTERMEDIATE, nx, ny, prm, **kw) as s:
        s.upload(W)
        t, n = s.run(dx, 0.8, **run)
        return s.download(), t, n


def _layout(ny, nx=None):
    if ny == 1:
        return wl.mhd_intermediate_from_reduced(wl.mhd_reduced_dumbser_1d(nx or 130))
    return wl.mhd_intermediate_from_reduced(wl.mhd_reduced_dumbser_2d(nx or 32, ny))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_mhd_intermediate_golden(gpu, path):
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
def test_mhd_intermediate_matches_oracle(gpu, oracle_lib, ny, limiter, reinit, subcycles):
    W = _layout(ny)
    steps = 15 if ny == 1 else 8
    dx = 1.0 / W.shape[-1]
    ref = W.copy()
    O.run_two_material(O.MHD_INTERMEDIATE, ref, dx, 0.8, steps=steps, limiter=limiter, params=PRM, reinit=reinit,
                       subcycles=subcycles)
    out, _, _ = _device(gpu, W, PRM, dx, steps=steps, limiter=limiter, reinit=reinit, subcycles=subcycles)
    _bitwise(out, ref)


def test_mhd_intermediate_time_driven_periodic(gpu, oracle_lib):
    W = _layout(1, 120)
    ref = W.copy()
    t_ref, n_ref = O.run_two_material(O.MHD_INTERMEDIATE, ref, 1 / 120, 0.8, t_end=0.03, bias=0.2, limiter=1,
                                      params=PRM, reinit=4, subcycles=1)
    out, t, n = _device(gpu, W, PRM, 1 / 120, t_end=0.03, bias=0.2, limiter=1, reinit=4, subcycles=1)
    assert (t, n) == (t_ref, n_ref)
    _bitwise(out, ref)
    W2 = _layout(22, 26)
    ref = W2.copy()
    O.run_two_material(O.MHD_INTERMEDIATE, ref, 1 / 26, 0.8, steps=6, limiter=2, params=PRM, subcycles=1,
                       bc=O.PERIODIC)
    out, _, _ = _device(gpu, W2, PRM, 1 / 26, boundary=gpu.PERIODIC, steps=6, limiter=2, subcycles=1)
    _bitwise(out, ref)


@pytest.mark.parametrize("ny", [1, 20])
def test_mhd_intermediate_first_order(gpu, oracle_lib, ny):
    prm = np.concatenate([PRM, [1.5]])
    W = _layout(ny, 90 if ny == 1 else 24)
    dx = 1.0 / W.shape[-1]
    ref = W.copy()
    O.run_first_order(O.MHD_INTERMEDIATE, ref, dx, 0.8, steps=12, params=prm)
    out, _, _ = _device(gpu, W, prm, dx, steps=12, order=1)
    _bitwise(out, ref)


def test_mhd_intermediate_argument_checks(gpu):
    with pytest.raises(gpu.VgError):
        gpu.Solver(gpu.MHD_INTERMEDIATE, 16, 1, PRM, precision=gpu.MIXED)
    with gpu.Solver(gpu.MHD_INTERMEDIATE, 32, 1, PRM) as s:
        s.upload(_layout(1, 32))
        with pytest.raises(gpu.VgError):
            s.run(1 / 32, 0.8, steps=3, order=1, reinit=2)
        t, n = s.run(1 / 32, 0.8, steps=3, subcycles=1, reinit=2)
        assert n == 3 and np.isfinite(s.download()).all()
