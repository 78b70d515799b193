"""Pin the CPU oracle (our C restatement, oracle/slic_oracle.c) before trusting it as the checker.

* Against the committed golden fixtures, produced by the reference's own unmodified code
  (tests/golden/make_golden.py): bit-for-bit.
* Against the live reference (oracle/_ref/libvgref.so, where it was built) on further seeded cases that
  exercise every limiter, a non-zero bias, both boundary kinds and 1D/2D: bit-for-bit.
"""
import glob
import math
import os

import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden(path, oracle_lib):
    z = np.load(path)
    model = int(z["model"])
    w = z["w0"].copy()
    kw = {k: (z[k].item() if z[k].ndim == 0 else z[k]) for k in z.files if k not in ("model", "w0", "out")}
    dx, cfl = kw.pop("dx"), kw.pop("cfl")
    if model in (O.EULER_REDUCED, O.EULER_MULTIPHYSICS, O.MHD_REDUCED, O.MHD_INTERMEDIATE, O.HPR_REDUCED,
                 O.HPR_INTERMEDIATE, O.HPR_MULTIPHYSICS, O.MHD_MULTIPHYSICS):
        O.run_two_material(model, w, dx, cfl, **kw)
    else:
        O.run(model, w, dx, cfl, **kw)
    assert np.array_equal(w, z["out"]), f"max diff {np.abs(w - z['out']).max():.3e}"


def test_golden_set_complete():
    names = {os.path.basename(p)[:-4] for p in GOLDEN}
    assert "euler1d_sod1000_minbee_t025" in names
    assert any(n.startswith("mhd2d") for n in names)


def test_slope_floor_is_1e5():
    # SlopeLimiters::computeSlopeVector floors |delta| < pow(10, -5) (Solvers/slopelimiters.cpp:232-239);
    # the device receives the host's pow(10.0, -5.0)
    assert math.pow(10.0, -5.0) == 1e-5


@pytest.mark.parametrize("lim", [0, 1, 2])
def test_limiter_values(oracle_lib, lim):
    L = O.lib()
    # hand-derived points of Solvers/slopelimiters.cpp:7-74 at bias 0: xi_R = 2 / (1 + r)
    expect = {
        0: {-1.0: 0.0, 0.25: 0.5, 0.75: 1.0, 1.5: min(1.5, 2 / 2.5, 2.0), 3.0: 0.5},
        1: {-1.0: 0.0, 0.25: min(0.5 / 1.25, 2 / 1.25), 3.0: min(6 / 4, 0.5)},
        2: {-1.0: 0.0, 0.25: 0.25, 0.75: 0.75, 3.0: min(1.0, 0.5)},
    }[lim]
    for r, v in expect.items():
        assert L.vo_slope_limiter(r, 0.0, lim) == v


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference not built (oracle/_ref)")


@needs_ref
@pytest.mark.parametrize("lim,bias", [(0, 0.0), (1, 0.3), (2, -0.5), (7, 0.0)])
def test_oracle_vs_reference_euler1d(lim, bias):
    rng = np.random.default_rng(100 + lim)
    n = 150
    W = wl.sod_1d(n, left=(rng.uniform(0.2, 2), rng.uniform(-1, 1), rng.uniform(0.2, 3)),
                  right=(rng.uniform(0.2, 2), rng.uniform(-1, 1), rng.uniform(0.2, 3)))
    a, b = W.copy(), W.copy()
    prm = wl.euler_params(1.4)
    O.run(O.EULER, a, 1 / n, 0.8, steps=60, bias=bias, limiter=lim, params=prm)
    O.ref_run(O.EULER, b, 1 / n, 0.8, steps=60, bias=bias, limiter=lim, params=prm)
    assert np.array_equal(a, b)


@needs_ref
def test_oracle_vs_reference_euler1d_stiffened_gas():
    n = 120
    W = wl.sod_1d(n, left=(1.0, 0.0, 5.0), right=(0.5, 0.0, 0.5))
    a, b = W.copy(), W.copy()
    prm = wl.euler_params(4.4, 0.6)
    O.run(O.EULER, a, 1 / n, 0.8, steps=50, limiter=0, params=prm)
    O.ref_run(O.EULER, b, 1 / n, 0.8, steps=50, limiter=0, params=prm)
    assert np.array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("bc", [0, 1])
def test_oracle_vs_reference_euler2d(bc):
    W = wl.euler_quadrants_2d(36, 28, seed=31 + bc)
    a, b = W.copy(), W.copy()
    prm = wl.euler_params(1.4)
    O.run(O.EULER, a, 1 / 36, 0.8, steps=15, bias=0.2, limiter=1, params=prm, bc=bc)
    O.ref_run(O.EULER, b, 1 / 36, 0.8, steps=15, bias=0.2, limiter=1, params=prm, bc=bc)
    assert np.array_equal(a, b)


@needs_ref
def test_oracle_vs_reference_mhd2d_full_components():
    W = wl.mhd_vortex_2d(24, 20, seed=5)
    W[3] = 0.05
    W[7] = 0.2 * np.cos(np.linspace(0, 3, 24))[None, :]
    a, b = W.copy(), W.copy()
    prm = wl.mhd_params(5 / 3)
    O.run(O.MHD, a, 1 / 24, 0.8, steps=12, limiter=2, params=prm, bc=1)
    O.ref_run(O.MHD, b, 1 / 24, 0.8, steps=12, limiter=2, params=prm, bc=1)
    assert np.array_equal(a, b)


@needs_ref
def test_reference_solve_matches_step_loop():
    """The harness's per-step loop reproduces the reference's own solve() (Solvers/secondordersolver.cpp:288)."""
    W = wl.sod_1d(200)
    a, b = W.copy(), W.copy()
    prm = wl.euler_params(1.4)
    O.ref_run(O.EULER, a, 1 / 200, 0.9, t_end=0.1, steps=0, limiter=2, params=prm)      # solve() itself
    O.ref_run(O.EULER, b, 1 / 200, 0.9, t_end=0.1, steps=100000, limiter=2, params=prm)  # step loop
    assert np.array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("thermal", [True, False])
def test_oracle_vs_reference_hpr_cell(thermal):
    """Conserved vector, x/y fluxes, relaxation source and both acoustic-tensor speeds of random states."""
    rng = np.random.default_rng(7 if thermal else 8)
    for trial in range(6):
        prm = wl.hpr_params(tau1=10 ** rng.uniform(-3, -1), tau2=10 ** rng.uniform(-3, -1), thermal=thermal,
                            p_inf=0.25 * trial)
        w = np.zeros(17)
        w[0], w[1] = rng.uniform(0.5, 2.0), rng.uniform(0.5, 2.0)
        w[2:11] = (np.eye(3) + 0.1 * rng.standard_normal((3, 3))).ravel()
        w[11:14] = 0.3 * rng.standard_normal(3)
        w[14:17] = 0.2 * rng.standard_normal(3)
        for a, b in zip(O.hpr_cell(w, prm), O.hpr_cell(w, prm, reference=True)):
            assert np.array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("sub,bc", [(0, 1), (1, 0)])
def test_oracle_vs_reference_hpr2d(sub, bc):
    W = wl.hpr_smooth_2d(14, 12, seed=10 + sub)
    a, b = W.copy(), W.copy()
    prm = wl.hpr_params(tau1=2e-2, tau2=3e-2)
    O.run(O.HPR, a, 1 / 14, 0.8, steps=3, limiter=1, params=prm, bc=bc, subcycles=sub)
    O.ref_run(O.HPR, b, 1 / 14, 0.8, steps=3, limiter=1, params=prm, bc=bc, subcycles=sub)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("bc", [0, 1])
def test_oracle_vs_reference_mhd_glm_subcycles(bc):
    """MHD with GLM damping sub-cycles (MHDForcingSolver's RK4 around the sweeps), 1D and 2D, bit for bit."""
    if not O.ref_available():
        pytest.skip("compiled reference not built")
    W = wl.mhd_vortex_2d(20, 16, seed=4)
    a, b = W.copy(), W.copy()
    O.run(O.MHD, a, 1 / 20, 0.8, steps=6, limiter=0, params=wl.mhd_params(5 / 3), bc=bc, subcycles=2)
    O.ref_run(O.MHD, b, 1 / 20, 0.8, steps=6, limiter=0, params=wl.mhd_params(5 / 3), bc=bc, subcycles=2)
    assert np.array_equal(a, b)
    assert np.abs(a[8] - W[8]).max() > 1e-4  # psi is damped and transported, not left alone
    W1 = wl.brio_wu_1d(60)
    W1[8] = 0.01 * np.sin(np.arange(60))
    a, b = W1.copy(), W1.copy()
    O.run(O.MHD, a, 1 / 60, 0.8, steps=8, limiter=1, params=wl.mhd_params(2.0), bc=bc, subcycles=3)
    O.ref_run(O.MHD, b, 1 / 60, 0.8, steps=8, limiter=1, params=wl.mhd_params(2.0), bc=bc, subcycles=3)
    assert np.array_equal(a, b)


def _first_order_cases():
    return [
        ("euler1d", O.EULER, wl.sod_1d(100), wl.euler_params(1.4), 1 / 100, 0),
        ("euler2d", O.EULER, wl.euler_quadrants_2d(24, 20, seed=3), wl.euler_params(1.4), 1 / 24, 0),
        ("euler2d_periodic", O.EULER, wl.euler_quadrants_2d(24, 20, seed=3), wl.euler_params(1.4), 1 / 24, 1),
        ("mhd2d_periodic", O.MHD, wl.mhd_vortex_2d(20, 16, seed=2), wl.mhd_params(5 / 3, c_h=1.3), 1 / 20, 1),
        ("mhd1d", O.MHD, wl.brio_wu_1d(80), wl.mhd_params(2.0, c_h=0.7), 1 / 80, 0),
        ("hpr2d", O.HPR, wl.hpr_smooth_2d(16, 14, seed=5), wl.hpr_params(), 1 / 16, 0),
        ("hpr1d_periodic", O.HPR, wl.hpr_heat_conduction_1d(40), wl.hpr_params(), 1 / 40, 1),
    ]


@pytest.mark.parametrize("case", _first_order_cases(), ids=lambda c: c[0])
def test_oracle_vs_reference_first_order(case):
    """FirstOrderSolver / MHDFirstOrderSolver / HPRFirstOrderSolver loops, bit for bit (the MHD c_h is not reset)."""
    if not O.ref_available():
        pytest.skip("compiled reference not built")
    _, model, W, prm, dx, bc = case
    a, b = W.copy(), W.copy()
    ta = O.run_first_order(model, a, dx, 0.8, steps=7, params=prm, bc=bc)
    tb = O.ref_run_first_order(model, b, dx, 0.8, steps=7, params=prm, bc=bc)
    assert ta == tb
    assert np.array_equal(a, b)


@pytest.mark.skipif(not O.ref_available(), reason="the compiled reference (oracle/_ref) was not built")
def test_reference_batch_harness_matches_per_problem_solves(oracle_lib):
    """The reference's ragged-batch baseline (one solve loop per problem, problems in parallel) equals the oracle's
    per-problem run bit for bit: the parallel schedule does not change any problem's arithmetic."""
    ncell, dx, gamma, theta, W = wl.ragged_riemann_batch(ninst=23, seed=8, nmin=3, nmax=300)
    out = W.copy()
    O.ref_batch_run(out, ncell, dx, gamma, 0.8, 25, bias=0.2, limiter=O.MINBEE, threads=4)
    off = 0
    for k, n in enumerate(ncell):
        ref = W[:, off:off + n].copy()
        O.run(O.EULER, ref, dx[k], 0.8, steps=25, bias=0.2, limiter=O.MINBEE, params=wl.euler_params(gamma[k]))
        assert np.array_equal(out[:, off:off + n], ref), k
        off += n
