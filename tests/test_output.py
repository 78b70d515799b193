"""The .dat solution writers (vanguard_b200.output) against the reference scenarios' own writers
(EulerTests / MHDTests / HPRTests::outputSolution{,2D}, compiled into oracle/_ref), file by file and byte for byte,
on solutions of the oracle; and the number rendering against libc's printf %g where the reference is absent."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
from vanguard_b200 import output
from vanguard_b200 import workloads as wl

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference not built (oracle/_ref)")


def _same_files(ours, ref_dir):
    for path in ours:
        with open(path) as f, open(os.path.join(ref_dir, os.path.basename(path))) as g:
            assert f.read() == g.read(), os.path.basename(path)
    assert sorted(os.listdir(ref_dir)) == sorted(os.path.basename(p) for p in ours)


def _dirs(tmp_path):
    a, b = tmp_path / "ours", tmp_path / "ref"
    a.mkdir()
    b.mkdir()
    return str(a), str(b)


def test_number_rendering_is_printf_g():
    libc = ctypes.CDLL(None)
    buf = ctypes.create_string_buffer(64)
    rng = np.random.default_rng(0)
    values = np.concatenate([rng.standard_normal(500) * 10.0 ** rng.integers(-12, 12, 500),
                             [0.0, -0.0, 1.0, 0.1, 1e-5, 123456.0, 1234567.0, 0.000123456, 2.5e-300, 1e300]])
    for v in values:
        libc.snprintf(buf, 64, b"%g", ctypes.c_double(float(v)))
        assert output._g(v) == buf.value.decode(), v


@needs_ref
def test_euler_writer_matches_reference(tmp_path, oracle_lib):
    W = wl.sod_1d(120)
    O.run(O.EULER, W, 1 / 120, 0.9, t_end=0.1, limiter=O.MINBEE, params=wl.euler_params(1.4))
    ours, ref = _dirs(tmp_path)
    files = output.write_euler(W, ours)
    O.ref_write(O.EULER, W, ref)
    _same_files(files, ref)


@needs_ref
@pytest.mark.parametrize("ny", [1, 12])
def test_mhd_writer_matches_reference(tmp_path, oracle_lib, ny):
    W = wl.brio_wu_1d(100) if ny == 1 else wl.mhd_vortex_2d(12, 12, seed=2)
    O.run(O.MHD, W, 1 / W.shape[-1], 0.8, steps=5, limiter=0, params=wl.mhd_params(5 / 3))
    ours, ref = _dirs(tmp_path)
    files = output.write_mhd(W, ours)
    O.ref_write(O.MHD, W, ref)
    _same_files(files, ref)


@needs_ref
@pytest.mark.parametrize("case", ["heat1d", "shock_mg1d", "smooth2d"])
def test_hpr_writer_matches_reference(tmp_path, oracle_lib, case):
    if case == "heat1d":
        prm, W = wl.hpr_params(tau1=1e-1, tau2=1e-1), wl.hpr_heat_conduction_1d(80)
    elif case == "shock_mg1d":
        prm = wl.hpr_shock_mg_params(thermal=True, tau1=0.1)
        W = wl.hpr_shock_riemann(60, 1, prm)
    else:
        prm, W = wl.hpr_params(), wl.hpr_smooth_2d(12, 10, seed=1)
    O.run(O.HPR, W, 1 / W.shape[-1], 0.8, steps=4, limiter=0, params=prm, subcycles=1)
    ours, ref = _dirs(tmp_path)
    files = output.write_hpr(W, prm, ours)
    O.ref_write(O.HPR, W, ref, params=prm)
    _same_files(files, ref)


@pytest.mark.parametrize("name", ["gas", "shock_mg", "gr"])
def test_hpr_temperature_matches_oracle(oracle_lib, name):
    prm = {"gas": wl.hpr_params(p_inf=0.2), "shock_mg": wl.hpr_shock_mg_params(), "gr": wl.hpr_zhang_params()}[name]
    rng = np.random.default_rng(3)
    planes = np.zeros((17, 64))
    planes[0] = prm[3] * rng.uniform(0.9, 1.1, 64)
    planes[1] = rng.uniform(0.1, 2.0, 64)
    T = output.hpr_temperature(planes, prm)
    ref = O.hpr_eos(prm, planes[0], planes[1], np.zeros(64))[:, 8]
    assert np.allclose(T, ref, rtol=1e-12, atol=0.0)
