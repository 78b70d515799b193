"""The HPR two-material models with solid materials on the device (VG_MODEL_HPR_REDUCED, _INTERMEDIATE,
_MULTIPHYSICS): the exact FP64 form against the oracle (pinned to the reference with ShockMieGruneisen solids in
test_hpr_two_material_solids.py) with the reference's own Barton (copper | copper) and Zhang (plastic aluminium |
copper) GodunovRomenski scenarios, ShockMieGruneisen pairs elastic, plastic and thermal, in 1D and 2D, with the
relaxation sub-cycles, the reinitialisation and the first-order loop; the CFL maximum wave speed.  The golden fixtures
with solid materials run in each model's own GPU test file.

The solid equations of state take pow (the GodunovRomenski density ratio, the ShockMieGruneisen cold curve) and so do
the relaxation source and the plastic rate, and CUDA's pow and glibc's may differ in the last place, so the runs are
compared plane by plane: the largest difference within 1e-10 of the plane's largest magnitude."""
import numpy as np
import pytest

import oracle as O
from vanguard_b200 import workloads as wl

from test_hpr_two_material_solids import (BARTON_V, ELASTIC1, ELASTIC2, MILD_PLASTIC2, MODEL_IDS, MODELS, PLASTIC2,
                                          THERMAL1, COLD2, ZHANG_V, solids)

pytestmark = pytest.mark.gpu
REL = 1e-10
MODEL_ENUM = {O.HPR_REDUCED: "HPR_REDUCED", O.HPR_INTERMEDIATE: "HPR_INTERMEDIATE",
              O.HPR_MULTIPHYSICS: "HPR_MULTIPHYSICS"}


def _matches(a, b, rel=REL):
    assert np.isfinite(a).all()
    d = np.abs(a - b).reshape(b.shape[0], -1).max(axis=1)
    scale = np.maximum(np.abs(b).reshape(b.shape[0], -1).max(axis=1), 1e-300)
    assert (d / scale).max() <= rel, f"max normwise diff {(d / scale).max():.3e} (plane {int(np.argmax(d / scale))})"


def _device(gpu, model, W, prm, dx, **run):
    ny = 1 if W.ndim == 2 else W.shape[1]
    with gpu.Solver(getattr(gpu, MODEL_ENUM[model]), W.shape[-1], ny, prm) as s:
        s.upload(W)
        t, n = s.run(dx, 0.8, **run)
        return s.download(), t, n


def _godunov_romenski(scenario):
    cu = wl.hpr_barton_params()
    if scenario == "barton":
        return cu, cu, wl.BARTON_F, ((0.0, 0.5, 1.0), (0.0, 0.0, 0.0))
    return wl.hpr_zhang_params(), cu, wl.ZHANG_F, ((2.0, 0.0, 0.1), (0.0, -0.03, -0.01))


@pytest.mark.parametrize("kw", [dict(steps=20, limiter=O.MINBEE, subcycles=1),
                                dict(steps=20, limiter=O.SUPERBEE),
                                dict(steps=16, limiter=O.VANLEER, subcycles=2, reinit=3, bias=0.2)],
                         ids=["minbee_sub1", "superbee", "vanleer_sub2_reinit3"])
@pytest.mark.parametrize("scenario", ["barton", "zhang"])
@pytest.mark.parametrize("model", MODELS, ids=MODEL_IDS)
def test_godunov_romenski_matches_oracle(gpu, oracle_lib, model, scenario, kw):
    m1, m2, F, v = _godunov_romenski(scenario)
    prm = wl.hpr_two_params(m1, m2)
    W = solids(model, m1, m2, F, v, 60)
    ref = W.copy()
    t_ref, n_ref = O.run_two_material(model, ref, 1 / 60, 0.8, params=prm, **kw)
    assert np.isfinite(ref).all()
    out, t, n = _device(gpu, model, W, prm, 1 / 60, **kw)
    assert n == n_ref
    assert abs(t - t_ref) <= 1e-12 * t_ref
    _matches(out, ref)


CASES = {
    "elastic_sub1_reinit3": (ELASTIC1, ELASTIC2, wl.ZHANG_F, ZHANG_V, 0.0,
                             dict(steps=20, limiter=O.MINBEE, subcycles=1, reinit=3)),
    "plastic_bias_sub2_reinit3": (ELASTIC1, PLASTIC2, wl.ZHANG_F, ZHANG_V, 0.0,
                                  dict(steps=20, limiter=O.MINBEE, subcycles=2, reinit=3, bias=0.2)),
    "plastic_superbee_sub1": (ELASTIC1, PLASTIC2, wl.BARTON_F, BARTON_V, 0.0,
                              dict(steps=20, limiter=O.SUPERBEE, subcycles=1)),
    "thermal_vanleer_sub1": (THERMAL1, COLD2, wl.BARTON_F, BARTON_V, 0.05,
                             dict(steps=12, limiter=O.VANLEER, subcycles=1)),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("model", MODELS, ids=MODEL_IDS)
def test_shock_mie_gruneisen_matches_oracle(gpu, oracle_lib, model, case):
    m1, m2, F, v, heat, kw = CASES[case]
    prm = wl.hpr_two_params(m1, m2)
    W = solids(model, m1, m2, F, v, 60, heat=heat)
    ref = W.copy()
    O.run_two_material(model, ref, 1 / 60, 0.8, params=prm, **kw)
    out, _, n = _device(gpu, model, W, prm, 1 / 60, **kw)
    assert n == kw["steps"]
    _matches(out, ref)


@pytest.mark.parametrize("m2,kw", [
    (ELASTIC2, dict(steps=6, limiter=O.MINBEE, subcycles=1, reinit=2, bias=-0.2)),
    (MILD_PLASTIC2, dict(steps=6, limiter=O.SUPERBEE, subcycles=2)),
], ids=["elastic_sub1_reinit2", "plastic_sub2"])
@pytest.mark.parametrize("model", MODELS[:2], ids=MODEL_IDS[:2])
def test_solids_2d_match_oracle(gpu, oracle_lib, model, m2, kw):
    prm = wl.hpr_two_params(ELASTIC1, m2)
    W = solids(model, ELASTIC1, m2, wl.BARTON_F, BARTON_V, 40, ny=24)
    ref = W.copy()
    O.run_two_material(model, ref, 1 / 40, 0.8, params=prm, **kw)
    out, _, _ = _device(gpu, model, W, prm, 1 / 40, **kw)
    _matches(out, ref)


@pytest.mark.parametrize("model", MODELS, ids=MODEL_IDS)
def test_solids_time_driven(gpu, oracle_lib, model):
    m1, m2, F, v = _godunov_romenski("zhang")
    prm = wl.hpr_two_params(m1, m2)
    W = solids(model, m1, m2, F, v, 80)
    ref = W.copy()
    t_ref, n_ref = O.run_two_material(model, ref, 1 / 80, 0.8, params=prm, t_end=0.01, limiter=O.MINBEE, subcycles=1)
    out, t, n = _device(gpu, model, W, prm, 1 / 80, t_end=0.01, limiter=O.MINBEE, subcycles=1)
    assert t == t_ref == 0.01 and n == n_ref
    _matches(out, ref)


@pytest.mark.parametrize("model", MODELS, ids=MODEL_IDS)
def test_solids_first_order(gpu, oracle_lib, model):
    m1, m2, F, v = _godunov_romenski("barton")
    prm = wl.hpr_two_params(m1, m2)
    W = solids(model, m1, m2, F, v, 50)
    ref = W.copy()
    O.run_first_order(model, ref, 1 / 50, 0.8, steps=8, params=prm)
    out, _, _ = _device(gpu, model, W, prm, 1 / 50, steps=8, order=1)
    _matches(out, ref)


@pytest.mark.parametrize("scenario", ["barton", "zhang", "smg"])
@pytest.mark.parametrize("model", MODELS, ids=MODEL_IDS)
def test_solids_max_wave_speed(gpu, oracle_lib, model, scenario):
    if scenario == "smg":
        m1, m2, F, v = ELASTIC1, PLASTIC2, wl.ZHANG_F, ZHANG_V
    else:
        m1, m2, F, v = _godunov_romenski(scenario)
    prm = wl.hpr_two_params(m1, m2)
    W = solids(model, m1, m2, F, v, 40)
    with gpu.Solver(getattr(gpu, MODEL_ENUM[model]), 40, 1, prm) as s:
        s.upload(W)
        got = s.max_wave_speed()
    want = O.max_wave(model, W, prm)
    assert abs(got - want) <= 1e-12 * want
