"""The C ABI library loads and exports every function include/*.h declares (no GPU needed)."""
import ctypes
import glob
import os
import re

import pytest

import vanguard_b200 as vg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(vg_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = _declared()
    assert {"vg_create", "vg_run", "vg_sweep", "vg_max_wave_speed"} <= names


def test_library_exports_every_declared_symbol():
    L = vg.lib()
    missing = [n for n in sorted(_declared()) if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_lists_every_declared_symbol():
    assert set(vg.EXPORTS) == _declared()


def test_status_strings():
    L = vg.lib()
    assert L.vg_status_string(vg.VG_OK) == b"VG_OK"
    assert L.vg_status_string(vg.VG_EUNSUPPORTED) == b"VG_EUNSUPPORTED"
    assert L.vg_model_nvar(vg.EULER) == 6 and L.vg_model_nvar(vg.MHD) == 9 and L.vg_model_nvar(vg.HPR) == 17
    for model, nvar in vg.NVAR.items():
        assert L.vg_model_nvar(model) == nvar
    assert L.vg_model_nvar(len(vg.NVAR)) == 0


def test_invalid_arguments_are_rejected_on_the_host():
    L = vg.lib()
    h = ctypes.c_void_p()
    assert L.vg_create(None, ctypes.byref(h)) == vg.VG_EINVAL
    d = vg.GridDesc()
    d.model, d.nx, d.ny = vg.EULER, 1, 1
    assert L.vg_create(ctypes.byref(d), ctypes.byref(h)) == vg.VG_EINVAL  # needs >= 2 cells per swept axis
    d.model, d.nx, d.ny = len(vg.NVAR), 16, 16  # the first id past the last model
    assert L.vg_create(ctypes.byref(d), ctypes.byref(h)) == vg.VG_EUNSUPPORTED
    assert L.vg_run(None, None, None, None, None) == vg.VG_EINVAL
    assert L.vg_sweep(None, 0, 1.0, 1.0, 0.0, 0, None) == vg.VG_EINVAL


def test_noalloc_rejects_on_host_without_gpu():
    out = ctypes.c_void_p(8)
    with pytest.raises(vg.VgError) as e:
        vg.max_wave_speed_noalloc(vg.EULER, 16, 4 * 70000, 4, 4, 70000, (1.4, 0.0), 16)
    assert e.value.status == vg.VG_EINVAL
    with pytest.raises(vg.VgError) as e:
        vg.max_wave_speed_noalloc(vg.HPR, 16, 16, 4, 4, 4, (1.4, 0.0), 16)
    assert e.value.status == vg.VG_EUNSUPPORTED
    del out
