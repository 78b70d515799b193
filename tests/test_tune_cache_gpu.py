"""The autotuner's on-disk cache (VG_TUNE_CACHE): a tuned choice -- X shape, Y shape, Y segment mode and schedule --
is written as one line and applied without timing by a later process (each process reads the file once)."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SCRIPT = """
import sys
import vanguard_b200 as vg
from vanguard_b200 import workloads as wl
n = 512
with vg.Solver(vg.MHD, n, n, wl.mhd_params(), precision=vg.MIXED, boundary=vg.PERIODIC) as s:
    s.upload(wl.mhd_vortex_2d(n, seed=3))
    s.autotune(1.0 / n, 0.8, limiter=0, measure=sys.argv[1] == "tune")
    x, y, xn, yn = s.launch_config()
    print(x, y, s.schedule())
"""


def _run(mode, cache):
    env = dict(os.environ, VG_TUNE_CACHE=str(cache), PYTHONPATH=os.path.dirname(HERE))
    out = subprocess.run([sys.executable, "-c", SCRIPT, mode], env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    return out.stdout.split()


def test_tuned_choice_is_cached_on_disk(tmp_path):
    cache = tmp_path / "tune.txt"
    tuned = _run("tune", cache)
    lines = cache.read_text().split("\n")
    fields = [ln.split() for ln in lines if ln.strip()]
    assert len(fields) == 1 and len(fields[0]) == 5  # key, X shape, Y shape, schedule, Y segment mode
    key, x, y, sched, yseg = fields[0]
    assert [x, y, sched] == tuned and yseg in ("0", "1")
    assert _run("apply", cache) == tuned
