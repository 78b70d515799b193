"""The N > 1 path of bench.py on CPU: two gloo ranks run the same timing protocol as the NCCL ranks of a torchrun
launch (barrier, max over ranks of the device times, whole-job value = all ranks' units / slowest rank), and the
reference arm does no work on ranks other than 0."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


WORKER = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1])
import bench
world, rank, local = bench.dist_setup()
g = bench.RankGroup(world, rank, "gloo", "cpu")
times = [3.0, 7.5, 5.0, 1.0]
g.barrier()
slowest = g.max(times[rank])
e2e = g.max(10.0 * (rank + 1))
value = bench.job_value(world, 1000, slowest)
g.barrier()
g.close()
print(json.dumps({"rank": rank, "world": world, "slowest": slowest, "e2e": e2e, "value": value}), flush=True)
"""


@pytest.mark.parametrize("world", [2, 4])
def test_gloo_ranks_follow_the_timing_protocol(world):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    times = [3.0, 7.5, 5.0, 1.0][:world]
    for o in outs:
        assert o["world"] == world
        assert o["slowest"] == max(times)  # every rank sees the max over ranks
        assert o["e2e"] == 10.0 * world
        assert o["value"] == pytest.approx(world * 1000 / max(times))


def test_job_value_and_single_rank_group():
    sys.path.insert(0, ROOT)
    import bench

    g = bench.RankGroup(1, 0, "gloo", "cpu")  # no process group for one rank
    assert g.dist is None and g.max(2.5) == 2.5
    g.barrier()
    g.close()
    assert bench.job_value(8, 16777216 * 200, 0.25) == pytest.approx(8 * 16777216 * 200 / 0.25)


def test_reference_arm_other_ranks_do_no_work():
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        steps, warmup = 3, 3

    assert bench.run_reference(Args(), 2, 1) == 0  # returns before touching the oracle


def test_dist_setup_reads_torchrun_environment(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("WORLD_SIZE", "4")
    monkeypatch.setenv("RANK", "3")
    monkeypatch.setenv("LOCAL_RANK", "3")
    assert bench.dist_setup() == (4, 3, 3)
