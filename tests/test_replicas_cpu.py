"""The N>1 path of bench.py on CPU: two gloo ranks (127.0.0.1).

bench.py runs one independent lattice per GPU (replicas only, no collective
on the data path) and reduces only the timing: a barrier around the timed
region and the max of the per-rank elapsed times, so the whole-job rate is
N * work / max(time). The reference arm under torchrun runs on rank 0 only.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import json, os, sys, time
sys.path.insert(0, {root!r})
import bench
d = bench.Dist()
d.init("gloo")
t0 = time.perf_counter()
time.sleep(0.05 * (d.rank + 1))          # rank-dependent work
d.barrier()
mine = 1.0 + d.rank                       # per-rank elapsed "seconds"
mx = d.max(mine)
total = d.sum(100.0)                      # units processed, all ranks
print(json.dumps({{"rank": d.rank, "world": d.world, "max": mx, "sum": total}}), flush=True)
d.close()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _launch(code: str, nproc: int = 2, extra_env=None, args=()):
    port = _free_port()
    procs = []
    for r in range(nproc):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(nproc), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, "-c", code, *args], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=120)
        assert p.returncode == 0, e
        outs.append(o)
    return outs


def test_two_rank_timing_is_max_over_ranks():
    outs = _launch(WORKER.format(root=ROOT))
    res = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert {r["rank"] for r in res} == {0, 1}
    for r in res:
        assert r["world"] == 2
        assert r["max"] == 2.0          # max over ranks, seen identically by all
        assert r["sum"] == 200.0


def test_reference_arm_runs_on_rank_zero_only():
    code = (f"import sys; sys.path.insert(0, {ROOT!r}); import bench; sys.argv = ['bench.py', '--impl', "
            "'reference', '--gpus', '2', '--steps', '1', '--warmup', '0']; "
            "import unittest.mock as m\n"
            "with m.patch.object(bench, 'cpu_reference_time', return_value=(0.5, 0.6, 1, 2, 'reference')), "
            "m.patch.object(bench, 'host_fields', return_value=(None, None)):\n"
            "    sys.exit(bench.main())")
    outs = _launch(code)
    lines = [o.strip() for o in outs]
    assert lines[1] == ""                      # rank 1 prints nothing and exits 0
    rec = json.loads(lines[0].splitlines()[-1])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2
    assert rec["e2e"]["h2d_bytes_per_step"] == 0 and rec["cpu_baseline"]["kind"] == "reference"
    V = 32 * 32 * 32 * 64
    assert abs(rec["value"] - V * 1320 / 0.5 / 1e9) < 1e-3
