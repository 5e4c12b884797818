"""The multi-GPU path's host side on CPU ranks (gloo, world size 2): each rank steps a fleet of its own (weak
scaling: islands are independent, so no data-path collective), the job's time is the slowest rank's and its work
every rank's nodes (bench.aggregate); the reference arm runs on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


WORKER = r"""
import json, os, sys
from datetime import timedelta
sys.path.insert(0, os.environ["BL_ROOT"])
import torch.distributed as dist
import bench
ws, rank, _ = bench.dist_setup()
dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
rig, n, m, desc = bench.workload("truss_car", rank)
ms, ms_e2e, total = bench.aggregate(10.0 + 5.0 * rank, 30.0 - 5.0 * rank, n * (rank + 1), ws, "cpu")
first = [float(x) for x in rig["bodies"][0]["pos"][0]]
print(json.dumps({"rank": rank, "ms": ms, "ms_e2e": ms_e2e, "total": total, "n": n, "first": first}), flush=True)
dist.destroy_process_group()
"""


def _run_ranks(code: str, ws: int = 2, extra=None):
    port = _free_port()
    procs = []
    for r in range(ws):
        env = dict(os.environ, BL_ROOT=ROOT, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(r), WORLD_SIZE=str(ws),
                   LOCAL_RANK=str(r), **(extra or {}))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True, cwd=ROOT))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    return outs


def test_two_ranks_aggregate_max_time_and_sum_of_nodes():
    outs = [json.loads(o.strip().splitlines()[-1]) for o in _run_ranks(WORKER)]
    a, b = sorted(outs, key=lambda d: d["rank"])
    for d in (a, b):
        assert d["ms"] == 15.0 and d["ms_e2e"] == 30.0  # (the slowest rank's)
        assert d["total"] == a["n"] * 1 + b["n"] * 2    # (every rank's nodes)
    assert a["first"] != b["first"]                      # (each rank its own seeded rig)


def test_reference_arm_runs_on_rank_zero_only():
    """bench.py --impl reference under two ranks: rank 0 prints the line, rank 1 exits 0 without work."""
    code = ("import os, sys; sys.path.insert(0, os.environ['BL_ROOT']); sys.argv = ['bench.py', '--impl', 'reference', "
            "'--gpus', '2', '--steps', '1', '--warmup', '3', '--workload', 'truss_car']; import bench; bench.main()")
    outs = _run_ranks(code)
    lines = [[ln for ln in o.strip().splitlines() if ln.startswith("{")] for o in outs]
    assert len(lines[1]) == 0
    rec = json.loads(lines[0][-1])
    assert rec["impl"] == "reference" and ("value" in rec or "unavailable" in rec)
