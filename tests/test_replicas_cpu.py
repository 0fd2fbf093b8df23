"""The N > 1 path of bench.py on CPU: two gloo ranks share the barrier and
the max-over-ranks time the GPU run takes over NCCL, the whole-job rate
counts every replica's units against the slowest rank, and the reference
arm runs on rank 0 only (the others exit 0 without output)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, json, time
sys.path.insert(0, os.environ["BENCH_ROOT"])
import torch.distributed as dist
from datetime import timedelta
import bench
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", timeout=timedelta(seconds=60))
r = bench.Ranks(world, "cpu")
t_local = 1.0 + rank          # rank 1 is the slower one
r.barrier()
t = r.max(t_local)
value = bench.whole_job_rate(world, 10, 1000.0, t)
r.barrier()
if rank == 0:
    print(json.dumps({"t": t, "value": value}), flush=True)
dist.destroy_process_group()
"""


def _launch(tmp_path, script, world=2, port=29571, extra_env=None):
    path = tmp_path / "worker.py"
    path.write_text(script)
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), BENCH_ROOT=ROOT, **(extra_env or {}))
        procs.append(subprocess.Popen([sys.executable, str(path)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    return [(p.returncode, o, e) for p, (o, e) in zip(procs, outs)]


def test_two_gloo_ranks_share_barrier_and_max(tmp_path):
    res = _launch(tmp_path, WORKER)
    for rc, _, err in res:
        assert rc == 0, err
    line = json.loads(res[0][1].strip().splitlines()[-1])
    assert line["t"] == 2.0  # the slower rank's time
    assert line["value"] == 2 * 10 * 1000.0 / 2.0  # both replicas' units
    assert res[1][1].strip() == ""  # only rank 0 prints


def test_reference_arm_runs_on_rank_zero_only(tmp_path):
    script = r"""
import os, sys
sys.path.insert(0, os.environ["BENCH_ROOT"])
import bench
class A:  # the parsed arguments run_reference reads
    steps, warmup, gpus = 1, 0, 2
sys.exit(bench.run_reference(A(), int(os.environ["RANK"])) if os.environ["RANK"] != "0" else 0)
"""
    res = _launch(tmp_path, script, port=29572)
    assert all(rc == 0 for rc, _, _ in res)
    assert res[1][1].strip() == ""


def test_single_rank_is_a_no_op():
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks(1, "cpu")
    r.barrier()
    assert r.max(3.5) == 3.5
    assert bench.whole_job_rate(1, 4, 10.0, 2.0) == 20.0
