"""bench.py's N > 1 replica logic on the CPU: two gloo ranks launched like the
driver's torchrun (RANK, WORLD_SIZE, MASTER_ADDR = 127.0.0.1).  The timed
region's length is the max over ranks, the value every rank's work over that
time, and the reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import bench
ws, rank, local = bench.dist_init()
m = bench.reduce_max(10.0 + rank, ws)
bench.barrier(ws)
v = bench.replica_value(1e6, m, 4, ws)
print(json.dumps(dict(rank=rank, ws=ws, max=m, value=v)), flush=True)
import torch.distributed as dist
dist.destroy_process_group()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _launch(code, ws=2, timeout=120):
    port = _free_port()
    procs = []
    for r in range(ws):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(ws), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=timeout)
        assert p.returncode == 0, e[-2000:]
        outs.append(o)
    return outs


def test_replicas_max_over_ranks():
    outs = _launch(CHILD.format(root=ROOT))
    recs = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert {r["rank"] for r in recs} == {0, 1}
    for r in recs:
        assert r["ws"] == 2 and r["max"] == 11.0
        assert r["value"] == pytest.approx(1e6 * 4 * 2 / 11e-3)


def test_reference_arm_rank1_exits_quietly():
    code = r"""
import sys, types
sys.path.insert(0, {root!r})
import bench
ws, rank, local = bench.dist_init()
args = types.SimpleNamespace(workload="weibel2d", steps=1, warmup=0, gpus=ws)
if rank == 1:
    rc = bench.run_reference_arm(args, ws, rank)
    print("rc", rc)
bench.barrier(ws)
import torch.distributed as dist
dist.destroy_process_group()
""".format(root=ROOT)
    outs = _launch(code)
    assert outs[1].strip().endswith("rc 0")
    assert outs[0].strip() == ""
