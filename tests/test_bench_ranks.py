"""The multi-rank steps of bench.py on CPU: two `gloo` ranks take the max of their
step times and report the whole-job rate; non-zero ranks of the reference arm exit
without work or output."""

import json
import os
import socket
import subprocess
import sys

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import datetime, json, os, sys
sys.path.insert(0, os.environ["PFB_ROOT"])
import torch.distributed as dist
import bench
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
r = dist.get_rank()
ms = bench.max_over_ranks(10.0 + 5.0 * r, dist.get_world_size(), "cpu")
print(json.dumps({"rank": r, "ms": ms, "rate": bench.whole_job_rate(dist.get_world_size(), 1000, ms)}))
dist.barrier()
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_whole_job_rate_and_single_rank():
    assert bench.whole_job_rate(1, 8_000_000, 40.0) == 2e8
    assert bench.whole_job_rate(4, 8_000_000, 40.0) == 8e8
    assert bench.max_over_ranks(12.5, 1, "cpu") == 12.5


def test_max_over_two_gloo_ranks():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(r), WORLD_SIZE="2",
                   LOCAL_RANK=str(r), PFB_ROOT=ROOT)
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    try:
        for p in procs:
            out, err = p.communicate(timeout=180)
            assert p.returncode == 0, err[-2000:]
            outs.append(json.loads(out.strip().splitlines()[-1]))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    assert sorted(o["rank"] for o in outs) == [0, 1]
    for o in outs:
        assert o["ms"] == 15.0  # the slower rank's time on every rank
        assert o["rate"] == 2 * 1000 / 0.015


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
