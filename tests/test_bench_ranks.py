"""The N > 1 host logic of bench.py on CPU: two gloo ranks reduce their
timings to the maximum (the number rank 0 reports), and under torchrun only
rank 0 runs the reference arm while the other ranks exit 0 without output."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import datetime, json, os, sys
sys.path.insert(0, os.environ["BENCH_ROOT"])
import torch.distributed as dist
import bench
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
r = dist.get_rank()
out = [bench.max_over_ranks(1.5 + r, dist, device="cpu"),
       bench.max_over_ranks(10.0 - r, dist, device="cpu"),
       bench.max_over_ranks(3.0, None)]
dist.barrier()
dist.destroy_process_group()
print(json.dumps({"rank": r, "out": out}))
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_two_gloo_ranks():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(r),
                   WORLD_SIZE="2", LOCAL_RANK=str(r), BENCH_ROOT=ROOT)
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    results = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        results.append(json.loads(out.strip().splitlines()[-1]))
    for res in results:
        assert res["out"] == [2.5, 10.0, 3.0]


def test_reference_arm_non_zero_rank_exits_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
