"""Multi-GPU runs are replicas (independent systems per rank, no data-path
collective): the only cross-rank steps are the whole-job totals of the
bench line (max of the ranks' times, sum of their rods) and the rank
filtering of the reference arm.  Checked here on CPU with world size 2 over
gloo, ranks as child processes."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import datetime, json, os, sys
sys.path.insert(0, os.environ["REPO_ROOT"])
import torch.distributed as dist
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
import bench
rank = dist.get_rank()
ms, rods = bench.job_totals(10.0 + rank, 1000 * (rank + 1), True, device="cpu")
e2e_s, _ = bench.job_totals(0.5 * (rank + 1), 1000 * (rank + 1), True, device="cpu")
print(json.dumps({"rank": rank, "ms": ms, "rods": rods, "e2e_s": e2e_s}))
dist.barrier()
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_job_totals_over_two_gloo_ranks():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                   REPO_ROOT=ROOT)
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["ms"] == 11.0      # the slowest rank's time
        assert o["rods"] == 3000    # rods of both replicas
        assert o["e2e_s"] == 1.0


def test_single_rank_totals_are_the_rank_own():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_totals(12.5, 777, False) == (12.5, 777)


def test_reference_arm_prints_only_on_rank_zero():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
