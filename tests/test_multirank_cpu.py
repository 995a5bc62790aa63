"""The multi-rank path of bench.py on the CPU (gloo, world size 2): the
max-over-ranks reduction of the step time, per-rank independent subdomains, and
the reference arm under torchrun printing one line from rank 0 only."""
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


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = bench.reduce_max(10.0 + 5.0 * rank, dist, "cpu")
    seed = bench.subdomain_seed(rank)
    dist.destroy_process_group()
    with open(os.path.join(out, f"r{rank}.json"), "w") as f:
        json.dump({"max": t, "seed": seed}, f)


def test_reduce_max_and_rank_seeds(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    r = [json.load(open(tmp_path / f"r{q}.json")) for q in range(2)]
    assert r[0]["max"] == r[1]["max"] == 15.0
    assert r[0]["seed"] != r[1]["seed"]


def test_reference_arm_under_torchrun_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference", "--workload", "cpu64",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--cpu-sample-iters", "2"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    j = json.loads(lines[0])
    assert j["impl"] == "reference" and j["value"] > 0 and j["cpu_baseline"]["kind"] == "port"
