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


def _decomposed_worker(rank, world, port, px, py, out):
    """One gloo rank of the decomposed BiCGStab (hicar_b200.decomp.rank_schedule
    driven by run_distributed over torch.distributed) on the numpy stand-in of
    the library's rank primitives (tests/dist_ref.py)."""
    import numpy as np
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import dist_ref
    from hicar_b200 import cases, decomp
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    case = cases.build_case(40, 36, 12, seed=3, adv_den=True, n_hills=5)
    s = O.OracleSolver(case.domain)
    s.set_alpha(case.alpha)
    u, v, w = (np.ascontiguousarray(a).copy() for a in (case.u, case.v, case.w))
    s.build_analytic(case.alpha)
    s.calibrate(True, u, v, w)
    div = s.divergence(case.u, case.v, case.w)
    s.prepare(div)
    coefs, rhs = s.coefs(), s.vec("rhs")
    dec = decomp.Decomposition(40, 36, px, py)
    r = dist_ref.NumpyRank(dec.interior(rank, coefs), dec.edges(rank), tol_rel=1e-10, max_iters=3000)
    st = decomp.run_distributed(decomp.rank_schedule(r, dec.neighbors(rank), dec.local(rank, rhs).copy(), 3000),
                                dec, rank, dist)
    parts = [None] * world
    dist.all_gather_object(parts, (rank, r.lam()[1:-1, 1:-1, 1:-1].copy(), st))
    dist.destroy_process_group()
    if rank == 0:
        lam = np.zeros((36, 12, 40))
        for q, part, _ in parts:
            i0, i1, j0, j1 = dec.block(q)
            lam[j0 - 1:j1, :, i0 - 1:i1] = part
        s.set_vec("x", np.zeros((38, 14, 42)))
        s.set_tolerance(1e-10)
        ref = s.bicgstab(3000)
        lam_ref = s.vec("x")[1:-1, 1:-1, 1:-1]
        err = float(np.linalg.norm(lam - lam_ref) / np.linalg.norm(lam_ref))
        with open(os.path.join(out, "decomp.json"), "w") as f:
            json.dump({"err": err, "stats": [p[2] for p in parts], "ref_iters": ref["iters"]}, f)


@pytest.mark.parametrize("px,py", [(2, 1), (2, 2)])
def test_decomposed_solve_on_gloo_ranks(tmp_path, px, py):
    """The reference's multi-rank BiCGStab (halo exchange of p^ and s^, FP64
    allreduce of 3, 1 and 5 values, block Jacobi-Richardson with a zero halo),
    run as 2 and 4 gloo ranks with the schedule of hicar_b200.decomp: every
    rank ends with the same status and iteration count, and the assembled
    lambda equals the one-rank solve to 1e-7."""
    import torch.multiprocessing as mp
    port = _free_port()
    world = px * py
    mp.start_processes(_decomposed_worker, args=(world, port, px, py, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    res = json.load(open(tmp_path / "decomp.json"))
    stats = res["stats"]
    assert all(st["status"] == 0 for st in stats), stats
    assert len({st["iterations"] for st in stats}) == 1
    assert res["err"] < 1e-7, res
