"""The multi-GPU path's host logic on two CPU ranks (gloo, world size 2): each rank draws its own
shard of the n = 8 batch, solves it (the oracle stands in for the device, which this test does
not need), and the job's figures are the sum of solved systems and the maximum of a per-rank
value over ranks — the reductions `bench.py --gpus N` applies to its counts and timings."""

import datetime
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.join(ROOT, "tests")


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, nsys, out):
    for p in (ROOT, TESTS):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import gsb200 as G
        from oracle import oracle_py as O

        X0, P = bench.workload(rank, nsys)
        ranks = bench.Ranks(world, torch.device("cpu"))
        # the shards are different draws
        mine = torch.tensor([float(np.sum(P))], dtype=torch.float64)
        every = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(every, mine)
        plain, _ = bench.methods(G)
        _, so = O.solve_batch(G.NonlinearProblem(G.CubicAffine(8)), plain, X0.copy(), P,
                              bench.options(G))
        solved = ranks.sum(float(np.sum(so["code"] == 0)))
        slowest = ranks.max(float(rank + 1))
        ranks.barrier()
        out.put((rank, [float(c) for c in every], solved, slowest))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, 256, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = [q.get(timeout=180) for _ in range(2)]
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    for _, every, solved, slowest in res:
        assert every[0] != every[1]
        assert solved == 512.0
        assert slowest == 2.0


def test_one_rank_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench

    r = bench.Ranks(1)
    assert r.max(3.5) == 3.5 and r.sum(7.0) == 7.0
    r.barrier()


def _bench_line(*args):
    import json
    import subprocess

    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], env=env,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_bench_starts_its_own_ranks():
    """`bench.py --gpus 2` with no launcher around it starts two ranks under torch.distributed.run;
    their collectives (barrier, maximum, sum) run over gloo, and rank 0 alone prints the world
    size it saw."""
    line = _bench_line("--gpus", "2", "--launch-check")
    assert line["n_gpus"] == 2 and line["max_rank"] == 1.0 and line["ranks_counted"] == 2.0


def test_reference_arm_reports_the_world_size():
    line = _bench_line("--gpus", "2", "--impl", "reference", "--steps", "1", "--warmup", "0",
                       "--nsys", "2048")
    assert line["impl"] == "reference" and line["n_gpus"] == 2
