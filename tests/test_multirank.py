"""The multi-GPU bench path on CPU: two gloo ranks.

Each rank runs whole cases of its own seeded sweep (no data exchange); the job's
throughput is the cells of all ranks over the slowest rank's time. The ranks here
stand in for GPUs: they run the bench's own rank functions (draws per rank, the
SUM/MAX reductions) over a gloo process group on 127.0.0.1.
"""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    draws = bench.rank_draws(16, rank)
    cells = sum(d["N"] * d["N"] for d in draws)
    ms = 100.0 + 25.0 * rank  # rank 1 is the slow one
    job_cells, ms_max = bench.job_totals(dist, "cpu", cells, ms, world)
    out.put((rank, [d["N"] for d in draws], [round(d["Re"], 9) for d in draws], cells, job_cells, ms_max))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_whole_cases_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, n0, re0, c0, j0, m0), (r1, n1, re1, c1, j1, m1) = res
    assert (r0, r1) == (0, 1)
    assert re0 != re1                      # different seeds: each rank has its own cases
    assert j0 == j1 == c0 + c1             # cells summed over ranks
    assert m0 == m1 == 125.0               # time = the slowest rank
    # rank 0's cases are the single-GPU sweep's first 16 draws
    sys.path.insert(0, str(ROOT))
    from cfd_solver_b200.workloads import SWEEP_SEED, sweep_draws
    assert n0 == [d["N"] for d in sweep_draws(16, seed=SWEEP_SEED)]
