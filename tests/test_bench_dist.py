"""CPU: the bench's multi-rank plumbing with two gloo ranks (the GPU runs use NCCL with the same
code): rendezvous on 127.0.0.1, the barrier, the max over ranks that every timed figure goes
through (the slowest replica sets the whole-job time), and leaving the process group."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import bench
    r, w, _ = bench.dist_setup(2)
    bench.barrier(w)
    slowest = bench.max_over_ranks(10.0 + 5.0 * r, w)
    bench.barrier(w)
    bench.dist_done(w)
    q.put((r, w, slowest))


def test_replica_timing_reductions_with_two_gloo_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank did not finish"
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2, 15.0), (1, 2, 15.0)]


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.dist_setup(1) == (0, 1, 0)
    assert bench.max_over_ranks(3.5, 1) == 3.5
    bench.barrier(1)
    bench.dist_done(1)
