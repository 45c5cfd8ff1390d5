"""Multi-GPU runs are replicas only: each rank sweeps its own copy and the process
group carries only the barrier and the max-over-ranks of the timings.  The
plumbing of bench.py, exercised here with two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    dist, r, w, local = bench.dist_init(backend="gloo")
    assert (r, w) == (rank, world)
    bench.barrier(dist, cuda=False)
    # each replica's "step time"; the job's time is the slowest one
    got = bench.max_over_ranks(dist, 10.0 + 5.0 * rank, device="cpu")
    out.put((rank, got))
    bench.barrier(dist, cuda=False)
    dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(world))
    assert res == {0: 15.0, 1: 15.0}


def test_reference_arm_other_ranks_do_no_work(monkeypatch):
    """Under torchrun only rank 0 runs the CPU reference arm; the others return at once."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        steps, warmup = 1, 1
    assert bench.run_reference(A()) is None
