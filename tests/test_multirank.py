"""The benchmark's multi-process plumbing on CPU: two gloo ranks (one process
per GPU on a B200 node, NCCL there) agree on the slowest rank's time and the
summed work, and their replicas' instances are disjoint."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    dist, r, w = bench.dist_init()
    assert (r, w) == (rank, world) and dist.get_backend() == "gloo"
    slowest = bench.max_over_ranks(10.0 + rank, dist)
    work = bench.sum_over_ranks(100.0 * (rank + 1), dist)
    seeds = bench.instance_seeds(4, rank)
    everyone = [None] * world
    dist.all_gather_object(everyone, seeds)
    dist.destroy_process_group()
    out.put((rank, slowest, work, everyone))


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, work, everyone in res:
        assert slowest == 11.0
        assert work == 300.0
        flat = [s for rs in everyone for s in rs]
        assert len(flat) == len(set(flat)) == 8


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun every rank starts the reference arm; ranks other than 0
    return at once, with no output and no work."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        scheme, steps, warmup = "ark23", 1, 3

    assert bench.run_reference(Args()) == 0
    assert capsys.readouterr().out == ""
