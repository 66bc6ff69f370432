"""The multi-GPU path of bench.py is N independent replicas (one process per
GPU, no data-path collective): ranks meet at barriers and the timed region
is the slowest rank's. Checked here with world_size 2 on gloo, on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q) -> None:
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    d = bench.Dist()
    d.init("gloo")
    d.barrier()
    slowest = d.max(1.0 + rank)          # rank 1 was the slower one
    units = 100.0
    value = bench.replica_throughput(d.world, units, slowest)
    d.barrier()
    d.close()
    q.put((rank, d.world, slowest, value))


def test_two_replicas_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, world, slowest, value in out:
        assert world == 2 and slowest == 2.0
        assert value == pytest.approx(2 * 100.0 / 2.0)


def test_single_process_needs_no_group():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    d.init("gloo")          # world 1: no process group
    assert d.pg is None and d.max(3.5) == 3.5
    assert bench.replica_throughput(1, 10.0, 2.0) == 5.0
