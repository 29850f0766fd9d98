"""Multi-rank host logic of bench.py on CPU: two gloo ranks take the max of
their timings, pass the barrier, and reconstruct different scans (one replica
per GPU, no data-path collective)."""

import datetime
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.ranks_max(10.0 + 2.5 * rank, "cpu")
        bench.barrier(world)
        q.put((rank, ms, bench.replica_seed(bench.CFG["seed"], rank)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_and_distinct_scans():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    got = sorted(q.get(timeout=5) for _ in range(world))
    assert [g[1] for g in got] == [12.5, 12.5]
    assert got[0][2] != got[1][2]


def test_barrier_is_a_no_op_for_one_rank():
    sys.path.insert(0, ROOT)
    import bench
    bench.barrier(1)
    assert bench.replica_seed(5, 0) == 5
