"""The replica (N > 1) reduction of bench.py on two gloo ranks on the CPU:
the whole-job time is the slowest rank's, the work is the sum over ranks."""
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=timedelta(seconds=60))
    times, units = bench.combine_ranks([1.0 + rank, 10.0 * (rank + 1)], [100 * (rank + 1), 7], 'cpu', world)
    out.put((rank, times, units))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_take_the_slowest_time_and_the_summed_work():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, times, units in results:
        assert times == [2.0, 20.0]
        assert units == [300.0, 14.0]


def test_one_rank_is_unchanged():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.combine_ranks([1.5], [3], 'cpu', 1) == ([1.5], [3])
