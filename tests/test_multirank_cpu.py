"""The N>1 path of bench.py on CPU: two gloo ranks (replicas) reduce their
timings to the max over ranks and report the whole-job aggregate.  Also a
rank that dies is noticed by the survivor through a short process-group
timeout instead of a hang."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    import bench
    ms = [12.5, 20.0][rank]
    total = bench.reduce_max(ms, dist, "cpu")
    out[rank] = (total, bench.aggregate_gbs(4_000_000_000, 10, world, total))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_max_reduction():
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    assert res[0][0] == res[1][0] == 20.0
    # 2 ranks x 10 steps x 4 GB in 20 ms
    assert abs(res[0][1] - 2 * 10 * 4.0 / 0.020) < 1e-6


def _dying_worker(rank, world, port, out):
    import datetime
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        os._exit(0)  # leaves between steps without telling anyone
    import bench
    try:
        bench.reduce_max(1.0, dist, "cpu")
        out[rank] = "returned"
    except Exception as e:  # the collective ends with an error after the timeout
        out[rank] = "error:" + type(e).__name__


def test_dead_rank_is_detected_by_timeout():
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        ctx = mp.start_processes(_dying_worker, args=(2, port, out), nprocs=2, join=False, start_method="spawn")
        for p in ctx.processes:
            p.join(timeout=120)
        for p in ctx.processes:
            if p.is_alive():
                p.kill()
                pytest.fail("a rank hung instead of timing out")
        res = dict(out)
    assert res.get(0, "").startswith("error:")
