"""The multi-GPU plumbing of bench.py -- one process per GPU, no data-path
collective, timing as the max over ranks, throughput summed over replicas --
run as two gloo ranks on the CPU (the path has no exchange step, so the
ranks only meet at barriers and the timing reduction)."""
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


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    r, w, local = bench.init_dist(None, backend="gloo")
    try:
        bench.barrier(w)
        ms = 10.0 + 5.0 * r  # the slower rank decides the job's time
        worst = bench.max_over_ranks(ms, w)
        bench.barrier(w)
        out.put((r, w, worst, bench.replica_throughput(1_000_000, worst, w)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_replicas_time_is_max_over_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=10) for _ in range(world))
    for r, w, worst, thr in res:
        assert w == world
        assert worst == 10.0 + 5.0 * (world - 1)
        assert thr == pytest.approx(world * 1_000_000 / (worst * 1e-3))
